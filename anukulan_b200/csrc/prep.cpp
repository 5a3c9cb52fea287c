// Host-side preparation: CSR copy/validation, transpose, diagonal scaling and
// the row-block schedule of the staged SpMV.
#include "prep.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>

namespace anu {

double now_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

std::string validate_csr(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                         const int32_t* index) {
  if (rows < 0 || cols < 0 || nnz < 0) return "negative dimensions";
  if (rows > 0 && start == nullptr) return "null row starts";
  if (nnz > 0 && index == nullptr) return "null column indices";
  if (start != nullptr) {
    if (start[0] != 0) return "start does not begin at 0";
    if (start[rows] != nnz) return "start does not end at nnz";
    for (int32_t r = 0; r < rows; ++r)
      if (start[r + 1] < start[r]) return "start is not monotone at row " + std::to_string(r);
  }
  for (int32_t k = 0; k < nnz; ++k)
    if (index[k] < 0 || index[k] >= cols) return "column index out of range";
  return "";
}

HostCsr copy_csr(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                 const int32_t* index, const double* value) {
  HostCsr a;
  a.rows = rows;
  a.cols = cols;
  a.start.assign(start, start + rows + 1);
  a.index.assign(index, index + nnz);
  a.value.assign(value, value + nnz);
  return a;
}

HostCsr transpose(const HostCsr& a) { return transpose(a, nullptr); }

HostCsr transpose(const HostCsr& a, std::vector<int32_t>* pos) {
  HostCsr t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.start.assign(static_cast<std::size_t>(a.cols) + 1, 0);
  t.index.resize(a.index.size());
  t.value.resize(a.value.size());
  for (const int32_t c : a.index) t.start[static_cast<std::size_t>(c) + 1]++;
  for (std::size_t i = 1; i < t.start.size(); ++i) t.start[i] += t.start[i - 1];
  std::vector<int32_t> cursor(t.start.begin(), t.start.end() - 1);
  if (pos != nullptr) pos->resize(a.index.size());
  for (int32_t r = 0; r < a.rows; ++r) {
    for (int32_t k = a.start[r]; k < a.start[r + 1]; ++k) {
      const int32_t dest = cursor[a.index[k]]++;
      t.index[dest] = r;
      t.value[dest] = a.value[k];
      if (pos != nullptr) (*pos)[dest] = k;
    }
  }
  return t;
}

void multiply(const HostCsr& a, const double* x, double* y) {
  for (int32_t r = 0; r < a.rows; ++r) {
    double sum = 0.0;
    for (int32_t k = a.start[r]; k < a.start[r + 1]; ++k) sum += a.value[k] * x[a.index[k]];
    y[r] = sum;
  }
}

namespace {

void row_norms(const HostCsr& a, bool one_norm, std::vector<double>* out) {
  out->assign(static_cast<std::size_t>(a.rows), 0.0);
  for (int32_t r = 0; r < a.rows; ++r) {
    double acc = 0.0;
    for (int32_t k = a.start[r]; k < a.start[r + 1]; ++k) {
      const double v = std::fabs(a.value[k]);
      acc = one_norm ? acc + v : std::fmax(acc, v);
    }
    (*out)[r] = acc;
  }
}

void col_norms(const HostCsr& a, bool one_norm, std::vector<double>* out) {
  out->assign(static_cast<std::size_t>(a.cols), 0.0);
  for (std::size_t k = 0; k < a.value.size(); ++k) {
    const double v = std::fabs(a.value[k]);
    double& acc = (*out)[a.index[k]];
    acc = one_norm ? acc + v : std::fmax(acc, v);
  }
}

double spread(const std::vector<double>& norms) {
  double lo = kInf, hi = 0.0;
  for (const double v : norms) {
    if (v <= 0.0) continue;
    lo = std::fmin(lo, v);
    hi = std::fmax(hi, v);
  }
  return hi == 0.0 ? 1.0 : hi / lo;
}

}  // namespace

double norm_spread(const std::vector<double>& norms) { return spread(norms); }

Scaling scale_matrix_sweeps(HostCsr* k, int ruiz_iterations, bool pock_chambolle,
                            ScalingSweeps* sweeps) {
  Scaling s;
  s.row_scale.assign(static_cast<std::size_t>(k->rows), 1.0);
  s.col_scale.assign(static_cast<std::size_t>(k->cols), 1.0);
  std::vector<double> rn, cn;
  row_norms(*k, false, &rn);
  col_norms(*k, false, &cn);
  s.row_spread_before = spread(rn);
  s.col_spread_before = spread(cn);
  const int total = ruiz_iterations + (pock_chambolle ? 1 : 0);
  sweeps->d1.clear();
  sweeps->d2.clear();
  for (int sweep = 0; sweep < total; ++sweep) {
    const bool one = sweep >= ruiz_iterations;
    row_norms(*k, one, &rn);
    col_norms(*k, one, &cn);
    std::vector<double> d1(rn.size()), d2(cn.size());
    for (std::size_t i = 0; i < rn.size(); ++i) d1[i] = rn[i] > 0.0 ? 1.0 / std::sqrt(rn[i]) : 1.0;
    for (std::size_t j = 0; j < cn.size(); ++j) d2[j] = cn[j] > 0.0 ? 1.0 / std::sqrt(cn[j]) : 1.0;
    for (int32_t r = 0; r < k->rows; ++r)
      for (int32_t e = k->start[r]; e < k->start[r + 1]; ++e) k->value[e] *= d1[r];
    for (std::size_t e = 0; e < k->value.size(); ++e) k->value[e] *= d2[k->index[e]];
    for (std::size_t i = 0; i < d1.size(); ++i) s.row_scale[i] *= d1[i];
    for (std::size_t j = 0; j < d2.size(); ++j) s.col_scale[j] *= d2[j];
    sweeps->d1.push_back(std::move(d1));
    sweeps->d2.push_back(std::move(d2));
  }
  row_norms(*k, false, &rn);
  col_norms(*k, false, &cn);
  s.row_spread_after = spread(rn);
  s.col_spread_after = spread(cn);
  return s;
}

void scale_vectors(const ScalingSweeps& sw, int32_t m, int32_t n, double* c, double* q,
                   double* lower, double* upper) {
  for (std::size_t s = 0; s < sw.d1.size(); ++s) {
    const std::vector<double>& d1 = sw.d1[s];
    const std::vector<double>& d2 = sw.d2[s];
    for (int32_t i = 0; i < m; ++i) q[i] *= d1[i];
    for (int32_t j = 0; j < n; ++j) {
      c[j] *= d2[j];
      lower[j] /= d2[j];
      upper[j] /= d2[j];
    }
  }
}

std::vector<RowBlock> row_blocks(const HostCsr& a, int32_t block_nnz, int32_t block_rows,
                                 int32_t long_row) {
  std::vector<RowBlock> blocks;
  int32_t r = 0;
  while (r < a.rows) {
    const int32_t len = a.start[r + 1] - a.start[r];
    if (len > long_row || len > block_nnz) {
      blocks.push_back({r, r + 1});
      ++r;
      continue;
    }
    const int32_t r0 = r;
    int32_t nnz = 0;
    while (r < a.rows && r - r0 < block_rows) {
      const int32_t l = a.start[r + 1] - a.start[r];
      if (l > long_row || l > block_nnz || nnz + l > block_nnz) break;
      nnz += l;
      ++r;
    }
    blocks.push_back({r0, r});
  }
  // Longest blocks first: a block of one long row runs longest, so starting it
  // in the first wave keeps it off the tail.
  std::stable_sort(blocks.begin(), blocks.end(), [&](const RowBlock& x, const RowBlock& y) {
    const int32_t nx = a.start[x.row_end] - a.start[x.row_begin];
    const int32_t ny = a.start[y.row_end] - a.start[y.row_begin];
    const bool lx = nx > block_nnz || (x.row_end - x.row_begin == 1 && nx > long_row);
    const bool ly = ny > block_nnz || (y.row_end - y.row_begin == 1 && ny > long_row);
    if (lx != ly) return lx;
    if (lx) return nx > ny;
    return false;
  });
  return blocks;
}

SegmentSchedule segment_schedule(const HostCsr& a, int32_t seg_nnz, int32_t seg_per_cta,
                                 int32_t row_max) {
  SegmentSchedule s;
  s.row_seg.assign(static_cast<size_t>(a.rows) + 1, 0);
  for (int32_t r = 0; r < a.rows; ++r) {
    const int32_t b = a.start[r], e = a.start[r + 1];
    const int32_t len = e - b;
    int32_t step = seg_nnz;
    if (len > seg_nnz * seg_per_cta) step = (len + seg_per_cta - 1) / seg_per_cta;
    s.row_seg[r] = static_cast<int32_t>(s.seg_begin.size());
    for (int32_t k = b; k < e; k += step) s.seg_begin.push_back(k);
  }
  s.row_seg[a.rows] = static_cast<int32_t>(s.seg_begin.size());
  s.seg_begin.push_back(a.nnz());
  s.cta_row.push_back(0);
  s.cta_seg.push_back(0);
  int32_t r = 0;
  while (r < a.rows) {
    const int32_t r0 = r;
    int32_t count = 0;
    while (r < a.rows && r - r0 < row_max) {
      const int32_t c = s.row_seg[r + 1] - s.row_seg[r];
      if (count + c > seg_per_cta && r > r0) break;
      count += c;
      ++r;
    }
    s.cta_row.push_back(r);
    s.cta_seg.push_back(s.row_seg[r]);
  }
  return s;
}

ClusterSchedule cluster_schedule(const HostCsr& a, int32_t parts, int32_t serial_row) {
  ClusterSchedule c;
  c.bounds.assign(static_cast<size_t>(parts) + 1, a.rows);
  c.bounds[0] = 0;
  const int64_t total = a.nnz();
  int32_t part = 1;
  for (int32_t r = 0; r < a.rows && part < parts; ++r) {
    // Part `part` starts at the first row whose nonzeros begin at or past
    // its share; a row never splits.
    while (part < parts && static_cast<int64_t>(a.start[r]) * parts >= total * part)
      c.bounds[part++] = r;
  }
  c.warp_start.assign(static_cast<size_t>(parts) + 1, 0);
  for (int32_t q = 0; q < parts; ++q) {
    for (int32_t r = c.bounds[q]; r < c.bounds[q + 1]; ++r) {
      const int32_t len = a.start[r + 1] - a.start[r];
      c.max_row = std::max(c.max_row, len);
      if (len > serial_row) c.warp_rows.push_back(r);
    }
    c.warp_start[q + 1] = static_cast<int32_t>(c.warp_rows.size());
    c.max_part_rows = std::max(c.max_part_rows, c.bounds[q + 1] - c.bounds[q]);
    c.max_part_nnz = std::max(c.max_part_nnz, a.start[c.bounds[q + 1]] - a.start[c.bounds[q]]);
  }
  return c;
}

}  // namespace anu
