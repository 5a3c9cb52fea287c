// Diagonal scaling of the matrix on the device: the restatement of scale_lp
// (src/anukulan/scaling.cpp:32-100) that scale_matrix_sweeps runs on the
// host, with the same arithmetic in the same order, so the scaled matrix and
// every factor are bit-identical to the host's.
//
//   - Row norms: one thread per row of K walks the row in stored order
//     (SparseMatrix::row_norms, sparse.cpp:120-131): a running sum for the
//     1-norm, a running maximum for the infinity norm.
//   - Column norms: SparseMatrix::col_norms (sparse.cpp:133-140) adds each
//     nonzero into its column in storage order, so column j accumulates its
//     entries in the order the transpose lists them. One thread per column
//     walks the transpose's row j and reads the current values from K
//     through pos (the position in K of each transpose entry).
//   - Factors: d = norm > 0 ? 1 / sqrt(norm) : 1, both operations correctly
//     rounded, as on the host.
//   - Values: each nonzero is multiplied by its row factor, then by its
//     column factor: the two roundings of scale_rows then scale_cols.
//
// Only multiplies, adds, maxima, square roots and divides occur, all in
// explicit round-to-nearest intrinsics, so nothing is contracted.
#include "engine.hpp"

namespace anu {
namespace {

__global__ void row_norms_kernel(int32_t rows, const int32_t* __restrict__ start,
                                 const double* __restrict__ value, int one, double* __restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    const int32_t end = start[r + 1];
    for (int32_t e = start[r]; e < end; ++e) {
      const double v = fabs(value[e]);
      acc = one ? __dadd_rn(acc, v) : fmax(acc, v);
    }
    out[r] = acc;
  }
}

__global__ void col_norms_kernel(int32_t cols, const int32_t* __restrict__ tstart,
                                 const int32_t* __restrict__ pos, const double* __restrict__ value,
                                 int one, double* __restrict__ out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cols;
       c += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    const int32_t end = tstart[c + 1];
    for (int32_t t = tstart[c]; t < end; ++t) {
      const double v = fabs(value[pos[t]]);
      acc = one ? __dadd_rn(acc, v) : fmax(acc, v);
    }
    out[c] = acc;
  }
}

__global__ void factors_kernel(int32_t len, const double* __restrict__ norm, double* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = norm[i];
    d[i] = v > 0.0 ? __ddiv_rn(1.0, __dsqrt_rn(v)) : 1.0;
  }
}

__global__ void scale_values_kernel(int32_t nnz, const int32_t* __restrict__ row_of,
                                    const int32_t* __restrict__ index,
                                    const double* __restrict__ d1, const double* __restrict__ d2,
                                    double* __restrict__ value) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
       e += (int64_t)gridDim.x * blockDim.x)
    value[e] = __dmul_rn(__dmul_rn(value[e], d1[row_of[e]]), d2[index[e]]);
}

int grid_of(int64_t n) { return grid_for(n, 256, 148 * 8); }

template <class T>
void put(cudaStream_t s, DevBuf<T>& d, const std::vector<T>& h) {
  d.alloc(std::max<size_t>(h.size(), 1));
  if (!h.empty())
    ANU_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
}

template <class T>
void get(cudaStream_t s, std::vector<T>* h, const T* d, size_t count) {
  h->resize(count);
  if (count > 0)
    ANU_CUDA(cudaMemcpyAsync(h->data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost, s));
}

}  // namespace

Scaling scale_matrix_sweeps_device(Exec& ex, HostCsr* k, HostCsr* kt, int ruiz_iterations,
                                   bool pock_chambolle, ScalingSweeps* sweeps) {
  const int32_t m = k->rows, n = k->cols, nnz = k->nnz();
  const int total = ruiz_iterations + (pock_chambolle ? 1 : 0);
  std::vector<int32_t> pos;
  HostCsr t = transpose(*k, &pos);
  std::vector<int32_t> row_of(static_cast<size_t>(nnz));
  for (int32_t r = 0; r < m; ++r)
    for (int32_t e = k->start[r]; e < k->start[r + 1]; ++e) row_of[e] = r;
  cudaStream_t s = ex.stream;
  DevBuf<int32_t> d_start, d_index, d_row_of, d_tstart, d_pos;
  DevBuf<double> d_value;
  put(s, d_start, k->start);
  put(s, d_index, k->index);
  put(s, d_row_of, row_of);
  put(s, d_tstart, t.start);
  put(s, d_pos, pos);
  put(s, d_value, k->value);
  const size_t tm = static_cast<size_t>(std::max(m, 1)), tn = static_cast<size_t>(std::max(n, 1));
  DevBuf<double> rn(tm), cn(tn), d1(tm * std::max(total, 1)), d2(tn * std::max(total, 1));
  DevBuf<double> rn0(tm), cn0(tn);
  auto norms = [&](int one, double* r_out, double* c_out) {
    if (m > 0) row_norms_kernel<<<grid_of(m), 256, 0, s>>>(m, d_start.p, d_value.p, one, r_out);
    if (n > 0)
      col_norms_kernel<<<grid_of(n), 256, 0, s>>>(n, d_tstart.p, d_pos.p, d_value.p, one, c_out);
    ANU_CUDA(cudaGetLastError());
    ex.launches += 2;
  };
  norms(0, rn0.p, cn0.p);
  for (int sweep = 0; sweep < total; ++sweep) {
    const int one = sweep >= ruiz_iterations ? 1 : 0;
    double* f1 = d1.p + static_cast<size_t>(sweep) * tm;
    double* f2 = d2.p + static_cast<size_t>(sweep) * tn;
    norms(one, rn.p, cn.p);
    if (m > 0) factors_kernel<<<grid_of(m), 256, 0, s>>>(m, rn.p, f1);
    if (n > 0) factors_kernel<<<grid_of(n), 256, 0, s>>>(n, cn.p, f2);
    if (nnz > 0)
      scale_values_kernel<<<grid_of(nnz), 256, 0, s>>>(nnz, d_row_of.p, d_index.p, f1, f2,
                                                       d_value.p);
    ANU_CUDA(cudaGetLastError());
    ex.launches += 3;
  }
  norms(0, rn.p, cn.p);
  std::vector<double> h_rn0, h_cn0, h_rn, h_cn, h_d1, h_d2;
  get(s, &h_rn0, rn0.p, static_cast<size_t>(m));
  get(s, &h_cn0, cn0.p, static_cast<size_t>(n));
  get(s, &h_rn, rn.p, static_cast<size_t>(m));
  get(s, &h_cn, cn.p, static_cast<size_t>(n));
  get(s, &h_d1, d1.p, tm * total);
  get(s, &h_d2, d2.p, tn * total);
  get(s, &k->value, d_value.p, static_cast<size_t>(nnz));
  ANU_CUDA(cudaStreamSynchronize(s));

  Scaling out;
  out.row_scale.assign(static_cast<size_t>(m), 1.0);
  out.col_scale.assign(static_cast<size_t>(n), 1.0);
  out.row_spread_before = norm_spread(h_rn0);
  out.col_spread_before = norm_spread(h_cn0);
  out.row_spread_after = norm_spread(h_rn);
  out.col_spread_after = norm_spread(h_cn);
  sweeps->d1.clear();
  sweeps->d2.clear();
  for (int sweep = 0; sweep < total; ++sweep) {
    const double* f1 = h_d1.data() + static_cast<size_t>(sweep) * tm;
    const double* f2 = h_d2.data() + static_cast<size_t>(sweep) * tn;
    std::vector<double> a(f1, f1 + m), b(f2, f2 + n);
    for (int32_t i = 0; i < m; ++i) out.row_scale[i] *= a[i];
    for (int32_t j = 0; j < n; ++j) out.col_scale[j] *= b[j];
    sweeps->d1.push_back(std::move(a));
    sweeps->d2.push_back(std::move(b));
  }
  // The transpose of the scaled matrix: the structure built above, the
  // values taken from K.
  for (size_t e = 0; e < pos.size(); ++e) t.value[e] = k->value[pos[e]];
  *kt = std::move(t);
  return out;
}

}  // namespace anu
