// Host-side preparation of an LP for the device: the CSR transpose, the
// diagonal scaling and the row-block schedule the SpMV kernels walk.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace anu {

constexpr double kInf = __builtin_inf();

// CSR with int32 indices, FP64 values (SparseMatrix, src/anukulan/sparse.hpp).
struct HostCsr {
  int32_t rows = 0;
  int32_t cols = 0;
  std::vector<int32_t> start{0};
  std::vector<int32_t> index;
  std::vector<double> value;
  int32_t nnz() const { return static_cast<int32_t>(index.size()); }
};

// Checks monotone starts and in-range indices; "" when valid.
std::string validate_csr(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                         const int32_t* index);

HostCsr copy_csr(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                 const int32_t* index, const double* value);

// SparseMatrix::transpose (src/anukulan/sparse.cpp:93-117): counting sort with
// rows visited in increasing order, so each transposed row is sorted.
HostCsr transpose(const HostCsr& a);
// The same, and pos[t] = the position in `a` of the transpose's entry t.
HostCsr transpose(const HostCsr& a, std::vector<int32_t>* pos);

// y = A x, each row summed left to right (sparse.cpp:72-80).
void multiply(const HostCsr& a, const double* x, double* y);

// Result of scale_lp (src/anukulan/scaling.cpp:75-100), applied in place to
// the matrix and to any number of (c, q, lower, upper) cases sharing it.
struct Scaling {
  std::vector<double> row_scale;  // D1
  std::vector<double> col_scale;  // D2
  double row_spread_before = 1.0, row_spread_after = 1.0;
  double col_spread_before = 1.0, col_spread_after = 1.0;
};

// Ruiz infinity-norm sweeps then one Pock-Chambolle 1-norm sweep on the
// matrix. The factors depend on the matrix alone; they are kept per sweep so
// the vectors of every case sharing the matrix can be scaled exactly the way
// the reference scales its single case (scaling.cpp:32-59: one multiply or
// divide per sweep, in order), which makes each case bit-identical to a
// separate solve.
struct ScalingSweeps {
  std::vector<std::vector<double>> d1;
  std::vector<std::vector<double>> d2;
};
Scaling scale_matrix_sweeps(HostCsr* k, int ruiz_iterations, bool pock_chambolle,
                            ScalingSweeps* sweeps);
// Largest over smallest positive norm (1 when all are zero), the spread
// scale_lp reports (scaling.cpp:18-28).
double norm_spread(const std::vector<double>& norms);

void scale_vectors(const ScalingSweeps& sw, int32_t m, int32_t n, double* c, double* q,
                   double* lower, double* upper);

// Row-block schedule for the staged (CSR-adaptive) SpMV: consecutive rows
// grouped so a block holds at most `block_nnz` nonzeros and `block_rows` rows;
// a row longer than `block_nnz` gets a block of its own. Blocks are ordered
// longest first so the long rows start in the first wave.
struct RowBlock {
  int32_t row_begin;
  int32_t row_end;
};
// Rows longer than long_row (or than block_nnz) get a block each.
std::vector<RowBlock> row_blocks(const HostCsr& a, int32_t block_nnz, int32_t block_rows,
                                 int32_t long_row);

// Segment schedule of the case-stack product (see seg_kernel): every row
// cut into segments of at most seg_nnz nonzeros (a longer row into
// seg_per_cta equal segments), and consecutive rows grouped into CTAs of at
// most seg_per_cta segments and row_max rows.
struct SegmentSchedule {
  std::vector<int32_t> seg_begin;  // segments + 1
  std::vector<int32_t> row_seg;    // rows + 1
  std::vector<int32_t> cta_row;    // ctas + 1
  std::vector<int32_t> cta_seg;    // ctas + 1
};
SegmentSchedule segment_schedule(const HostCsr& a, int32_t seg_nnz, int32_t seg_per_cta,
                                 int32_t row_max);

// The rows of a matrix dealt to the `parts` CTAs of one thread-block cluster
// (see cluster_chunk_kernel): contiguous ranges, cut where the running
// nonzero count crosses each part's even share. Rows of more than
// serial_row nonzeros are summed by a warp; each part lists its own.
struct ClusterSchedule {
  std::vector<int32_t> bounds;      // parts + 1 row bounds
  std::vector<int32_t> warp_start;  // parts + 1 offsets into warp_rows
  std::vector<int32_t> warp_rows;   // the rows longer than serial_row, by part
  int32_t max_row = 0;              // longest row
  int32_t max_part_rows = 0;        // most rows in one part
  int32_t max_part_nnz = 0;         // most nonzeros in one part
};
ClusterSchedule cluster_schedule(const HostCsr& a, int32_t parts, int32_t serial_row);

double now_seconds();

}  // namespace anu
