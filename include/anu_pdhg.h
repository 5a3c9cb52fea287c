/*
 * anu_pdhg.h - C ABI of the B200 (sm_100a) PDHG / PDLP engine.
 *
 * Drop-in for the first-order LP path of anukulan:
 *   - solve_pdhg(const StandardLp&, const PdhgOptions&)   src/anukulan/pdhg.hpp:543
 *   - evaluate_residual(lp, x, y)                         src/anukulan/pdhg.hpp:548
 *   - estimate_matrix_norm(lp, iterations, tolerance)     src/anukulan/pdhg.hpp:580
 *   - the LinAlgBackend seam                              src/anukulan/backend.hpp:24-215
 * plus the batched case stack, the packed uneven batch and the adjoint, which
 * have no counterpart in the reference.
 *
 * Conventions (all entry points):
 *   - C linkage, plain pointers and sizes, no exceptions across the boundary.
 *   - Every function returns an int status: ANU_OK (0) or an ANU_ERR_* code.
 *     The message of the last failure on the calling thread is returned by
 *     anu_last_error(). The reference throws std::runtime_error from
 *     cuda_check (src/anukulan/cuda_backend.cu:32-37); here that becomes
 *     ANU_ERR_CUDA plus the message.
 *   - Host pointers unless the name says "device". Inputs are copied; the
 *     caller keeps ownership of every array it passes.
 *   - One CUDA stream per handle. A handle is not thread safe; distinct
 *     handles may be used from distinct threads.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     entry point returns ANU_ERR_NO_DEVICE.
 */
#ifndef ANU_PDHG_H
#define ANU_PDHG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: options.stop is a const volatile uint8_t* (std::atomic<bool>'s byte).
 * 3: options.tile_threads and options.cluster_chunks; the result's
 *    row_product_threads, column_product_threads and tile_trial_seconds. */
#define ANU_PDHG_ABI_VERSION 3

/* Return codes. */
enum {
  ANU_OK = 0,
  ANU_ERR_INVALID = 1,   /* bad argument, shape or option */
  ANU_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  ANU_ERR_NO_DEVICE = 3, /* no CUDA device */
  ANU_ERR_MEMORY = 4,    /* device or host allocation failed */
  ANU_ERR_DEVICE_WAIT = 5, /* a bounded device-side wait gave up */
  ANU_ERR_INTERNAL = 6
};

/* PdhgStatus, src/anukulan/pdhg.hpp:417-423 (same order). */
enum {
  ANU_PDHG_OPTIMAL = 0,
  ANU_PDHG_PRIMAL_INFEASIBLE = 1,
  ANU_PDHG_ITERATION_LIMIT = 2,
  ANU_PDHG_TIME_LIMIT = 3,
  ANU_PDHG_NUMERICAL_ERROR = 4
};

/* PdhgOptions::Termination, src/anukulan/pdhg.hpp:372-373. */
enum {
  ANU_TERMINATION_FULL = 0,
  ANU_TERMINATION_PRIMAL_FEASIBILITY = 1,
  ANU_TERMINATION_DUAL_FEASIBILITY = 2
};

/* Arithmetic of the iteration (no counterpart in the reference, which is
 * FP64 throughout). */
enum {
  ANU_PRECISION_FP64 = 0, /* matrix and iterates in FP64 */
  ANU_PRECISION_FP32 = 1  /* matrix and iterates in FP32; checks, restart and
                             termination decisions and refinement in FP64 */
};

/* Compressed sparse rows, SparseMatrix (src/anukulan/sparse.hpp:37-101):
 * start[rows+1], index[nnz] (column indices, sorted and unique within a row),
 * value[nnz]. Int is int32 as in the reference (sparse.hpp:11). */
typedef struct anu_csr {
  int32_t rows;
  int32_t cols;
  int32_t nnz;
  const int32_t* start;
  const int32_t* index;
  const double* value;
} anu_csr;

/* StandardLp, src/anukulan/standard_form.hpp:23-66:
 *   min c'x  s.t.  K_eq x = q_eq (first num_equalities rows),
 *                  K_ineq x >= q_ineq (the rest),  lower <= x <= upper.
 * Infinite bounds are +-INFINITY. The transpose the reference caches in
 * StandardLp::kt is built by the engine. */
typedef struct anu_lp {
  anu_csr k;
  const double* c;     /* n */
  const double* q;     /* m */
  const double* lower; /* n */
  const double* upper; /* n */
  int32_t num_equalities;
  double objective_scale;  /* model objective = scale * c'x + offset */
  double objective_offset;
} anu_lp;

/* PdhgOptions, src/anukulan/pdhg.hpp:19-415, field for field (bools as
 * int32 0/1), followed by the engine's own additions. Fill it with
 * anu_pdhg_default_options() and then change what differs. */
typedef struct anu_pdhg_options {
  double tolerance;                       /* 1e-6 */
  double gap_tolerance;                   /* 0: same as tolerance */
  int32_t max_iterations;                 /* 200000 */
  double time_limit_seconds;              /* 300 */
  int32_t termination_check_frequency;    /* 40 */
  double absolute_tolerance;              /* 0 */
  int32_t require_inf_norm_termination;   /* 1 */
  int32_t adaptive_step_size;             /* 1 */
  int32_t primal_weight_updates;          /* 1 */
  int32_t restarts;                       /* 1 */
  int32_t halpern;                        /* 1 */
  int32_t halpern_restart;                /* 0 */
  int32_t halpern_minimum_epoch;          /* 16 */
  int32_t polish_feasibility;             /* 1 */
  int32_t polish_first_iteration;         /* 100 */
  double polish_iteration_factor;         /* 0.125 */
  int32_t polish_minimum_iterations;      /* 40 */
  int32_t polish_maximum_iterations;      /* 20000 */
  int32_t polish_on_exit;                 /* 1 */
  double reflection;                      /* 1.0 */
  int32_t constant_step_size;             /* 1 */
  double constant_step_scale;             /* 0.90 */
  int32_t restart_on_fixed_point;         /* 1 */
  int32_t pid_primal_weight;              /* 1 */
  double primal_weight_kp;                /* 0.5 */
  double primal_weight_ki;                /* 0.0 */
  double primal_weight_kd;                /* 0.3 */
  int32_t ruiz_iterations;                /* ScalingOptions: 10 */
  int32_t pock_chambolle;                 /* ScalingOptions: 1 */
  int32_t reuse_products;                 /* 1 */
  int32_t detect_infeasibility;           /* 1 */
  double infeasibility_tolerance;         /* 1e-8 */
  int32_t termination;                    /* ANU_TERMINATION_FULL */
  double known_matrix_norm;               /* 0: estimate it */
  double initial_step_size;               /* 0: derive it */
  double initial_primal_weight;           /* 0: derive it */
  int32_t verbose;                        /* 0 */
  int32_t log_frequency;                  /* 5000 */
  /* PdhgOptions::stop (pdhg.hpp:414, a const std::atomic<bool>*): a one-byte
   * flag that another thread may set at any time. The engine reads it with
   * an acquire load at every termination check; once it is nonzero the
   * solve (every case still running, for a case stack) ends at that check
   * with ANU_PDHG_TIME_LIMIT, as a stop request ends the reference's solve.
   * A std::atomic<bool>, which is one lock-free byte holding a bool, binds
   * as reinterpret_cast<const volatile uint8_t*>(ptr). NULL: no
   * cancellation. */
  const volatile uint8_t* stop;

  /* --- engine additions, no counterpart in PdhgOptions --- */
  int32_t precision;            /* ANU_PRECISION_FP64 (default) or _FP32 */
  /* Iterative refinement, FP32 only: the FP32 iterate is an offset from an
   * FP64 base point. At every termination check the offset is folded into
   * the base and the correction LP is re-formed from the FP64 residual
   * there (cost c - K'y*, right-hand side q - K x*, bounds and dual floor
   * shifted by the base); the PDHG state is shifted with it, so the
   * trajectory continues unchanged while FP32 carries only the movement
   * since the last check. 0 = plain FP32 iterates. */
  int32_t refinement;           /* 1 */
  int32_t device;               /* CUDA device ordinal, 0 */
  int32_t use_graphs;           /* capture iteration chunks in CUDA graphs, 1 */
  /* Record CUDA events around every iteration chunk on the engine's stream
   * and report their total in anu_pdhg_result::device_iteration_seconds.
   * Events do not serialise the stream. 0 = off. */
  int32_t profile;
  /* Case stacks of 16 or more cases run as two half-stacks at once, each on
   * its own stream and host thread. 0 = one stack on one stream. 1.
   * Not used when the stack runs persistent chunks (below). */
  int32_t split_stacks;
  /* 1: a case stack of 17 to 64 cases whose segment schedule fits in one
   * wave of CTAs runs each chunk of iterations between termination checks
   * as one cooperative kernel with grid barriers between its products, as
   * one stack. 0 (default): graphs of two launches per iteration. On B200
   * a grid barrier costs about as much as the launch it replaces, so the
   * graphs of two half-stacks are faster on the stacks measured so far. */
  int32_t persistent_chunks;
  /* 1: anu_pdhg_create / anu_pdhg_solve relabel the rows and columns of the
   * scaled matrix so the gathers of the two products share cache lines: rows
   * by decreasing length (within the equality and the inequality block),
   * columns by the first such row they touch. Scaling runs before it, in the
   * original order; every row keeps its nonzeros in their original order, so
   * each product entry is summed as without it. x, y and warm starts stay in
   * the caller's order. The reductions of the checks then sum in another
   * order, so FP64 results agree with the unrelabelled solve to rounding,
   * not bit for bit. Case stacks, packed batches and the unrolled program
   * ignore it. 0 (default) = off. */
  int32_t locality_order;
  /* 1 (default): scale_lp's Ruiz and Pock-Chambolle sweeps run on the
   * device, with the same norms in the same summation order, the same
   * correctly rounded factors and the same two roundings per nonzero, so the
   * scaled matrix and every factor are bit-identical to the host sweeps.
   * 0 = on the host. */
  int32_t scaling_on_device;
  /* CTA size of the single-LP product kernels (K~ x and K~' y): 128 or 256
   * fixes it for both. 0 (default): anu_pdhg_create / anu_pdhg_solve on an
   * LP of at least 2^20 nonzeros runs short trial solves of the LP (4
   * checks each, results discarded), two for each of the four pairs, and
   * keeps the pair with the least device time per iteration when it beats
   * 128/128 by 1%; smaller LPs and case stacks take 128; packed batches time
   * both tiles on a sample of their LPs at their worker count. Every tile
   * size sums every row in the same order, so the choice changes timing
   * only, never a result. The result reports the pair and the trial time. */
  int32_t tile_threads;
  /* 1: a single LP (or the last case of a stack) whose y, x_bar, matrix
   * slices and step vectors fit in the shared memory of a cluster's CTAs,
   * with no row longer than 1,024 nonzeros, runs each check period as ONE
   * launch of one thread-block cluster of 16 CTAs (8 where 16 does not fit)
   * that stays resident for the period's iterations, instead of two
   * launches per iteration. Rows are summed in the same order, so the
   * iterates are the same bit for bit. Packed batches keep two launches per
   * iteration. 0 (default): two launches per iteration; measured faster on
   * the LPs the engine is benchmarked on. */
  int32_t cluster_chunks;
} anu_pdhg_options;

/* PdhgResidual, src/anukulan/pdhg.hpp:429-496. */
typedef struct anu_pdhg_residual {
  double primal_residual;
  double dual_residual;
  double primal_residual_inf;
  double dual_residual_inf;
  double primal_objective;
  double dual_objective;
  double absolute_gap;
  double relative_primal;
  double relative_dual;
  double relative_gap;
  double relative_primal_inf;
  double relative_dual_inf;
} anu_pdhg_residual;

/* PdhgResult::Phases, src/anukulan/pdhg.hpp:516-536. */
typedef struct anu_pdhg_phases {
  double scaling;
  double matrix_norm;
  double setup;
  double iterating;
  double checks;
  double polishing;
} anu_pdhg_phases;

/* PdhgResult, src/anukulan/pdhg.hpp:498-541. x and y are written to the
 * caller's arrays; everything else is here. */
typedef struct anu_pdhg_result {
  int32_t status;            /* ANU_PDHG_* */
  double objective;          /* model sense, including the offset */
  int32_t iterations;
  int32_t restarts;
  int32_t polish_attempts;
  int32_t polish_iterations;
  int32_t polished;
  double solve_seconds;
  double matrix_norm_estimate;
  double final_step_size;
  double final_primal_weight;
  anu_pdhg_phases phases;
  anu_pdhg_residual residual;
  /* ScalingReport, src/anukulan/scaling.hpp:36-44 */
  double row_spread_before;
  double row_spread_after;
  double col_spread_before;
  double col_spread_after;
  /* engine additions */
  int32_t refinement_rounds; /* refinements (re-centrings) performed */
  int32_t kernel_launches;   /* kernels this solve launched (graph nodes included) */
  /* With options.profile: device time of the iteration chunks (CUDA events
   * on the engine stream) and the iterations they ran, summed over every
   * case run this result shares (a case stack runs its cases together). A
   * stack whose last case was handed to the single-LP kernels counts its
   * full-width chunks only. */
  double device_iteration_seconds;
  int64_t device_iterations;
  /* CTA size of the single-LP products K~ x (row) and K~' y (column):
   * options.tile_threads, or the pair the handle's trial solves chose. */
  int32_t row_product_threads;
  int32_t column_product_threads;
  double tile_trial_seconds; /* host time of those trial solves; 0 when none ran */
  char message[160];
} anu_pdhg_result;

/* ---------------------------------------------------------------- basics */

/* Version string of the library ("anu-pdhg-b200 <semver> sm_100a"). */
const char* anu_pdhg_version(void);

/* PdhgOptions{} defaults, src/anukulan/pdhg.hpp:19-415. */
void anu_pdhg_default_options(anu_pdhg_options* options);

/* Copies the last error message of this thread into buf (NUL terminated).
 * Returns the code of that error, ANU_OK if there was none. */
int anu_last_error(char* buf, int32_t size);

/* Number of CUDA devices visible (0 when none). Never fails. */
int32_t anu_device_count(void);

/* Destroyed handles leave their device and pinned host blocks in a
 * process-wide cache, from which the next handles on the same device take
 * them instead of allocating. This frees every cached block and returns the
 * bytes freed. Safe at any time: no live handle owns a cached block. No
 * counterpart in the reference, which allocates through its backend per
 * solve (src/anukulan/pdhg.cpp:377-1285). */
int64_t anu_release_cached_memory(void);

/* ----------------------------------------------------------- single LP */

/* solve_pdhg, src/anukulan/pdhg.hpp:543 / pdhg.cpp:377-1285.
 * warm_x (n) and warm_y (m) may be NULL together (cold start) and follow
 * PdhgOptions::warm_x/warm_y semantics. x (n) and y (m) receive the unscaled
 * primal and dual solution. */
int anu_pdhg_solve(const anu_lp* lp, const anu_pdhg_options* options,
                   const double* warm_x, const double* warm_y, double* x,
                   double* y, anu_pdhg_result* result);

/* The same solve split in two, so the setup (scaling, upload, transpose,
 * the ||K|| power iteration) can be paid once and the solve repeated with
 * different starts. anu_pdhg_create does everything up to the loop; the
 * handle owns its device memory and its stream. */
typedef struct anu_pdhg anu_pdhg;
int anu_pdhg_create(const anu_lp* lp, const anu_pdhg_options* options,
                    anu_pdhg** handle);
int anu_pdhg_run(anu_pdhg* handle, const double* warm_x, const double* warm_y,
                 double* x, double* y, anu_pdhg_result* result);
/* Replaces the handle's objective, right-hand side and bounds (n, m, n, n
 * entries, the caller's order; NULL keeps that vector) and keeps its scaled
 * matrix, product schedules and ||K~||, so the next anu_pdhg_run solves
 * another LP with the same matrix without the set-up: the reference's
 * backends keep a prepared matrix per SparseMatrix::id() the same way
 * (src/anukulan/cuda_backend.cu:561-588). Scaling factors depend on the
 * matrix alone, so the run is the one a fresh anu_pdhg_solve of that LP would
 * make, bit for bit in FP64. */
int anu_pdhg_set_case(anu_pdhg* handle, const double* c, const double* q,
                      const double* lower, const double* upper);
void anu_pdhg_destroy(anu_pdhg* handle);

/* evaluate_residual, src/anukulan/pdhg.hpp:548 / pdhg.cpp:112-174: the FP64
 * convergence measures of any primal-dual pair against the unscaled LP,
 * computed on the device. */
int anu_evaluate_residual(const anu_lp* lp, const double* x, const double* y,
                          anu_pdhg_residual* out);

/* The relabelling options.locality_order applies (no counterpart in the
 * reference), computed on the host without a device: row_old[r] (m entries)
 * is the original row of relabelled row r, col_old[c] (n entries) the
 * original column of relabelled column c. Rows are ordered by decreasing
 * length within the equality block and within the inequality block (ties
 * keep their order); columns by the first relabelled row they appear in
 * (ties keep their order, empty columns last). An LP without rows or columns
 * gets the identity. */
int anu_locality_relabel(const anu_lp* lp, int32_t* row_old, int32_t* col_old);

/* estimate_matrix_norm, src/anukulan/pdhg.hpp:580 / pdhg.cpp:223-282: power
 * iteration on K'K on the device, FP64. */
int anu_estimate_matrix_norm(const anu_lp* lp, int32_t iterations,
                             double tolerance, double* norm);

/* ------------------------------------------------------ LinAlgBackend seam
 * The coarse operations of LinAlgBackend (src/anukulan/backend.hpp:24-215) on
 * device memory, so a thin C++ adapter can implement LinAlgBackend over this
 * library and run the reference's own solve_pdhg on these kernels. Vectors
 * are FP64 device arrays from anu_backend_allocate. Matrices are uploaded by
 * anu_backend_prepare under the caller's identity key (SparseMatrix::id(),
 * src/anukulan/sparse.hpp:51), never by address. All operations run in order
 * on one library-owned stream, a blocking stream (ordered with the legacy
 * default stream). Those that hand the host a value or read a host buffer
 * (upload, download, dot, the norms and terms, allocate, prepare) return when
 * done; fill, copy, multiply, the two updates, accumulate and scale_into
 * return once queued, as the reference's CUDA backend's kernel launches do. */
int anu_backend_allocate(int64_t n, double** device_ptr);        /* backend.hpp:50, zeroed */
int anu_backend_deallocate(double* device_ptr);                  /* backend.hpp:51 */
int anu_backend_upload(const double* host, double* device_ptr, int64_t n);    /* :52 */
int anu_backend_download(const double* device_ptr, double* host, int64_t n);  /* :53 */
int anu_backend_fill(double* device_ptr, int64_t n, double value);            /* :54 */
int anu_backend_copy(const double* source, double* target, int64_t n);        /* :55 */
int anu_backend_prepare(uint64_t id, const anu_csr* a);          /* backend.hpp:35 */
int anu_backend_release(void);                                    /* backend.hpp:36 */
int anu_backend_multiply(uint64_t id, const double* x, double* y);  /* :58, y = A x */
int anu_backend_dot(const double* a, const double* b, int64_t n, double* out);  /* :64 */
int anu_backend_two_norm(const double* a, int64_t n, double* out);              /* :65 */
int anu_backend_inf_norm(const double* a, int64_t n, double* out);              /* :66 */
int anu_backend_primal_update(int64_t n, double tau, double gamma, double halpern,
                              const double* x, const double* c, const double* kt_y,
                              const double* lower, const double* upper,
                              const double* anchor, double* x_out, double* dx,
                              double* x_bar);                     /* backend.hpp:89-93 */
int anu_backend_dual_update(int64_t m, int64_t num_equalities, double sigma,
                            double gamma, double halpern, const double* y,
                            const double* q, const double* k_x_bar,
                            const double* k_x, const double* anchor_y,
                            const double* anchor_kx, double* y_out, double* dy,
                            double* k_out, double* k_dx);         /* backend.hpp:114-119 */
int anu_backend_accumulate(int64_t n, double weight, const double* v, double* sum); /* :123 */
int anu_backend_scale_into(int64_t n, double weight, const double* sum, double* out); /* :126 */
int anu_backend_weighted_norm_squared(int64_t n, int64_t m, const double* dx,
                                      const double* dy, double omega,
                                      double* out);               /* backend.hpp:129-130 */
int anu_backend_step_size_terms(int64_t n, int64_t m, const double* dx,
                                const double* dy, const double* k_dx, double omega,
                                double* interaction, double* movement); /* :146-148 */
/* ConvergenceProblem (backend.hpp:157-165) flattened; out[7] receives
 * primal_sq, primal_inf, q_dot_y, dual_sq, dual_inf, bound_term, c_dot_x
 * (ConvergenceTerms, backend.hpp:168-176). */
int anu_backend_convergence_terms(int64_t n, int64_t m, const double* c,
                                  const double* lower, const double* upper,
                                  const double* q, const double* row_scale,
                                  const double* col_scale, int64_t num_equalities,
                                  const double* x, const double* k_x,
                                  const double* y, const double* kt_y,
                                  double* out);                   /* backend.hpp:198-202 */

/* LinAlgBackend::set_profiling (backend.hpp:213): on = 1 times the device
 * work of every seam operation above with CUDA events on the library stream,
 * waiting for each, so a profiled run is slower than a plain one and its
 * shares are what it is for; 0 stops and clears the timings. */
int anu_backend_set_profiling(int32_t on);
/* LinAlgBackend::profile_report (backend.hpp:214): one line per operation
 * (device seconds, share, calls, microseconds per call), the total, and the
 * prepared matrices with their product schedules. Writes at most size-1
 * characters and a NUL into buf (NULL: nothing); *length (may be NULL) gets
 * the report's full length. Empty when nothing was timed. */
int anu_backend_profile_report(char* buf, int32_t size, int32_t* length);

/* anu_backend_convergence_terms without any device allocation. There is no
 * counterpart in the reference.
 *
 * It is for hosts that may not call cudaMalloc: a plugin inside an application
 * that owns the device memory pool, or a process whose allocations all go
 * through another runtime's allocator. Such a host can hand over its own
 * input and output arrays, but a library that allocates behind its back
 * breaks its accounting. The caller passes inputs and outputs exactly as for
 * anu_backend_convergence_terms and gets the same 7 terms.
 *
 * - Scratch: the partial sums live in one fixed array in the library's device
 *   image, 42,768 bytes, which every GPU that loads the library holds until
 *   the process exits.
 * - Limits: n and m up to 2^31-1 (every loop index is 64-bit). Larger or
 *   negative lengths return ANU_ERR_INVALID with a message.
 * - Set-up: the first call on each device looks the array up on that device
 *   (cudaGetSymbolAddress) and caches the address. Make that first call
 *   before any stream capture begins.
 * - Stream: work runs on the legacy default stream, which waits for and
 *   blocks every stream created without cudaStreamNonBlocking, and the call
 *   returns when its work is done.
 * - Sharing: every call shares the one array. Calls that overlap on the same
 *   GPU (from several host threads, say) race on it and must be serialised by
 *   the caller. */
int anu_backend_convergence_terms_noalloc(int64_t n, int64_t m, const double* c,
                                          const double* lower, const double* upper,
                                          const double* q, const double* row_scale,
                                          const double* col_scale,
                                          int64_t num_equalities, const double* x,
                                          const double* k_x, const double* y,
                                          const double* kt_y, double* out);

/* ------------------------------------------------------ batched case stack
 * K cases that share K (the matrix) and differ in c, q, lower and upper.
 * No counterpart in the reference, whose solve_pdhg takes one LP. The stack
 * runs as one SpMM-shaped iteration over case-interleaved vectors: every
 * nonzero of the matrix read serves all active cases. Each case keeps its own
 * step size, primal weight, restarts and termination; a case that terminates
 * is retired, and its lanes skip their gathers and updates from then on. In
 * FP32, a stack of 8 or more cases whose last case runs on alone moves that
 * case, state unchanged, to the single-LP kernels, which are quicker for one
 * case; its FP32 sums then round as a single solve's do. FP64 stacks keep
 * their layout.
 *
 * Case arrays are case-major: c[k*n + j], q[k*m + i], and so on. A NULL case
 * array means every case uses the base LP's vector. */
typedef struct anu_pdhg_batch anu_pdhg_batch;
int anu_pdhg_batch_create(const anu_lp* base, int32_t num_cases,
                          const double* c, const double* q, const double* lower,
                          const double* upper, const anu_pdhg_options* options,
                          anu_pdhg_batch** handle);
/* Runs every case to termination. x is num_cases*n, y is num_cases*m, results
 * num_cases entries. */
int anu_pdhg_batch_solve(anu_pdhg_batch* handle, double* x, double* y,
                         anu_pdhg_result* results);
/* The same, each case warm started as solve_pdhg takes a warm start
 * (PdhgOptions::warm_x / warm_y, src/anukulan/pdhg.cpp:478-502): warm_x is
 * num_cases*n, warm_y num_cases*m, case-major; both or neither. */
int anu_pdhg_batch_solve_warm(anu_pdhg_batch* handle, const double* warm_x,
                              const double* warm_y, double* x, double* y,
                              anu_pdhg_result* results);
void anu_pdhg_batch_destroy(anu_pdhg_batch* handle);

/* A streaming case stack: cases admitted as the caller produces them and
 * results handed back as cases retire. The reference has no counterpart;
 * it is the admit / retire / results cycle of a rolling stack (the cases of
 * anu_pdhg_batch_create are not used), for callers whose next cases depend on
 * earlier results, such as the open nodes of branch and bound
 * (src/anukulan/branch_and_bound.cpp:532-565).
 *
 * - source: fills the next case and returns 1, or returns 0 when it has none
 *   now. Its arrays (c: n, q: m, lower and upper: n) arrive holding the base
 *   LP's vectors, so it writes only what its case changes; *case_id is the
 *   caller's label for the case. It is asked for up to `slots` cases at the
 *   start, which fixes the stack's width, and again whenever a case retires at
 *   a termination check and no case is waiting.
 * - sink: receives each case's x (n), y (m) and result when the case retires,
 *   before its slot is refilled, so it may decide what the source hands out.
 * - Both run on the calling thread. Every case starts cold and runs the
 *   iteration it would run alone (its counts start at its admission).
 * - slots: 1 to 64. The call returns when the source has nothing more and
 *   every admitted case has retired. */
typedef int32_t (*anu_pdhg_case_source)(void* user, int32_t* case_id, double* c, double* q,
                                        double* lower, double* upper);
typedef void (*anu_pdhg_case_sink)(void* user, int32_t case_id, const double* x,
                                   const double* y, const anu_pdhg_result* result);
int anu_pdhg_batch_stream(anu_pdhg_batch* handle, int32_t slots, anu_pdhg_case_source source,
                          anu_pdhg_case_sink sink, void* user);

/* ------------------------------------------------------ packed batches
 * Independent LPs of different shapes solved together on one GPU. No
 * counterpart in the reference, whose callers loop solve_pdhg over such a
 * set. Every LP is solved exactly as anu_pdhg_solve solves it (same
 * iterates, same result); what the batch adds is concurrency: W host
 * workers take LPs from one queue, largest first, each on its own stream,
 * and a worker that retires an LP admits the next one at once.
 *
 * workers: 0 = choose W by a short autotuning run at creation (each
 * candidate W runs W LPs drawn evenly from the batch for a few check
 * periods; the most nonzero-iterations per second wins), else W itself.
 * With options.tile_threads 0, the single-LP product tile of every LP (128
 * or 256 threads per CTA) is then chosen the same way at that W; the tile
 * changes timing only, never a result. Each result reports it. */
typedef struct anu_pdhg_packed anu_pdhg_packed;
int anu_pdhg_packed_create(int32_t num_lps, const anu_lp* lps,
                           const anu_pdhg_options* options, int32_t workers,
                           anu_pdhg_packed** handle);
/* x[i] (n_i entries) and y[i] (m_i entries) receive LP i's answer (a NULL
 * array or entry skips it); results has num_lps entries. */
int anu_pdhg_packed_solve(anu_pdhg_packed* handle, double* const* x,
                          double* const* y, anu_pdhg_result* results);
/* The worker count in use (the autotuner's choice when it ran). */
int32_t anu_pdhg_packed_workers(const anu_pdhg_packed* handle);
void anu_pdhg_packed_destroy(anu_pdhg_packed* handle);

/* ------------------------------------------------------ unrolled adjoint
 * d(loss)/d(c, q) through a truncated, unrolled PDHG. No counterpart in the
 * reference. The unrolled program is `iterations` steps of reflected
 * Halpern PDHG (reflection 1) on the scaled problem, step sizes fixed at the
 * values solve_pdhg starts from (or options.initial_step_size /
 * initial_primal_weight), the Halpern anchor restarted at the new iterate
 * every `checkpoint_every` steps, from solve_pdhg's cold start. It is
 * piecewise linear in (c, q); the adjoint is exact wherever no projection
 * sits on its kink.
 *
 * Cases as in anu_pdhg_batch_create (case-major arrays, NULL = base), at
 * most 64. The forward pass keeps the iterate every `checkpoint_every`
 * steps; the backward pass recomputes each segment from its checkpoint,
 * recording the projection masks, and reverses it with hand-written
 * kernels (two fused SpMV launches per step); gradients accumulate in FP64.
 * options.precision selects FP32 or FP64 iterates. */
typedef struct anu_pdhg_unrolled anu_pdhg_unrolled;
int anu_pdhg_unrolled_create(const anu_lp* base, int32_t num_cases,
                             const double* c, const double* q,
                             const double* lower, const double* upper,
                             const anu_pdhg_options* options, int32_t iterations,
                             int32_t checkpoint_every, anu_pdhg_unrolled** handle);
/* The fixed primal and dual step sizes of each case (num_cases each). */
int anu_pdhg_unrolled_step_sizes(const anu_pdhg_unrolled* handle, double* tau,
                                 double* sigma);
/* x_T (num_cases*n) and y_T (num_cases*m), unscaled, case-major; either
 * may be NULL. */
int anu_pdhg_forward_unrolled(anu_pdhg_unrolled* handle, double* x, double* y);
/* Given dloss/dx_T (num_cases*n) and dloss/dy_T (num_cases*m, NULL = 0),
 * writes dloss/dc (num_cases*n) and dloss/dq (num_cases*m). A loss that
 * depends on c directly (such as c'x_T) adds that term itself. */
int anu_pdhg_backward(anu_pdhg_unrolled* handle, const double* dloss_dx,
                      const double* dloss_dy, double* grad_c, double* grad_q);
void anu_pdhg_unrolled_destroy(anu_pdhg_unrolled* handle);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* ANU_PDHG_H */
