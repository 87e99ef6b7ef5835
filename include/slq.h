/*
 * slq.h -- C ABI of the B200 stochastic Lanczos quadrature engine
 * (libslq_b200.so).
 *
 * The engine replaces the GPU SLQ path of ameli/imate v0.25.2: the linear
 * operator (imate/_cu_linear_operator/), the trace estimator
 * (imate/_cu_trace_estimator/), the probe generator (imate/_random_generator/)
 * and the CUDA loader (imate/_cuda_dynamic_loading/).  All device memory is
 * owned by the caller (PyTorch tensors in the Python host); the engine only
 * carves the buffers it is given.  Every entry point returns a status and
 * never aborts; slq_last_error() describes the last failure of the calling
 * thread.
 *
 * Stream: every call takes a cudaStream_t (passed as void*; NULL = legacy
 * default stream) and enqueues all device work on it.
 */

#ifndef SLQ_B200_H_
#define SLQ_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLQ_ABI_VERSION 5

typedef enum {
    SLQ_OK = 0,
    SLQ_ERR_BAD_ARG = 1,          /* argument out of range / inconsistent   */
    SLQ_ERR_BAD_CSR = 2,          /* malformed index arrays                 */
    SLQ_ERR_WORKSPACE = 3,        /* workspace pointer/size too small       */
    SLQ_ERR_CUDA = 4,             /* a CUDA runtime call failed             */
    SLQ_ERR_NAN = 5,              /* NaN/Inf in a Lanczos coefficient       */
    SLQ_ERR_EIGEN = 6,            /* tridiagonal eigen-solve did not converge */
    SLQ_ERR_UNSUPPORTED = 7,      /* valid request this library does not serve */
    SLQ_ERR_TIMEOUT = 8           /* a bounded device-side wait ran out     */
} slq_status;

typedef enum { SLQ_F32 = 0, SLQ_F64 = 1 } slq_dtype;
typedef enum { SLQ_CSR = 0, SLQ_CSC = 1 } slq_format;
/* Matrix functions f applied at the quadrature nodes as f(theta^p), with
 * their coefficients in slq_params.func_coeff: log (logdet,
 * imate/functions/logarithm.cpp), 1/x (traceinv, inverse.cpp), x (trace,
 * identity.cpp), exp(c0 x) (trexp, exponential.cpp), (c0 x + c1) /
 * (c2 x + c3) (trlinfrac, homographic.cpp), 1 on [c0, c1] else 0
 * (eigencount, indicator.cpp), exp(-((x - c0) / c1)^2 / 2) / (c1 sqrt(2 pi))
 * (density, gaussian.cpp) and (1 + tanh(c0 x)) / 2 (smoothstep.cpp). */
typedef enum {
    SLQ_FUNC_LOG = 0, SLQ_FUNC_INV = 1, SLQ_FUNC_ID = 2, SLQ_FUNC_EXP = 3,
    SLQ_FUNC_LINFRAC = 4, SLQ_FUNC_INDICATOR = 5, SLQ_FUNC_GAUSSIAN = 6,
    SLQ_FUNC_SMOOTHSTEP = 7
} slq_func;
typedef enum { SLQ_RNG_PARITY = 0, SLQ_RNG_FAST = 1 } slq_rng;

/* Opaque operator: a sparse matrix A (or A + t I when affine != 0) resident
 * on one device. */
typedef struct slq_op slq_op;

/* Bytes of device workspace slq_operator_create needs for the layouts it
 * derives: a CSR copy of A^T for gram runs, a CSR copy of A for CSC input,
 * and the symmetrically permuted matrix when a permutation is given.
 * Replaces the device upload of cuCSRMatrix / cuCSCMatrix
 * (imate/_cu_linear_operator/cu_csr_matrix.cu:165-224,
 *  cu_csc_matrix.cu:165-230). */
slq_status slq_operator_workspace_bytes(int64_t num_rows, int64_t num_cols,
                                        int64_t nnz, int dtype, int format,
                                        int need_transpose, int has_perm,
                                        int group_rows, size_t* bytes);

/* Wrap caller-owned device arrays (values dtype, int32 indices, int32 index
 * pointer of length num_rows+1 for CSR / num_cols+1 for CSC) as an operator.
 * need_transpose requests A^T as well (gram / Golub-Kahn runs).  affine marks
 * the operator as A + t I (imate.AffineMatrixFunction with B = I; the
 * eigenvalue shift relation of c_affine_matrix_function.cpp:98-113 holds),
 * or, in normal-equations runs (slq_params.gram = 2), as A^T A + t I.
 * check_indices != 0 validates indptr monotonicity and index range on the
 * device first (SLQ_ERR_BAD_CSR on failure).
 *
 * perm (device int32[num_rows], or NULL; square CSR input only) is a
 * locality ordering: the engine stores B = P A P^T with B[i][j] =
 * A[perm[i]][perm[j]] and writes probe element e to row perm^-1[e], so every
 * inner product -- hence every Lanczos coefficient, node, weight and sample --
 * is that of A; only the order of floating-point sums changes.  A
 * bandwidth-reducing order (reverse Cuthill-McKee) keeps each SpMM gather
 * window inside L2.  slq_operator_dot on such an operator acts on permuted
 * vectors (y' = B x').
 *
 * group_rows (0, 4, 8 or 16) additionally stores A (and A^T) in a row-group
 * format: per group of consecutive rows, the sorted union of their column
 * indices with a dense value per (union column, row), zero where absent.
 * One gathered row of a probe block then feeds group_rows rows of FMAs, which
 * cuts the SpMM's L1/L2 gather traffic for wide blocks (32 <= b <= 256).
 * slq_group_order makes the groups of consecutive rows overlap well.
 * Results are bit-identical to the CSR kernel (same summation order; the
 * padding adds exact zeros).
 *
 * Replaces pycuMatrix.__cinit__ (imate/_cu_linear_operator/py_cu_matrix.pyx:
 * 118-200) and cuCSRMatrix / cuCSCMatrix / cuCSRAffineMatrixFunction
 * construction. */
slq_status slq_operator_create(const void* data, const int32_t* indices,
                               const int32_t* indptr, int64_t num_rows,
                               int64_t num_cols, int64_t nnz, int dtype,
                               int format, int affine, int need_transpose,
                               int check_indices, const int32_t* perm,
                               int group_rows, void* workspace,
                               size_t workspace_bytes, void* stream,
                               slq_op** out);

/* Tensor-core block format of a float32 sparse operator (no counterpart in
 * the reference, whose products are one cusparseSpMV per probe,
 * imate/_cu_basic_algebra/cusparse_interface.cu:243, through
 * cuCSRMatrix::dot, imate/_cu_linear_operator/cu_csr_matrix.cu:278-318).
 * The stored rows of A (transpose = 0) or of A^T (transpose = 1) are cut
 * into blocks of 128 consecutive rows; each block keeps the sorted union of
 * its column indices (padded to a multiple of 16) and its values as a dense
 * 128 x union matrix.  Every row is scaled by a power of two and split into
 * FP16 high and low parts, so one SpMM over b = 128 or 256 probes runs on
 * the tensor cores (tcgen05 kind::f16, three products hi*hi, hi*lo, lo*hi
 * of the scaled operands, FP32 accumulation: samples within about 1e-5 of
 * FP64).  Its cost follows the union sizes: store the operator with a row
 * order whose consecutive 128-row blocks share columns
 * (slq_block_group_order, slq_block_order).  Built on the device in two
 * calls on the same scratch: slq_operator_blocks_bytes prepares the scratch
 * (the union sizes, from a bitmap of each block's columns in shared memory,
 * or from sorted (block, column) keys where a block's columns span more
 * than 262,144) and sizes the format (it synchronizes the stream);
 * slq_operator_add_blocks, given that scratch as it was left, builds the
 * format into `format` (caller memory that must outlive the operator) and
 * attaches it (given another scratch it prepares that one first); the
 * scratch can be released after it returns.  Duplicate (row, column)
 * entries are summed.  Products at b = 128 / 256 then use it (slq_run,
 * batch plans, the tuner) unless the tuner picked another candidate. */
slq_status slq_operator_blocks_scratch_bytes(const slq_op* op, int transpose,
                                             size_t* bytes);
slq_status slq_operator_blocks_bytes(const slq_op* op, int transpose,
                                     void* scratch, size_t scratch_bytes,
                                     void* stream, size_t* format_bytes);
slq_status slq_operator_add_blocks(slq_op* op, int transpose, void* scratch,
                                   size_t scratch_bytes, void* format,
                                   size_t format_bytes, void* stream);

/* The block format attached to one direction of an operator: its 128-row
 * blocks and 16-column stages (both 0 when none).  A product over b probes
 * issues 3 x stages x 128 x 16 x b multiply-adds on the tensor cores
 * against 2 nnz b useful flops; each stage moves 8 KB of A parts. */
slq_status slq_operator_blocks_info(const slq_op* op, int transpose,
                                    int64_t* blocks, int64_t* stages);

/* Reverse Cuthill-McKee order of a square CSR pattern (host arrays; the
 * pattern is taken as symmetric).  Each connected component starts at its
 * lowest-degree row and is visited breadth-first with the children of a row
 * in increasing degree;
 * order[k] receives the row at position k of the reversed visit order.  A
 * bandwidth-reducing order for the locality of the SpMM gathers (no
 * counterpart in the reference). */
slq_status slq_rcm_order(int64_t n, const int32_t* indptr,
                         const int32_t* indices, int32_t* order);

/* Row-group aggregation order (host; no counterpart in the reference).
 * For a square CSR pattern (host arrays; data of dtype or NULL), visits the
 * rows in base_order (NULL = identity) and makes each row not yet placed the
 * seed of a group of group_rows rows: the seed, its not-yet-placed
 * neighbours by decreasing |a_ij|, their neighbours, and, when the
 * neighbourhood runs out, the next unplaced rows of the base order.  Orders
 * of at least 32768 rows are cut into K = min(8, n / 16384) segments of the
 * base order swept independently on the host threads, each group from one
 * segment's rows; groups are then listed by their seeds' base positions,
 * the short groups at the segments' ends last.  The order depends on n and
 * the inputs only, not on the thread count.
 * order[k] receives the row at position k; every group but the short ones
 * has exactly group_rows rows, so passing order as slq_operator_create's perm
 * lines the groups up with the row-group format's, whose cost falls with
 * the overlap of the rows' column sets. */
slq_status slq_group_order(int64_t n, const int32_t* indptr,
                           const int32_t* indices, const void* data,
                           int dtype, int group_rows,
                           const int32_t* base_order, int32_t* order);

/* Block aggregation order (host; no counterpart in the reference): merges
 * the groups of group_rows consecutive rows of group_order (a row order such
 * as slq_group_order gives) into blocks of groups_per_block groups whose
 * column sets overlap.  Blocks start at the unplaced groups in order; each
 * then takes the unplaced group with the most row pairs (a row of the
 * group, a neighbour row in the block) per row pair of its own (ties: the
 * earlier group), or the next unplaced groups when no row links them (the
 * group graph is counted once, in parallel).  order[k] receives
 * the row at position k: blocks in order, their groups in joining order,
 * each group's rows as in group_order; the n % group_rows rows after the
 * last whole group stay last.  On the benchmark correlation matrix, blocks
 * of eight 16-row groups have a mean column union of about 650 against
 * about 1,500 for 128 consecutive rows of group_order (about 70 ms on 8
 * host threads). */
slq_status slq_block_order(int64_t n, const int32_t* indptr,
                           const int32_t* indices, const int32_t* group_order,
                           int group_rows, int groups_per_block,
                           int32_t* order);

/* Blocks, then groups inside them (host; no counterpart in the reference):
 * the rows aggregated as slq_group_order does but into blocks of block_rows
 * rows (a seed and its strongest neighbours, theirs, ...), then the rows of
 * every whole block, in base order, aggregated the same way into groups of
 * group_rows rows drawn from that block only.  order[k] receives the row at
 * position k: every whole block of the tensor-core block format holds whole
 * row groups, so one order serves both formats.  On the benchmark
 * correlation matrix (n = 262144, RCM base order) 128-row blocks of 16-row
 * groups have about 2 % smaller column unions than slq_block_order's blocks
 * of slq_group_order's groups, with 16-row groups about 3 % larger, at a
 * fraction of the cost (no group graph).  block_rows must be a multiple of
 * group_rows, at most 16384.  The order does not depend on the thread
 * count. */
slq_status slq_block_group_order(int64_t n, const int32_t* indptr,
                                 const int32_t* indices, const void* data,
                                 int dtype, int block_rows, int group_rows,
                                 const int32_t* base_order, int32_t* order);

/* Workspace for slq_rcm_order_device (device bytes). */
slq_status slq_rcm_order_device_workspace_bytes(int64_t n, size_t* bytes);

/* slq_rcm_order on the device: the same order for a square CSR pattern of n
 * rows and nnz entries in device memory (int32 indptr / indices, validated
 * first); order (device, n entries) receives it.  When no row has more than
 * 1024 entries every breadth-first level runs inside one cooperative launch
 * (grid barriers between a level's phases, each wait bounded: a wait that
 * runs out returns SLQ_ERR_TIMEOUT); otherwise one level per host round (a
 * synchronisation per level and per component).  *done = 1 on success;
 * *done = 0, with SLQ_OK and order undefined, when the pattern has more than
 * max_components connected components or, on the round-per-level path, its
 * sort keys (level offset, degree, row) need more than 64 bits -- the caller
 * then uses slq_rcm_order.  No counterpart in the reference. */
slq_status slq_rcm_order_device(int64_t n, int64_t nnz, const int32_t* indptr,
                                const int32_t* indices, int max_components,
                                int32_t* order, int* done, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Mean |position(i) - position(j)| over the nonzeros (i, j) of sampled rows
 * of a square CSR pattern (host arrays): the rows numpy's
 * unique(linspace(0, n - 1, min(n, sample_rows)).astype(int64)) picks,
 * positions the identity (perm NULL) or perm^-1 (perm[k] = row at position
 * k).  Decides whether a locality order pays (no counterpart in the
 * reference). */
slq_status slq_order_spread(int64_t n, const int32_t* indptr,
                            const int32_t* indices, const int32_t* perm,
                            int64_t sample_rows, double* spread);

/* Mean fill nnz / (group_rows x union size) of sampled groups of group_rows
 * consecutive rows of `order` (NULL = identity) of a CSR pattern (host
 * arrays): the groups numpy's unique(linspace(0, n / group_rows - 1,
 * min(sample_groups, n / group_rows)).astype(int64)) picks, groups without
 * entries left out.  Predicts the row-group format's padding (no
 * counterpart in the reference). */
slq_status slq_group_fill(int64_t n, const int32_t* indptr,
                          const int32_t* indices, const int32_t* order,
                          int group_rows, int64_t sample_groups,
                          double* fill);

/* Dense FP32 operator (the role of cuDenseMatrix: construction and upload
 * imate/_cu_linear_operator/cu_dense_matrix.cu:39-61 and :94-122, cuBLAS
 * gemv products :130-238): A is num_rows x num_cols, row-major, in device
 * memory.  Creation splits A (and, with need_transpose, A^T) into TF32
 * hi/lo parts in the workspace; products run on the tensor cores
 * (tcgen05 kind::tf32, three terms: ~FP32 accuracy) with the SpMM
 * epilogue.  The workspace also holds the probe-block parts of one product,
 * so an operator serves one product at a time (not two runs at once, and
 * not batch plans); the tuner does not apply to it.  Float32 only. */
slq_status slq_dense_operator_workspace_bytes(int64_t num_rows,
                                              int64_t num_cols, int dtype,
                                              int need_transpose,
                                              size_t* bytes);
slq_status slq_dense_operator_create(const void* data, int64_t num_rows,
                                     int64_t num_cols, int dtype, int affine,
                                     int need_transpose, void* workspace,
                                     size_t workspace_bytes, void* stream,
                                     slq_op** out);

/* Release the host-side operator record (device arrays stay with their
 * owners).  Replaces the cuLinearOperator destructors
 * (imate/_cu_linear_operator/cu_csr_matrix.cu:95-154). */
slq_status slq_operator_destroy(slq_op* op);

/* y = A x (transpose=0) or y = A^T x (transpose=1), plus t x for affine
 * operators, for a block of `width` column vectors stored row-major
 * ([len][width], contiguous), in the operator's dtype.  Replaces
 * cuCSRMatrix::dot / transpose_dot (cu_csr_matrix.cu:278-414),
 * cuCSCMatrix::dot / transpose_dot (cu_csc_matrix.cu:287-470) and
 * cuCSRAffineMatrixFunction::dot (cu_csr_affine_matrix_function.cu:124-211),
 * which the reference's tests check against scipy
 * (imate/_cu_linear_operator/tests/test_cu_matrix.pyx:50-187). */
slq_status slq_operator_dot(slq_op* op, int transpose, double t,
                            const void* x, void* y, int width, void* stream);

/* Estimator settings: the keyword arguments of imate's slq methods
 * (imate/logdet/_slq_method.pyx:24-44, trace_estimator.pyx:38-61) plus the
 * engine's own block width and probe-generator choice. */
typedef struct {
    int func;                      /* slq_func                               */
    int gram;                      /* 0 Lanczos on A; 1 Golub-Kahn on A      */
                                   /* (spectrum of A^T A); 2 Lanczos on the  */
                                   /* normal operator A^T A (+ t I if the    */
                                   /* operator is affine; no counterpart in  */
                                   /* the reference: imate cannot shift a    */
                                   /* Gram matrix)                           */
    double exponent;               /* p in f(A^p)                            */
    int orthogonalize;             /* 0 none, <0 full, k last-k              */
    int64_t seed;                  /* >= 0 (the host maps None to a clock seed) */
    int lanczos_degree;            /* m, 1..SLQ_MAX_DEGREE                   */
    double lanczos_tol;            /* breakdown tolerance (eps of dtype)     */
    int min_num_samples;
    int max_num_samples;
    double error_atol;
    double error_rtol;
    double confidence_level;
    double outlier_significance_level;
    int block_size;                /* probes advanced together; 0 = auto     */
    int rng;                       /* slq_rng                                */
    int64_t first_probe;           /* global index of sample 0 (probe shards) */
    double func_coeff[4];          /* coefficients of func (see slq_func)    */
} slq_params;

#define SLQ_MAX_DEGREE 256

/* Host-side outputs, caller-allocated (same arrays the reference fills in
 * py_cu_trace_estimator.pyx:199-247).  samples is [max_num_samples][q]
 * row-major and NaN where not computed.  lanczos_size is per sample.
 * alpha/beta (optional, may be NULL) receive the per-sample coefficients,
 * [max_num_samples][lanczos_degree].  probe_status (optional, may be NULL)
 * receives per sample a bit mask, -1 where not computed: 1 non-finite
 * Lanczos coefficients or eigen-solve results, 2 the eigen-solve did not
 * converge, 4 a quadrature node under log was not positive (or a node under
 * 1/x was zero), 8 a non-finite sample.  The reference prints a warning for
 * a vanishing basis vector in its Gram-Schmidt step
 * (imate/_c_trace_estimator/c_orthogonalization.cpp:186-192) and otherwise
 * averages whatever the samples are; here the flags say which samples are
 * suspect. */
typedef struct {
    double* trace;                     /* [q]   */
    double* error;                     /* [q]   */
    double* samples;                   /* [max][q] */
    int32_t* processed_samples_indices;/* [max] */
    int32_t* num_samples_used;         /* [q]   */
    int32_t* num_outliers;             /* [q]   */
    int32_t* converged;                /* [q]   */
    int32_t* lanczos_size;             /* [max] */
    double* alpha;                     /* [max][m] or NULL */
    double* beta;                      /* [max][m] or NULL */
    int32_t* probe_status;             /* [max] or NULL */
    int32_t all_converged;
    int32_t num_blocks;                /* probe blocks launched              */
    int64_t num_probes_computed;       /* incl. the unused tail of a block   */
    int64_t gpu_launches;              /* kernels launched by the call       */
    float alg_wall_time;               /* seconds, CUDA events on the stream */
} slq_result;

/* Device workspace slq_run needs for these settings. */
slq_status slq_run_workspace_bytes(const slq_op* op, const slq_params* p,
                                   int num_inquiries, size_t* bytes);

/* The estimator.  parameters (host, length num_inquiries) are the t values
 * of an affine operator (ignored otherwise; num_inquiries must then be 1).
 * Replaces cuTraceEstimator<T>::cu_trace_estimator
 * (imate/_cu_trace_estimator/cu_trace_estimator.cu:197-315) with
 * _cu_stochastic_lanczos_quadrature (:419-660), cu_lanczos_tridiagonalization
 * (cu_lanczos_tridiagonalization.cu:119-248), cu_golub_kahn_bidiagonalization
 * (cu_golub_kahn_bidiagonalization.cu:113-242) and
 * cuOrthogonalization::gram_schmidt_process (cu_orthogonalization.cu:128-228),
 * and the host LAPACK eigensolve it called (diagonalization.cpp:89-231). */
slq_status slq_run(slq_op* op, const slq_params* p, const double* parameters,
                   int num_inquiries, void* workspace, size_t workspace_bytes,
                   void* stream, slq_result* result);

/* SpMM autotuner (no counterpart in the reference, whose products are one
 * cusparseSpMV per probe, cusparse_interface.cu:243).  The candidates for a
 * block width are the storage formats the operator holds crossed with their
 * tiles: CSR warp per row; row-group (the operator's group_rows rows sharing
 * a union of columns) with LV probes per lane and NS warps per row group,
 * b = 32 LV NS; in FP32 with 8- or 16-row groups at b = 128 or 256, the
 * row-group kernel whose X rows arrive by TMA gathers; and in FP32 with
 * 16-row groups at b = 128 or 256, the tensor-core row-group kernel
 * (tcgen05 kind::tf32 on TF32 hi/lo splits of both operands, accumulators
 * in tensor memory; FP32-level accuracy, chosen only by the tuner or
 * slq_operator_set_variant).  slq_operator_tune times every candidate (reps
 * launches each, CUDA events, after one untimed launch) on workspace blocks
 * and makes the fastest the operator's choice for that width and
 * direction; every later product the operator takes at that width
 * (slq_run, slq_batch_*, slq_operator_dot) uses it, except that
 * slq_operator_dot, which has no tensor map or error word, falls back to the
 * built-in choice for the TMA and tensor-core kernels.  Results of different
 * candidates agree to rounding, not bitwise (their partial-sum orders
 * differ). */
#define SLQ_TUNE_MAX_CANDIDATES 16

typedef struct {
    int32_t width;
    int32_t transpose;
    int32_t num_candidates;
    int32_t chosen;                                /* fastest candidate      */
    int32_t kind[SLQ_TUNE_MAX_CANDIDATES];         /* 0 CSR, 1 row-group,    */
                                                   /* 2 row-group + TMA,     */
                                                   /* 3 row-group, tensor    */
                                                   /*   cores                */
    int32_t group_rows[SLQ_TUNE_MAX_CANDIDATES];
    int32_t lanes_vec[SLQ_TUNE_MAX_CANDIDATES];    /* LV probes per lane     */
    int32_t slices[SLQ_TUNE_MAX_CANDIDATES];       /* NS warps per row group */
    double milliseconds[SLQ_TUNE_MAX_CANDIDATES];  /* mean per launch        */
} slq_tune_result;

slq_status slq_operator_tune_workspace_bytes(const slq_op* op, int width,
                                             size_t* bytes);
slq_status slq_operator_tune(slq_op* op, int width, int transpose, int reps,
                             void* workspace, size_t workspace_bytes,
                             void* stream, slq_tune_result* result);
/* Force candidate `candidate` (an index as reported by slq_operator_tune) for
 * this width and direction; -1 restores the built-in choice. */
slq_status slq_operator_set_variant(slq_op* op, int width, int transpose,
                                    int candidate);

/* Batched estimator (no counterpart in the reference, which runs one matrix
 * per call).  A batch plan holds `count` independent estimator runs -- any
 * mix of operators, sizes, dtypes, functions and settings -- and records
 * every probe block of every run into one CUDA graph, each run on its own
 * branch so that runs of small matrices overlap on the device.  A run
 * computes all max_num_samples probes (there is no host decision inside the
 * graph) and the host then applies the reference's sequential stopping rule
 * to them, so each slq_result equals that of slq_run with the same operator,
 * settings and SpMM choice: the samples it would have used, its estimate,
 * error, sample counts and outliers.  Differences from slq_run's result:
 * num_blocks and num_probes_computed count every block, alg_wall_time is the
 * time of the whole graph, and gpu_launches counts the run's kernels in the
 * graph.  parameters[i] (host, num_inquiries[i] values) are run i's t values
 * (NULL for a non-affine operator).  The plan keeps pointers into the
 * workspace and the operators; both must outlive it.  slq_batch_create
 * synchronizes `stream` (it uploads the probe start states). */
typedef struct slq_batch slq_batch;

slq_status slq_batch_workspace_bytes(int count, slq_op* const* ops,
                                     const slq_params* params,
                                     const int* num_inquiries, size_t* bytes);
slq_status slq_batch_create(int count, slq_op* const* ops,
                            const slq_params* params,
                            const double* const* parameters,
                            const int* num_inquiries, void* workspace,
                            size_t workspace_bytes, void* stream,
                            slq_batch** out);
/* One launch of the plan's graph on `stream`, then the host stopping rule
 * into results[0..count). */
slq_status slq_batch_run(slq_batch* batch, void* stream, slq_result* results);
/* Kernel nodes in the plan's graph. */
slq_status slq_batch_info(const slq_batch* batch, int64_t* kernels,
                          int64_t* nodes);
slq_status slq_batch_destroy(slq_batch* batch);

/* Tensor-core self-test (no counterpart in the reference): D = A B for one
 * 128 x 8 by 8 x 16 FP32 tile (device arrays, row-major) through tcgen05,
 * the building blocks of the tensor-core SpMM checked on one tile.  mode 0:
 * A in tensor memory, B in shared memory, one kind::tf32 MMA; mode 1: as 0
 * with both operands split into TF32 hi/lo parts, D = A_lo B_hi + A_hi B_lo
 * + A_hi B_hi; mode 2: tensor-memory round trip (D[m][0..7] and [8..15]
 * receive the stored TF32 hi and lo parts of A[m]); mode 3: A and B in
 * shared memory, one MMA.  error: one device int32 of scratch (set when the
 * MMA's completion wait runs out, SLQ_ERR_TIMEOUT). */
slq_status slq_tc_selftest(const float* a, const float* b, float* d, int mode,
                           int32_t* error, void* stream);

/* No counterpart in the reference: one kind::tf32 MMA with an MN-major
 * operand, D[128][32] = A[128][8] B'[8][32] (device arrays, row-major).  B'
 * sits in shared memory in the MN-major layout a TF32 operand needs: the
 * 128-byte swizzle with 32-byte atoms (descriptor layout type 1; 4-row K
 * atoms of 128-byte rows, 32-byte chunks swizzled by the row; the plain
 * 128-byte swizzle reads such an operand as zeros).  gather 0: B' = B, written by
 * the threads; gather 1: B' rows k = B rows perm[k], perm = 3 0 7 1 6 2 5 4,
 * loaded by two TMA tile::gather4 copies (the load form of a block SpMM's
 * probe rows).  Only TF32 hi parts are used.  b must be 16-byte aligned;
 * error as slq_tc_selftest. */
slq_status slq_tc_selftest_mn(const float* a, const float* b, float* d,
                              int gather, int32_t* error, void* stream);

/* Probe generator alone: writes probes [first, first+count) of the stream for
 * (seed, rng) as a row-major block [len][width] of +-1 in the given dtype
 * (columns >= count are zero).  Replaces
 * RandomArrayGenerator::generate_random_array
 * (imate/_random_generator/random_array_generator.cpp:63-165) driven as in
 * c_trace_estimator.cpp:235,449 with one thread. */
slq_status slq_generate_probes(int64_t seed, int rng, int64_t len,
                               int64_t first, int count, int width, int dtype,
                               void* out, void* workspace,
                               size_t workspace_bytes, void* stream);
slq_status slq_generate_probes_workspace_bytes(int64_t len, int width,
                                               size_t* bytes);

/* The probe generator above without any workspace (no counterpart in the
 * reference).  For callers that cannot allocate device memory -- code whose
 * device memory is entirely owned by a caching allocator or a fixed arena,
 * and latency-critical paths that must not take the synchronisation cudaFree
 * can cause.  Its scratch (probe start states and jump polynomials) is a
 * fixed 288 KB array inside the library, held by every GPU that loads it.
 * Limit: width <= 1024 probes per call (SLQ_ERR_BAD_ARG beyond).  The first
 * call on a device resolves the array's device address, so make that first
 * call before any stream capture; the address is kept for the process, so
 * after a reset of the device's context (cudaDeviceReset) do not call this
 * function on that device again.  All calls share the array: calls that
 * overlap on the GPU (other streams, other host threads) race.  In parity
 * mode (SLQ_RNG_PARITY) each call stages the scratch through host memory and
 * synchronizes its stream, and it returns SLQ_ERR_BAD_ARG, before touching
 * the stream, when that stream is capturing. */
slq_status slq_generate_probes_noalloc(int64_t seed, int rng, int64_t len,
                                       int64_t first, int count, int width,
                                       int dtype, void* out, void* stream);

/* Nodes (theta) and weights (tau) of a batch of Jacobi matrices, on the
 * device, by implicit QL in FP64.  All arrays are device memory in
 * probe-minor layout: alpha, beta, theta, tau are [m][count] (entry i of
 * matrix p at i*count + p); sizes [count] gives each matrix's order; status
 * [count] receives a bit mask: 1 non-finite coefficients or results, 2 QL
 * did not converge (0 when neither).
 * gram != 0 treats (alpha, beta) as an upper bidiagonal B and solves B^T B.
 * Replaces Diagonalization::eigh_tridiagonal / svd_bidiagonal
 * (imate/_c_trace_estimator/diagonalization.cpp:89-231). */
slq_status slq_nodes_weights(const double* alpha, const double* beta,
                             const int32_t* sizes, int count, int m, int gram,
                             double* theta, double* tau, int32_t* status,
                             void* stream);

/* Reference-style convergence test and outlier-trimmed averaging on host
 * arrays (imate/_c_trace_estimator/convergence_tools.cpp:95-376); exported so
 * the host logic can be checked without a GPU. */
int slq_check_convergence(const double* samples, int num_inquiries,
                          int min_num_samples, const int32_t* order,
                          int num_processed, double confidence_level,
                          double error_atol, double error_rtol, double* error,
                          int32_t* num_samples_used, int32_t* converged);
void slq_average_estimates(double confidence_level,
                           double outlier_significance_level,
                           int num_inquiries, int max_num_samples,
                           const int32_t* num_samples_used,
                           const int32_t* order, const double* samples,
                           int32_t* num_outliers, double* trace,
                           double* error);
double slq_erfinv(double x);

/* xoshiro256** jump-ahead on the host: advances state (4 words) by k draws.
 * Exported so the parity probe stream can be checked without a GPU. */
void slq_xoshiro_jump_ahead(uint64_t* state, uint64_t k);

/* Per-kernel timing.  Between slq_profile_begin() and slq_profile_end()
 * every kernel the calling thread launches is bracketed by CUDA events on its
 * stream; slq_profile_end() synchronizes and returns, per kernel class, the
 * launch count, the summed device time and the summed algorithmic bytes
 * (compulsory HBM traffic of the operation as launched).  Replaces the
 * CudaTimer around the reference's sample loop (cuda_timer.cu:28-84) with a
 * per-kernel breakdown. */
typedef enum {
    SLQ_K_SPMM = 0, SLQ_K_DOTS = 1, SLQ_K_REORTH = 2, SLQ_K_FINALIZE = 3,
    SLQ_K_EIG = 4, SLQ_K_PROBE = 5, SLQ_K_OTHER = 6,
    SLQ_K_SPLIT = 7,  /* the FP16 split of the probe block before a block SpMM */
    SLQ_K_COUNT = 8
} slq_kernel_kind;

typedef struct {
    int64_t launches;
    double milliseconds;
    double bytes;
} slq_kernel_stat;

slq_status slq_profile_begin(void);
slq_status slq_profile_end(slq_kernel_stat* stats /* [SLQ_K_COUNT] */);

/* Learned surrogate of a parameter sweep t -> trace f(A + t I): a fully
 * connected network 1 -> 64 -> 64 -> 1 with tanh hidden units in FP32,
 * fitted on the device to SLQ samples of the sweep.  It stands in for
 * imate's interpolators of such sweeps (imate/interpolator/,
 * interpolate_schatten.py:426-492; no counterpart of the network itself).
 * Parameters: float[SLQ_MLP_PARAMS] packed as W1[64] b1[64] W2[64][64]
 * b2[64] W3[64] b3[1] (device).  All pointers are device memory. */
#define SLQ_MLP_WIDTH 64
#define SLQ_MLP_PARAMS (64 + 64 + 64 * 64 + 64 + 64 + 1)
#define SLQ_MLP_MAX_BATCH 64

/* y[i] = net(x[i]) for count inputs. */
slq_status slq_mlp_forward(const float* params, const float* x, int count,
                           float* y, void* stream);

/* Gradient of mean_i (net(x_i) - t_i)^2 over a batch (<= 64 points) into
 * grad[SLQ_MLP_PARAMS], and the loss into *loss. */
slq_status slq_mlp_grad(const float* params, const float* x, const float* t,
                        int batch, float* grad, float* loss, void* stream);

/* `steps` full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) in one
 * launch.  adam_m / adam_v (float[SLQ_MLP_PARAMS]) carry the moments across
 * calls; steps_done is the number of steps already taken.  loss_history
 * (float[steps] or NULL) receives the loss before each step. */
slq_status slq_mlp_train(float* params, float* adam_m, float* adam_v,
                         const float* x, const float* t, int batch, int steps,
                         int steps_done, float lr, float* loss_history,
                         void* stream);

/* Device count / properties (replaces query_device.cu:48-64). */
slq_status slq_device_info(int* num_devices, int* num_sms,
                           int* max_threads_per_sm);

const char* slq_last_error(void);
int slq_abi_version(void);

/* Test hook (no counterpart in the reference): the next `count` launches of
 * the streaming update / reorthogonalisation kernel treat their first
 * mbarrier wait as timed out.  That wait then takes the path of a real one
 * that ran out -- the CTA sets the run's error word, stops, waits (with the
 * full bound) for the copies it issued, and the call returns
 * SLQ_ERR_TIMEOUT -- so the failure path can be exercised without a fault.
 * 0 switches it off. */
slq_status slq_debug_fail_stream_waits(int count);

/* Test hook (no counterpart in the reference): 1 builds the block format's
 * union columns by sorting (block, column) keys, the path the build
 * otherwise takes only for a block whose columns span more than 262,144;
 * 0 (the default) lets it use per-block bitmaps.  Both give the same
 * format. */
slq_status slq_debug_blocks_sorted_keys(int on);

#ifdef __cplusplus
}
#endif

#endif /* SLQ_B200_H_ */
