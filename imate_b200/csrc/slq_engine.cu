// B200 SLQ engine: operator set-up, the block Krylov driver and the C ABI
// declared in include/slq.h.
//
// The reference GPU path (imate/_cu_trace_estimator/cu_trace_estimator.cu)
// runs one probe at a time per device: a host-generated probe is copied to
// the device, every Lanczos step issues a cuSPARSE SpMV and a series of
// cuBLAS level-1 calls whose dot/nrm2 results return to the host, and the
// tridiagonal eigen-solve runs in host LAPACK.  Here a block of b probes
// advances together and stays on the device: probes are generated in place,
// each Krylov step is one SpMM over the block plus fused update /
// reorthogonalisation passes whose reductions are finalised on the device,
// and the eigen-solve and quadrature run on the device.  The host reads b
// samples per block and replays the reference's sequential stopping rule.

#include <cub/cub.cuh>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/slq.h"
#include "slq_blk.cuh"
#include "slq_kernels.cuh"
#include "slq_rng.h"

using namespace slq;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

namespace {

thread_local std::string g_error;

slq_status fail(slq_status s, const std::string& msg)
{
    g_error = msg;
    return s;
}

#define SLQ_CK(call)                                                        \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess)                                              \
            return fail(SLQ_ERR_CUDA, std::string(#call) + ": " +           \
                                          cudaGetErrorString(e_));          \
    } while (0)

#define SLQ_LAUNCH_CK()                                                     \
    do {                                                                    \
        cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess)                                              \
            return fail(SLQ_ERR_CUDA, std::string("kernel launch: ") +      \
                                          cudaGetErrorString(e_));          \
    } while (0)

#define SLQ_TRY(...)                                                        \
    do {                                                                    \
        slq_status s_ = (__VA_ARGS__);                                      \
        if (s_ != SLQ_OK) return s_;                                        \
    } while (0)

// Bump allocator over a caller-provided device buffer (256-byte aligned
// pieces).  With base == nullptr it only measures.
struct Carver {
    char* base;
    size_t cap;
    size_t off = 0;
    Carver(void* b, size_t c) : base(static_cast<char*>(b)), cap(c) {}
    template <typename T>
    T* take(size_t count)
    {
        off = (off + 255) & ~static_cast<size_t>(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
    bool fits() const { return off <= cap; }
};

int g_num_sms = 0;

// test hook (slq_debug_fail_stream_waits): streaming launches left whose
// first wait is to run out at once
std::atomic<int> g_fail_stream_waits{0};
// test hook (slq_debug_blocks_sorted_keys): build block unions by sorting
// (block, column) keys even where the bitmap path applies
std::atomic<int> g_blk_sorted_keys{0};

slq_status device_sms(int* sms)
{
    if (g_num_sms == 0)
    {
        int dev = 0;
        SLQ_CK(cudaGetDevice(&dev));
        SLQ_CK(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    *sms = g_num_sms;
    return SLQ_OK;
}

inline bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

inline int next_pow2(int x)
{
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

inline size_t dsize(int dtype) { return dtype == SLQ_F64 ? 8 : 4; }

// A small read of device memory into pageable host memory, issued once the
// stream's work has finished.  A pageable read queued behind running kernels
// holds the calling thread in the driver until they end, and another host
// thread's page-locked upload (the values' upload beside the operator's
// set-up) was measured waiting behind it for the kernels' whole duration.
inline cudaError_t read_back(void* host, const void* dev, size_t bytes, cudaStream_t st)
{
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

// Per-kernel event timing (slq_profile_begin / slq_profile_end).
struct ProfRecord {
    int kind;
    cudaEvent_t start, stop;
    double bytes;
};

struct Profiler {
    bool on = false;
    std::vector<ProfRecord> records;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    cudaEvent_t next_event()
    {
        if (used == pool.size())
        {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            pool.push_back(e);
        }
        return pool[used++];
    }
};

thread_local Profiler g_prof;

// Brackets one launch with events when profiling is on.
struct ProfScope {
    int kind;
    double bytes;
    cudaStream_t st;
    cudaEvent_t start = nullptr;
    ProfScope(int k, double by, cudaStream_t s) : kind(k), bytes(by), st(s)
    {
        if (g_prof.on)
        {
            start = g_prof.next_event();
            if (start) cudaEventRecord(start, st);
        }
    }
    ~ProfScope()
    {
        if (g_prof.on && start)
        {
            cudaEvent_t stop = g_prof.next_event();
            if (stop)
            {
                cudaEventRecord(stop, st);
                g_prof.records.push_back({kind, start, stop, bytes});
            }
        }
    }
};

}  // namespace

extern "C" slq_status slq_profile_begin(void)
{
    g_prof.records.clear();
    g_prof.used = 0;
    g_prof.on = true;
    return SLQ_OK;
}

extern "C" slq_status slq_profile_end(slq_kernel_stat* stats)
{
    if (!stats) return fail(SLQ_ERR_BAD_ARG, "profile_end: stats is NULL");
    for (int k = 0; k < SLQ_K_COUNT; ++k) stats[k] = {0, 0.0, 0.0};
    g_prof.on = false;
    if (!g_prof.records.empty())
        SLQ_CK(cudaEventSynchronize(g_prof.records.back().stop));
    for (const ProfRecord& r : g_prof.records)
    {
        float ms = 0.0f;
        SLQ_CK(cudaEventElapsedTime(&ms, r.start, r.stop));
        stats[r.kind].launches += 1;
        stats[r.kind].milliseconds += ms;
        stats[r.kind].bytes += r.bytes;
    }
    g_prof.records.clear();
    g_prof.used = 0;
    return SLQ_OK;
}


// ---------------------------------------------------------------------------
// operator
// ---------------------------------------------------------------------------

struct slq_op {
    int dtype;
    int affine;
    int64_t nrows, ncols, nnz;
    // CSR of A (rows = nrows) and CSR of A^T (rows = ncols)
    const void* a_data = nullptr;
    const int32_t* a_ind = nullptr;
    const int32_t* a_ptr = nullptr;
    const void* t_data = nullptr;
    const int32_t* t_ind = nullptr;
    const int32_t* t_ptr = nullptr;
    // symmetric locality permutation: probe element e lives in row inv[e]
    const int32_t* inv = nullptr;
    // row-group format (0 = none) of A and of A^T
    int group_rows = 0;
    const int32_t* a_gptr = nullptr;
    const int32_t* a_gcol = nullptr;
    const void* a_gval = nullptr;
    const int32_t* t_gptr = nullptr;
    const int32_t* t_gcol = nullptr;
    const void* t_gval = nullptr;
    // dense FP32 operator (tensor-core product): TF32 parts of A, [nrows][ldk],
    // and of A^T, [ncols][ldk_t], K-major with zero-padded pitches; the
    // probe-block parts scratch [256][ldx]; running totals of split products
    // (dense_ksplit of the SM count at creation); TMA maps of the A parts
    int dense = 0;
    float* d_acc = nullptr;
    int dense_sms = 0;
    float* d_hi = nullptr;
    float* d_lo = nullptr;
    float* dt_hi = nullptr;
    float* dt_lo = nullptr;
    int64_t ldk = 0, ldk_t = 0, ldx = 0;
    float* xt_hi = nullptr;
    float* xt_lo = nullptr;
    int32_t* d_error = nullptr;
    CUtensorMap map_hi, map_lo, map_t_hi, map_t_lo;
    // tensor-core block format (k_spmm_blk, FP32 operators) of A and of A^T:
    // 128-row blocks, first stage per block, union columns, row scales,
    // FP16 stage images
    int64_t a_nblk = 0, t_nblk = 0;
    int64_t a_stages = 0, t_stages = 0;  // 16-column stages of the block formats
    const int32_t* a_bstage = nullptr;
    const int32_t* a_ucol = nullptr;
    const float* a_rsc = nullptr;
    const __half* a_img = nullptr;
    const int32_t* t_bstage = nullptr;
    const int32_t* t_ucol = nullptr;
    const float* t_rsc = nullptr;
    const __half* t_img = nullptr;
    const int32_t* a_order = nullptr;
    const int32_t* t_order = nullptr;
    // slq_operator_dot's error word and per-probe maxima of X for the block
    // kernel (inside the first format buffer)
    int32_t* blk_error = nullptr;
    unsigned int* blk_xmax = nullptr;
    // the scratch slq_operator_blocks_bytes prepared per direction (sorted
    // keys, unions, stages) and its stage count, so that
    // slq_operator_add_blocks on the same scratch does not sort again
    const void* blk_prep_scratch[2] = {nullptr, nullptr};
    int64_t blk_prep_stages[2] = {0, 0};
    bool blk_prep_bitmap[2] = {false, false};
    // autotuned SpMM candidate per direction and log2(block width); -1 = built-in
    int8_t tuned[2][11];
    slq_op()
    {
        for (auto& d : tuned)
            for (auto& v : d) v = -1;
    }
};

namespace {

// Plan of the transpose of an R x C CSR matrix into caller memory.
struct TransposeBufs {
    int32_t* t_ptr;
    int32_t* t_ind;
    void* t_data;
    int32_t* row_of;
    int32_t* keys_out;
    int32_t* iota;
    int32_t* perm;
    void* temp;
    size_t temp_bytes;
};

slq_status transpose_layout(Carver& c, int64_t R, int64_t C, int64_t nnz,
                            int dtype, TransposeBufs* t)
{
    size_t temp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, temp_bytes, static_cast<const int32_t*>(nullptr),
        static_cast<int32_t*>(nullptr), static_cast<const int32_t*>(nullptr),
        static_cast<int32_t*>(nullptr), static_cast<int>(std::max<int64_t>(nnz, 1)));
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub sort sizing: ") + cudaGetErrorString(e));
    t->t_ptr = c.take<int32_t>(C + 1);
    t->t_ind = c.take<int32_t>(nnz);
    t->t_data = c.take<char>(nnz * dsize(dtype));
    t->row_of = c.take<int32_t>(nnz);
    t->keys_out = c.take<int32_t>(nnz);
    t->iota = c.take<int32_t>(nnz);
    t->perm = c.take<int32_t>(nnz);
    t->temp = c.take<char>(temp_bytes);
    t->temp_bytes = temp_bytes;
    (void)R;
    return SLQ_OK;
}

// Deterministic transpose: stable radix sort of (column, position) pairs
// keeps the original row order inside every output row.
slq_status transpose_csr(const int32_t* ptr, const int32_t* ind, const void* data,
                         int64_t R, int64_t C, int64_t nnz, int dtype,
                         TransposeBufs* t, cudaStream_t st)
{
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int grid = sms * 4;
    if (nnz > 0)
    {
        k_row_ids<<<grid, 256, 0, st>>>(ptr, R, t->row_of);
        SLQ_LAUNCH_CK();
        k_iota<<<grid, 256, 0, st>>>(t->iota, nnz);
        SLQ_LAUNCH_CK();
        int end_bit = 1;
        while ((int64_t(1) << end_bit) <= C && end_bit < 31) ++end_bit;
        size_t tb = t->temp_bytes;
        cudaError_t e = cub::DeviceRadixSort::SortPairs(
            t->temp, tb, ind, t->keys_out, t->iota, t->perm,
            static_cast<int>(nnz), 0, end_bit, st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub sort: ") + cudaGetErrorString(e));
        if (dtype == SLQ_F64)
            k_gather_transpose<double><<<grid, 256, 0, st>>>(
                t->perm, t->row_of, static_cast<const double*>(data), nnz, t->t_ind,
                static_cast<double*>(t->t_data));
        else
            k_gather_transpose<float><<<grid, 256, 0, st>>>(
                t->perm, t->row_of, static_cast<const float*>(data), nnz, t->t_ind,
                static_cast<float*>(t->t_data));
        SLQ_LAUNCH_CK();
    }
    k_bounds<<<std::max<int64_t>(1, std::min<int64_t>(grid, (C + 256) / 256)), 256, 0, st>>>(
        t->keys_out, nnz, C, t->t_ptr);
    SLQ_LAUNCH_CK();
    return SLQ_OK;
}

struct PermBufs {
    int32_t* inv;
    int32_t* p_ptr;
    int32_t* p_ind;
    void* p_data;
    uint64_t* keys_in;
    uint64_t* keys_out;
    int32_t* pos_in;
    int32_t* pos_out;
    int32_t* deg;       // [n + 1] row lengths in B's order
    int32_t* flag;      // [4]: largest row length
    void* temp;
    size_t temp_bytes;
};

slq_status perm_layout(Carver& c, int64_t n, int64_t nnz, int dtype, PermBufs* t)
{
    size_t temp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, temp_bytes, static_cast<const uint64_t*>(nullptr),
        static_cast<uint64_t*>(nullptr), static_cast<const int32_t*>(nullptr),
        static_cast<int32_t*>(nullptr), static_cast<int>(std::max<int64_t>(nnz, 1)));
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub sort sizing: ") + cudaGetErrorString(e));
    size_t scan_bytes = 0;
    e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<const int32_t*>(nullptr),
                                      static_cast<int32_t*>(nullptr),
                                      static_cast<int>(n + 1));
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub scan sizing: ") + cudaGetErrorString(e));
    temp_bytes = std::max(temp_bytes, scan_bytes);
    t->inv = c.take<int32_t>(n);
    t->p_ptr = c.take<int32_t>(n + 1);
    t->deg = c.take<int32_t>(n + 1);
    t->flag = c.take<int32_t>(4);
    t->p_ind = c.take<int32_t>(nnz);
    t->p_data = c.take<char>(nnz * dsize(dtype));
    t->keys_in = c.take<uint64_t>(nnz);
    t->keys_out = c.take<uint64_t>(nnz);
    t->pos_in = c.take<int32_t>(nnz);
    t->pos_out = c.take<int32_t>(nnz);
    t->temp = c.take<char>(temp_bytes);
    t->temp_bytes = temp_bytes;
    return SLQ_OK;
}

// B = P A P^T with B[i][j] = A[perm[i]][perm[j]]: sort (new row, new column)
// keys; rows of B come out with ascending column indices.
slq_status permute_csr(const int32_t* ptr, const int32_t* ind, const void* data,
                       const int32_t* perm, int64_t n, int64_t nnz, int dtype,
                       PermBufs* t, cudaStream_t st)
{
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int grid = sms * 4;
    k_inverse_perm<<<grid, 256, 0, st>>>(perm, n, t->inv);
    SLQ_LAUNCH_CK();
    // rows of at most PERM_ROW_MAX entries: each row relabelled and sorted in
    // one warp (no global sort); else one radix sort of (row, column) keys
    SLQ_CK(cudaMemsetAsync(t->flag, 0, sizeof(int32_t), st));
    k_perm_deg<<<grid, 256, 0, st>>>(ptr, perm, n, t->deg, t->flag);
    SLQ_LAUNCH_CK();
    int32_t maxdeg = 0;
    SLQ_CK(read_back(&maxdeg, t->flag, sizeof(int32_t), st));
    if (maxdeg <= PERM_ROW_MAX)
    {
        size_t tb = t->temp_bytes;
        cudaError_t e = cub::DeviceScan::ExclusiveSum(t->temp, tb, t->deg, t->p_ptr,
                                                      static_cast<int>(n + 1), st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub scan: ") + cudaGetErrorString(e));
        if (nnz > 0)
        {
            const int rg = static_cast<int>(std::min<int64_t>((n + PERM_WARPS - 1) / PERM_WARPS,
                                                              int64_t(sms) * 16));
            if (dtype == SLQ_F64)
                k_perm_rows<double><<<rg, PERM_WARPS * 32, 0, st>>>(
                    ptr, ind, static_cast<const double*>(data), perm, t->inv, t->p_ptr, n,
                    t->p_ind, static_cast<double*>(t->p_data));
            else
                k_perm_rows<float><<<rg, PERM_WARPS * 32, 0, st>>>(
                    ptr, ind, static_cast<const float*>(data), perm, t->inv, t->p_ptr, n,
                    t->p_ind, static_cast<float*>(t->p_data));
            SLQ_LAUNCH_CK();
        }
        return SLQ_OK;
    }
    if (nnz > 0)
    {
        k_perm_keys<<<grid, 256, 0, st>>>(ptr, ind, t->inv, n, t->keys_in, t->pos_in);
        SLQ_LAUNCH_CK();
        int bits = 1;
        while ((int64_t(1) << bits) <= n && bits < 31) ++bits;
        size_t tb = t->temp_bytes;
        cudaError_t e = cub::DeviceRadixSort::SortPairs(
            t->temp, tb, t->keys_in, t->keys_out, t->pos_in, t->pos_out,
            static_cast<int>(nnz), 0, 32 + bits, st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub sort: ") + cudaGetErrorString(e));
        if (dtype == SLQ_F64)
            k_perm_gather<double><<<grid, 256, 0, st>>>(
                t->keys_out, t->pos_out, static_cast<const double*>(data), nnz, t->p_ind,
                static_cast<double*>(t->p_data));
        else
            k_perm_gather<float><<<grid, 256, 0, st>>>(
                t->keys_out, t->pos_out, static_cast<const float*>(data), nnz, t->p_ind,
                static_cast<float*>(t->p_data));
        SLQ_LAUNCH_CK();
    }
    k_bounds64<<<std::max<int64_t>(1, std::min<int64_t>(grid, (n + 256) / 256)), 256, 0, st>>>(
        t->keys_out, nnz, n, t->p_ptr);
    SLQ_LAUNCH_CK();
    return SLQ_OK;
}

struct GroupBufs {
    int32_t* counts;
    int32_t* gptr;
    int32_t* gcol;
    void* gval;
    void* temp;
    size_t temp_bytes;
};

// Union entries never exceed nnz, so the format fits in nnz (col + G values).
slq_status group_layout(Carver& c, int64_t rows, int64_t nnz, int G, int dtype, GroupBufs* t)
{
    const int64_t ng = (rows + G - 1) / G;
    size_t temp_bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes,
                                                  static_cast<const int32_t*>(nullptr),
                                                  static_cast<int32_t*>(nullptr),
                                                  static_cast<int>(ng + 1));
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub scan sizing: ") + cudaGetErrorString(e));
    t->counts = c.take<int32_t>(ng + 1);
    t->gptr = c.take<int32_t>(ng + 1);
    t->gcol = c.take<int32_t>(std::max<int64_t>(nnz, 1));
    t->gval = c.take<char>(std::max<int64_t>(nnz, 1) * G * dsize(dtype));
    t->temp = c.take<char>(temp_bytes);
    t->temp_bytes = temp_bytes;
    return SLQ_OK;
}

slq_status group_build(const int32_t* ptr, const int32_t* ind, const void* val, int64_t rows,
                       int G, int dtype, GroupBufs* t, cudaStream_t st)
{
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int64_t ng = (rows + G - 1) / G;
    SLQ_CK(cudaMemsetAsync(t->counts, 0, sizeof(int32_t) * (ng + 1), st));
    k_rg_count<<<sms * 8, 256, 0, st>>>(ptr, ind, rows, G, t->counts, ng);
    SLQ_LAUNCH_CK();
    size_t tb = t->temp_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(t->temp, tb, t->counts, t->gptr,
                                                  static_cast<int>(ng + 1), st);
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub scan: ") + cudaGetErrorString(e));
    if (dtype == SLQ_F64)
        k_rg_fill<double><<<sms * 8, 256, 0, st>>>(ptr, ind, static_cast<const double*>(val),
                                                   rows, G, t->gptr, t->gcol,
                                                   static_cast<double*>(t->gval), ng);
    else
        k_rg_fill<float><<<sms * 8, 256, 0, st>>>(ptr, ind, static_cast<const float*>(val), rows,
                                                  G, t->gptr, t->gcol,
                                                  static_cast<float*>(t->gval), ng);
    SLQ_LAUNCH_CK();
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_operator_workspace_bytes(int64_t num_rows, int64_t num_cols,
                                                   int64_t nnz, int dtype, int format,
                                                   int need_transpose, int has_perm,
                                                   int group_rows, size_t* bytes)
{
    if (group_rows != 0 && group_rows != 4 && group_rows != 8 && group_rows != 16)
        return fail(SLQ_ERR_BAD_ARG, "group_rows must be 0, 4, 8 or 16");
    if (!bytes || num_rows < 0 || num_cols < 0 || nnz < 0)
        return fail(SLQ_ERR_BAD_ARG, "operator_workspace_bytes: bad argument");
    if (has_perm && (format != SLQ_CSR || num_rows != num_cols))
        return fail(SLQ_ERR_BAD_ARG, "a permutation needs a square CSR matrix");
    Carver c(nullptr, 0);
    TransposeBufs t;
    PermBufs pb;
    c.take<int32_t>(1);  // index-check flag
    if (has_perm) SLQ_TRY(perm_layout(c, num_rows, nnz, dtype, &pb));
    const bool build = (format == SLQ_CSC) || need_transpose;
    if (build)
    {
        const int64_t R = (format == SLQ_CSC) ? num_cols : num_rows;
        const int64_t C = (format == SLQ_CSC) ? num_rows : num_cols;
        SLQ_TRY(transpose_layout(c, R, C, nnz, dtype, &t));
    }
    if (group_rows)
    {
        GroupBufs g;
        SLQ_TRY(group_layout(c, num_rows, nnz, group_rows, dtype, &g));
        if (need_transpose || format == SLQ_CSC)
            SLQ_TRY(group_layout(c, num_cols, nnz, group_rows, dtype, &g));
    }
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_operator_create(const void* data, const int32_t* indices,
                                          const int32_t* indptr, int64_t num_rows,
                                          int64_t num_cols, int64_t nnz, int dtype,
                                          int format, int affine, int need_transpose,
                                          int check_indices, const int32_t* perm,
                                          int group_rows, void* workspace,
                                          size_t workspace_bytes, void* stream, slq_op** out)
{
    if (!out) return fail(SLQ_ERR_BAD_ARG, "operator_create: out is NULL");
    *out = nullptr;
    if (dtype != SLQ_F32 && dtype != SLQ_F64)
        return fail(SLQ_ERR_BAD_ARG, "operator_create: dtype must be SLQ_F32 or SLQ_F64");
    if (format != SLQ_CSR && format != SLQ_CSC)
        return fail(SLQ_ERR_BAD_ARG, "operator_create: format must be SLQ_CSR or SLQ_CSC");
    if (num_rows <= 0 || num_cols <= 0 || nnz < 0 || nnz > INT32_MAX ||
        num_rows > INT32_MAX || num_cols > INT32_MAX)
        return fail(SLQ_ERR_BAD_ARG, "operator_create: sizes out of range (int32 indices)");
    if (!indptr || (nnz > 0 && (!indices || !data)))
        return fail(SLQ_ERR_BAD_ARG, "operator_create: NULL array");
    size_t need = 0;
    SLQ_TRY(slq_operator_workspace_bytes(num_rows, num_cols, nnz, dtype, format,
                                         need_transpose, perm != nullptr, group_rows, &need));
    if (!workspace || workspace_bytes < need)
        return fail(SLQ_ERR_WORKSPACE, "operator_create: workspace too small (need " +
                                           std::to_string(need) + " bytes)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Carver c(workspace, workspace_bytes);
    int32_t* flag = c.take<int32_t>(1);

    // stored arrays: CSR over `srows` rows, `scols` columns
    const int64_t srows = (format == SLQ_CSC) ? num_cols : num_rows;
    const int64_t scols = (format == SLQ_CSC) ? num_rows : num_cols;
    if (check_indices)
    {
        int sms = 0;
        SLQ_TRY(device_sms(&sms));
        SLQ_CK(cudaMemsetAsync(flag, 0, sizeof(int32_t), st));
        k_check_csr<<<sms * 4, 256, 0, st>>>(indptr, indices, srows, scols, nnz, flag);
        SLQ_LAUNCH_CK();
        int32_t h = 0;
        SLQ_CK(read_back(&h, flag, sizeof(int32_t), st));
        if (h & 1) return fail(SLQ_ERR_BAD_CSR, "index pointer must start at 0 and end at nnz");
        if (h & 2) return fail(SLQ_ERR_BAD_CSR, "index pointer must be non-decreasing");
        if (h & 4) return fail(SLQ_ERR_BAD_CSR, "index out of range");
    }

    slq_op* op = new slq_op();
    op->dtype = dtype;
    op->affine = affine;
    op->nrows = num_rows;
    op->ncols = num_cols;
    op->nnz = nnz;
    const void* src_data = data;
    const int32_t* src_ind = indices;
    const int32_t* src_ptr = indptr;
    if (perm)
    {
        PermBufs pb;
        slq_status s = perm_layout(c, num_rows, nnz, dtype, &pb);
        if (s == SLQ_OK)
            s = permute_csr(indptr, indices, data, perm, num_rows, nnz, dtype, &pb, st);
        if (s != SLQ_OK)
        {
            delete op;
            return s;
        }
        src_data = pb.p_data;
        src_ind = pb.p_ind;
        src_ptr = pb.p_ptr;
        op->inv = pb.inv;
    }
    const bool build = (format == SLQ_CSC) || need_transpose;
    TransposeBufs t;
    if (build)
    {
        slq_status s = transpose_layout(c, srows, scols, nnz, dtype, &t);
        if (s == SLQ_OK)
            s = transpose_csr(src_ptr, src_ind, src_data, srows, scols, nnz, dtype, &t, st);
        if (s != SLQ_OK)
        {
            delete op;
            return s;
        }
    }
    if (format == SLQ_CSR)
    {
        op->a_data = src_data;
        op->a_ind = src_ind;
        op->a_ptr = src_ptr;
        if (build)
        {
            op->t_data = t.t_data;
            op->t_ind = t.t_ind;
            op->t_ptr = t.t_ptr;
        }
    }
    else
    {   // CSC arrays are the CSR of A^T; their transpose is the CSR of A
        op->t_data = data;
        op->t_ind = indices;
        op->t_ptr = indptr;
        op->a_data = t.t_data;
        op->a_ind = t.t_ind;
        op->a_ptr = t.t_ptr;
    }
    if (group_rows)
    {
        GroupBufs ga;
        slq_status s = group_layout(c, num_rows, nnz, group_rows, dtype, &ga);
        if (s == SLQ_OK)
            s = group_build(op->a_ptr, op->a_ind, op->a_data, num_rows, group_rows, dtype, &ga,
                            st);
        if (s == SLQ_OK && op->t_ptr)
        {
            GroupBufs gt;
            s = group_layout(c, num_cols, nnz, group_rows, dtype, &gt);
            if (s == SLQ_OK)
                s = group_build(op->t_ptr, op->t_ind, op->t_data, num_cols, group_rows, dtype,
                                &gt, st);
            op->t_gptr = gt.gptr;
            op->t_gcol = gt.gcol;
            op->t_gval = gt.gval;
        }
        if (s != SLQ_OK)
        {
            delete op;
            return s;
        }
        op->group_rows = group_rows;
        op->a_gptr = ga.gptr;
        op->a_gcol = ga.gcol;
        op->a_gval = ga.gval;
    }
    *out = op;
    return SLQ_OK;
}

extern "C" slq_status slq_operator_destroy(slq_op* op)
{
    delete op;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// tensor-core block format (k_spmm_blk)
// ---------------------------------------------------------------------------

namespace {

struct BlkScratch {
    uint64_t* keys_in;
    uint64_t* keys_out;
    int32_t* pos_in;
    int32_t* pos_out;
    uint8_t* rr;
    int32_t* flags;
    int32_t* uidx;
    int32_t* cnt;     // [nblk + 1]
    int32_t* stg;     // [nblk + 1]
    int32_t* bstage;  // [nblk + 1]
    int32_t* ufirst;  // [nblk + 1]
    float* fsc;       // [nblk * 128] row scales 2^f_r
    void* temp;
    size_t temp_bytes;
};

int bits_for(int64_t v)  // bits to hold 0 .. v
{
    int b = 1;
    while (b < 63 && (int64_t(1) << b) <= v) ++b;
    return b;
}

slq_status blk_scratch_layout(Carver& c, int64_t rows, int64_t nnz, BlkScratch* s)
{
    const int64_t nblk = (rows + BLK_ROWS - 1) / BLK_ROWS;
    const int nz = static_cast<int>(std::max<int64_t>(nnz, 1));
    size_t t1 = 0, t2 = 0, t3 = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, t1, static_cast<const uint64_t*>(nullptr), static_cast<uint64_t*>(nullptr),
        static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr), nz);
    if (e == cudaSuccess)
        e = cub::DeviceScan::InclusiveSum(nullptr, t2, static_cast<const int32_t*>(nullptr),
                                          static_cast<int32_t*>(nullptr), nz);
    if (e == cudaSuccess)
        e = cub::DeviceScan::ExclusiveSum(nullptr, t3, static_cast<const int32_t*>(nullptr),
                                          static_cast<int32_t*>(nullptr),
                                          static_cast<int>(nblk + 1));
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub sizing (blocks): ") + cudaGetErrorString(e));
    s->keys_in = c.take<uint64_t>(nz);
    s->keys_out = c.take<uint64_t>(nz);
    s->pos_in = c.take<int32_t>(nz);
    s->pos_out = c.take<int32_t>(nz);
    s->rr = c.take<uint8_t>(nz);
    s->flags = c.take<int32_t>(nz);
    s->uidx = c.take<int32_t>(nz);
    s->cnt = c.take<int32_t>(nblk + 1);
    s->stg = c.take<int32_t>(nblk + 1);
    s->bstage = c.take<int32_t>(nblk + 1);
    s->ufirst = c.take<int32_t>(nblk + 1);
    s->fsc = c.take<float>(nblk * BLK_ROWS);
    s->temp_bytes = std::max({t1, t2, t3});
    s->temp = c.take<char>(s->temp_bytes);
    return SLQ_OK;
}

// Union sizes and first stages of the 128-row blocks of an R x C CSR
// matrix in the scratch, by per-block bitmaps (*bitmap = true) or, where a
// block's columns span too far, by sorted (block, column) keys; *stages
// receives the total (host synchronisation).
slq_status blk_prepare(const int32_t* ptr, const int32_t* ind, int64_t R, int64_t C, int64_t nnz,
                       BlkScratch* s, cudaStream_t st, int64_t* stages, bool* bitmap)
{
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int grid = sms * 4;
    const int64_t nblk = (R + BLK_ROWS - 1) / BLK_ROWS;
    const int cbits = bits_for(std::max<int64_t>(C - 1, 1));
    const int bbits = bits_for(std::max<int64_t>(nblk - 1, 1));
    SLQ_CK(cudaMemsetAsync(s->cnt, 0, sizeof(int32_t) * (nblk + 1), st));
    *bitmap = false;
    if (nnz > 0 && nblk > 0 && g_blk_sorted_keys.load() == 0)
    {
        // the word that flags a block too wide for its bitmap (the flags
        // array is free on this path)
        SLQ_CK(cudaMemsetAsync(s->flags, 0, sizeof(int32_t), st));
        k_blk_ucount<<<static_cast<int>(std::min<int64_t>(nblk, int64_t(sms) * 6)),
                       BLK_UNION_THREADS, 0, st>>>(ptr, ind, R, nblk, s->cnt, s->flags);
        SLQ_LAUNCH_CK();
        int32_t wide = 0;
        SLQ_CK(read_back(&wide, s->flags, sizeof(int32_t), st));
        *bitmap = wide == 0;
        if (!*bitmap) SLQ_CK(cudaMemsetAsync(s->cnt, 0, sizeof(int32_t) * (nblk + 1), st));
    }
    if (nnz > 0 && !*bitmap)
    {
        k_blk_keys<<<grid, 256, 0, st>>>(ptr, ind, R, cbits, s->keys_in, s->pos_in, s->rr);
        SLQ_LAUNCH_CK();
        size_t tb = s->temp_bytes;
        cudaError_t e = cub::DeviceRadixSort::SortPairs(s->temp, tb, s->keys_in, s->keys_out,
                                                        s->pos_in, s->pos_out,
                                                        static_cast<int>(nnz), 0, cbits + bbits,
                                                        st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub sort (blocks): ") + cudaGetErrorString(e));
        k_blk_flags<<<grid, 256, 0, st>>>(s->keys_out, nnz, s->flags);
        SLQ_LAUNCH_CK();
        tb = s->temp_bytes;
        e = cub::DeviceScan::InclusiveSum(s->temp, tb, s->flags, s->uidx, static_cast<int>(nnz),
                                          st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub scan (blocks): ") + cudaGetErrorString(e));
        k_blk_count<<<grid, 256, 0, st>>>(s->keys_out, s->flags, nnz, cbits, s->cnt);
        SLQ_LAUNCH_CK();
    }
    k_blk_stages<<<std::max<int64_t>(1, std::min<int64_t>(grid, (nblk + 256) / 256)), 256, 0,
                   st>>>(s->cnt, nblk, s->stg);
    SLQ_LAUNCH_CK();
    size_t tb = s->temp_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(s->temp, tb, s->stg, s->bstage,
                                                  static_cast<int>(nblk + 1), st);
    if (e == cudaSuccess)
    {
        tb = s->temp_bytes;
        e = cub::DeviceScan::ExclusiveSum(s->temp, tb, s->cnt, s->ufirst,
                                          static_cast<int>(nblk + 1), st);
    }
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub scan (blocks): ") + cudaGetErrorString(e));
    int32_t total = 0;
    SLQ_CK(read_back(&total, s->bstage + nblk, sizeof(int32_t), st));
    *stages = total;
    return SLQ_OK;
}

struct BlkFormat {
    int32_t* error;
    unsigned int* xmax;  // [256]
    int32_t* bstage;
    int32_t* order;      // [nblk] block of each slot of the kernel's waves
    int32_t* ucol;
    float* rsc;
    __half* img;
};

void blk_format_layout(Carver& c, int64_t nblk, int64_t stages, BlkFormat* f)
{
    f->error = c.take<int32_t>(1);
    f->xmax = c.take<unsigned int>(256);
    f->bstage = c.take<int32_t>(nblk + 1);
    f->order = c.take<int32_t>(nblk);
    f->ucol = c.take<int32_t>(stages * BLK_BK);
    f->rsc = c.take<float>(nblk * BLK_ROWS);
    f->img = c.take<__half>(stages * BLK_IMG_STAGE);
}

// The slot order of the block SpMM's G CTAs (CTA c takes slots c, c + G,
// ...): wave w = slots w G .. w G + G - 1 holds blocks w G .. w G + G - 1,
// consecutive blocks so that a wave's X rows stay in L2, and within each
// wave the blocks with the most stages go to the CTAs with the least work
// so far (longest first onto the least loaded).  The last, partial wave can
// only use CTAs 0 .. rem - 1; it is dealt first.  Deterministic.
void blk_balance(const int32_t* bstage, int64_t nblk, int G, int32_t* order)
{
    if (nblk <= 0) return;
    G = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(G, nblk)));
    const int64_t W = (nblk + G - 1) / G;
    std::vector<int64_t> load(static_cast<size_t>(G), 0);
    std::vector<int32_t> blocks, ctas;
    auto deal = [&](int64_t w) {
        const int64_t b0 = w * G, b1 = std::min<int64_t>(nblk, b0 + G);
        const int n = static_cast<int>(b1 - b0);
        blocks.resize(static_cast<size_t>(n));
        ctas.resize(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) blocks[i] = static_cast<int32_t>(b0 + i);
        for (int i = 0; i < n; ++i) ctas[i] = i;
        std::sort(blocks.begin(), blocks.end(), [&](int32_t x, int32_t y) {
            const int sx = bstage[x + 1] - bstage[x], sy = bstage[y + 1] - bstage[y];
            return sx != sy ? sx > sy : x < y;
        });
        std::sort(ctas.begin(), ctas.end(), [&](int32_t x, int32_t y) {
            return load[x] != load[y] ? load[x] < load[y] : x < y;
        });
        for (int i = 0; i < n; ++i)
        {
            order[b0 + ctas[i]] = blocks[i];
            load[ctas[i]] += bstage[blocks[i] + 1] - bstage[blocks[i]];
        }
    };
    if (nblk % G != 0) deal(W - 1);
    for (int64_t w = 0; w < ((nblk % G != 0) ? W - 1 : W); ++w) deal(w);
}

slq_status blk_source(const slq_op* op, int transpose, const int32_t** ptr, const int32_t** ind,
                      const float** val, int64_t* R, int64_t* C)
{
    if (!op) return fail(SLQ_ERR_BAD_ARG, "blocks: NULL operator");
    if (op->dense || op->dtype != SLQ_F32)
        return fail(SLQ_ERR_UNSUPPORTED, "blocks: the block format serves float32 sparse operators");
    if (transpose != 0 && transpose != 1)
        return fail(SLQ_ERR_BAD_ARG, "blocks: transpose must be 0 or 1");
    if (transpose && !op->t_ptr) return fail(SLQ_ERR_BAD_ARG, "blocks: operator has no transpose");
    *ptr = transpose ? op->t_ptr : op->a_ptr;
    *ind = transpose ? op->t_ind : op->a_ind;
    *val = static_cast<const float*>(transpose ? op->t_data : op->a_data);
    *R = transpose ? op->ncols : op->nrows;
    *C = transpose ? op->nrows : op->ncols;
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_operator_blocks_scratch_bytes(const slq_op* op, int transpose,
                                                        size_t* bytes)
{
    if (!bytes) return fail(SLQ_ERR_BAD_ARG, "blocks: bytes is NULL");
    const int32_t *ptr, *ind;
    const float* val;
    int64_t R, C;
    SLQ_TRY(blk_source(op, transpose, &ptr, &ind, &val, &R, &C));
    Carver c(nullptr, 0);
    BlkScratch s;
    SLQ_TRY(blk_scratch_layout(c, R, op->nnz, &s));
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_operator_blocks_bytes(const slq_op* op, int transpose, void* scratch,
                                                size_t scratch_bytes, void* stream,
                                                size_t* format_bytes)
{
    if (!format_bytes) return fail(SLQ_ERR_BAD_ARG, "blocks: format_bytes is NULL");
    const int32_t *ptr, *ind;
    const float* val;
    int64_t R, C;
    SLQ_TRY(blk_source(op, transpose, &ptr, &ind, &val, &R, &C));
    Carver c(scratch, scratch_bytes);
    BlkScratch s;
    SLQ_TRY(blk_scratch_layout(c, R, op->nnz, &s));
    if (!scratch || !c.fits()) return fail(SLQ_ERR_WORKSPACE, "blocks: scratch too small");
    int64_t stages = 0;
    bool bitmap = false;
    SLQ_TRY(blk_prepare(ptr, ind, R, C, op->nnz, &s, static_cast<cudaStream_t>(stream), &stages,
                        &bitmap));
    slq_op* mop = const_cast<slq_op*>(op);  // the preparation cache only
    mop->blk_prep_scratch[transpose] = scratch;
    mop->blk_prep_stages[transpose] = stages;
    mop->blk_prep_bitmap[transpose] = bitmap;
    Carver f(nullptr, 0);
    BlkFormat bf;
    blk_format_layout(f, (R + BLK_ROWS - 1) / BLK_ROWS, stages, &bf);
    *format_bytes = f.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_operator_add_blocks(slq_op* op, int transpose, void* scratch,
                                              size_t scratch_bytes, void* format,
                                              size_t format_bytes, void* stream)
{
    const int32_t *ptr, *ind;
    const float* val;
    int64_t R, C;
    SLQ_TRY(blk_source(op, transpose, &ptr, &ind, &val, &R, &C));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Carver c(scratch, scratch_bytes);
    BlkScratch s;
    SLQ_TRY(blk_scratch_layout(c, R, op->nnz, &s));
    if (!scratch || !c.fits()) return fail(SLQ_ERR_WORKSPACE, "blocks: scratch too small");
    int64_t stages = 0;
    bool bitmap = false;
    if (op->blk_prep_scratch[transpose] == scratch && scratch)
    {
        // prepared by slq_operator_blocks_bytes
        stages = op->blk_prep_stages[transpose];
        bitmap = op->blk_prep_bitmap[transpose];
    }
    else
        SLQ_TRY(blk_prepare(ptr, ind, R, C, op->nnz, &s, st, &stages, &bitmap));
    op->blk_prep_scratch[transpose] = nullptr;
    const int64_t nblk = (R + BLK_ROWS - 1) / BLK_ROWS;
    Carver f(format, format_bytes);
    BlkFormat bf;
    blk_format_layout(f, nblk, stages, &bf);
    if (!format || !f.fits())
        return fail(SLQ_ERR_WORKSPACE, "blocks: format buffer too small (need " +
                                           std::to_string(f.off) + " bytes)");
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int grid = sms * 4;
    const int cbits = bits_for(std::max<int64_t>(C - 1, 1));
    SLQ_CK(cudaMemcpyAsync(bf.bstage, s.bstage, sizeof(int32_t) * (nblk + 1),
                           cudaMemcpyDeviceToDevice, st));
    // the FP32 staging images take the same bytes as the FP16 parts
    SLQ_CK(cudaMemsetAsync(bf.img, 0, sizeof(__half) * stages * BLK_IMG_STAGE, st));
    k_blk_rowscale<<<grid, 256, 0, st>>>(ptr, val, R, nblk * BLK_ROWS, s.fsc, bf.rsc);
    SLQ_LAUNCH_CK();
    if (bitmap)
    {
        // union columns, padding and values of each block from its bitmap
        k_blk_ufill<<<static_cast<int>(std::min<int64_t>(nblk, int64_t(sms) * 6)),
                      BLK_UNION_THREADS, 0, st>>>(ptr, ind, val, R, nblk, bf.bstage, bf.ucol,
                                                  reinterpret_cast<float*>(bf.img));
        SLQ_LAUNCH_CK();
    }
    else
    {
        if (op->nnz > 0)
        {
            k_blk_ucol<<<grid, 256, 0, st>>>(s.keys_out, s.flags, s.uidx, op->nnz, cbits,
                                             s.ufirst, bf.bstage, bf.ucol);
            SLQ_LAUNCH_CK();
        }
        k_blk_pad<<<std::max<int64_t>(1, std::min<int64_t>(grid, (nblk + 255) / 256)), 256, 0,
                    st>>>(s.cnt, bf.bstage, nblk, bf.ucol);
        SLQ_LAUNCH_CK();
        if (op->nnz > 0)
        {
            k_blk_scatter<<<grid, 256, 0, st>>>(s.keys_out, s.pos_out, s.uidx, op->nnz, cbits,
                                                s.ufirst, bf.bstage, val, s.rr,
                                                reinterpret_cast<float*>(bf.img));
            SLQ_LAUNCH_CK();
        }
    }
    k_blk_split<<<std::max<int64_t>(1, std::min<int64_t>(stages, int64_t(sms) * 8)), 256, 0, st>>>(
        bf.img, bf.bstage, nblk, s.fsc, stages);
    SLQ_LAUNCH_CK();
    SLQ_CK(cudaMemsetAsync(bf.error, 0, sizeof(int32_t), st));
    // the scratch may be released once the build has run
    SLQ_CK(cudaStreamSynchronize(st));
    {
        // the kernel's slot order, balanced for this device's SM count
        std::vector<int32_t> hb(static_cast<size_t>(nblk + 1)), ho(static_cast<size_t>(nblk));
        SLQ_CK(read_back(hb.data(), bf.bstage, sizeof(int32_t) * (nblk + 1), st));
        blk_balance(hb.data(), nblk, sms, ho.data());
        if (nblk > 0)
            SLQ_CK(cudaMemcpyAsync(bf.order, ho.data(), sizeof(int32_t) * nblk,
                                   cudaMemcpyHostToDevice, st));
        SLQ_CK(cudaStreamSynchronize(st));  // ho is released on return
    }
    if (!op->blk_error)
    {
        op->blk_error = bf.error;
        op->blk_xmax = bf.xmax;
    }
    if (transpose)
    {
        op->t_nblk = nblk;
        op->t_stages = stages;
        op->t_bstage = bf.bstage;
        op->t_order = bf.order;
        op->t_ucol = bf.ucol;
        op->t_rsc = bf.rsc;
        op->t_img = bf.img;
    }
    else
    {
        op->a_nblk = nblk;
        op->a_stages = stages;
        op->a_bstage = bf.bstage;
        op->a_order = bf.order;
        op->a_ucol = bf.ucol;
        op->a_rsc = bf.rsc;
        op->a_img = bf.img;
    }
    return SLQ_OK;
}

extern "C" slq_status slq_operator_blocks_info(const slq_op* op, int transpose, int64_t* blocks,
                                               int64_t* stages)
{
    if (!op || !blocks || !stages) return fail(SLQ_ERR_BAD_ARG, "blocks_info: NULL argument");
    if (transpose != 0 && transpose != 1)
        return fail(SLQ_ERR_BAD_ARG, "blocks_info: transpose must be 0 or 1");
    *blocks = transpose ? op->t_nblk : op->a_nblk;
    *stages = transpose ? op->t_stages : op->a_stages;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------

namespace {

struct Launcher {
    cudaStream_t st;
    int sms;
    int64_t launches = 0;
};

template <typename VT, int LV, int KS>
slq_status spmm_inst(Launcher& L, int grid, const int32_t* ptr, const int32_t* ind,
                     const VT* vals, int64_t nrows, int b, const VT* X,
                     const double* sx, double shift, VT* Y, const VT* Z,
                     const double* zc, const double* zs, int epi, double* partials,
                     int64_t nnz, int64_t xrows)
{
    // compulsory traffic: matrix once, X once, Y written once, Z read once
    const double s = sizeof(VT);
    const double bytes = nnz * (s + 4.0) + (nrows + 1) * 4.0 + double(xrows) * b * s +
                         double(nrows) * b * s * (Z ? 2.0 : 1.0);
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    static bool attr = false;
    const size_t smem = (epi != 0) ? 8 * static_cast<size_t>(b) * sizeof(double) : 0;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_spmm<VT, LV, KS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        attr = true;
    }
    k_spmm<VT, LV, KS><<<grid, 256, smem, L.st>>>(ptr, ind, vals, nrows, b, X, sx, shift, Y, Z,
                                                  zc, zs, epi, partials);
    SLQ_LAUNCH_CK();
    ++L.launches;
    return SLQ_OK;
}

// blocks of k_spmm<VT, LV, KS> resident per SM (occupancy query, at most 4)
template <typename VT, int LV, int KS>
int spmm_blocks_per_sm(int b)
{
    static int cached = 0;
    if (cached == 0)
    {
        int v = 0;
        const size_t smem = 8 * static_cast<size_t>(b) * sizeof(double);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_spmm<VT, LV, KS>, 256, smem) !=
                cudaSuccess ||
            v < 1)
            v = 1;
        cached = std::min(v, 4);
    }
    return cached;
}

// persistent grid of the CSR kernel: as many blocks as are resident on the
// SMs at once (a partial second wave would leave SMs idle at the end)
template <typename VT>
int spmm_grid(const Launcher& L, int64_t nrows, int b)
{
    int per_sm = 4;
    switch (b)
    {
        case 64: per_sm = spmm_blocks_per_sm<VT, 2, 1>(b); break;
        case 128: per_sm = spmm_blocks_per_sm<VT, 4, 1>(b); break;
        case 256: per_sm = spmm_blocks_per_sm<VT, 8, 1>(b); break;
        case 512: per_sm = spmm_blocks_per_sm<VT, 16, 1>(b); break;
        case 1024: per_sm = spmm_blocks_per_sm<VT, 32, 1>(b); break;
        default: break;
    }
    const int64_t g = (nrows + 7) / 8;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, int64_t(L.sms) * per_sm)));
}

template <typename VT>
slq_status spmm(Launcher& L, int grid, const int32_t* ptr, const int32_t* ind, const VT* vals,
                int64_t nrows, int b, const VT* X, const double* sx, double shift, VT* Y,
                const VT* Z, const double* zc, const double* zs, int epi, double* partials,
                int64_t nnz, int64_t xrows)
{
#define SLQ_SPMM_CASE(BB, LV, KS)                                                         \
    case BB:                                                                              \
        return spmm_inst<VT, LV, KS>(L, grid, ptr, ind, vals, nrows, b, X, sx, shift, Y,  \
                                     Z, zc, zs, epi, partials, nnz, xrows);
    switch (b)
    {
        SLQ_SPMM_CASE(1, 1, 32)
        SLQ_SPMM_CASE(2, 1, 16)
        SLQ_SPMM_CASE(4, 1, 8)
        SLQ_SPMM_CASE(8, 1, 4)
        SLQ_SPMM_CASE(16, 1, 2)
        SLQ_SPMM_CASE(32, 1, 1)
        SLQ_SPMM_CASE(64, 2, 1)
        SLQ_SPMM_CASE(128, 4, 1)
        SLQ_SPMM_CASE(256, 8, 1)
        SLQ_SPMM_CASE(512, 16, 1)
        SLQ_SPMM_CASE(1024, 32, 1)
        default:
            return fail(SLQ_ERR_BAD_ARG, "block width must be a power of two <= 1024");
    }
#undef SLQ_SPMM_CASE
}

template <typename VT>
slq_status finalize(Launcher& L, const double* partials, int nparts, int cols, int mode,
                    double* out, VT* coef, const double* scales, int b, int bs, int last,
                    double* next_scale, int32_t* active, int32_t* size, int check_break,
                    double thr, int step)
{
    const int grid = (cols + 31) / 32;
    ProfScope prof(SLQ_K_FINALIZE, double(nparts) * cols * 8.0, L.st);
    k_finalize<VT><<<grid, 1024, 0, L.st>>>(partials, nparts, cols, mode, out, coef, scales, b,
                                           bs, last, next_scale, active, size, check_break, thr,
                                           step);
    SLQ_LAUNCH_CK();
    ++L.launches;
    return SLQ_OK;
}

// Tensor maps for the TMA row gathers of k_spmm_rgt: one per probe-block
// buffer, [rows][b] FP32, box = 128 values of one row (a warp's slice).
PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

slq_status row_map(CUtensorMap* m, const float* base, int64_t rows, int b)
{
    if (!g_encode_tiled)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SLQ_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess)
            return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(b), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(b) * sizeof(float)};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(std::min(b, 128)), 1};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode_tiled(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                const_cast<float*>(base), dims, strides, box, es,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return SLQ_OK;
}

// The tensor map of one probe-block buffer for the row gathers of the TMA
// and tensor-core row-group kernels (has_row = false: none), and, for the
// block SpMM, a buffer that receives the probe block split into FP16 parts
// (has_x16; x16_b probes per row).
struct XMaps {
    CUtensorMap row;
    bool has_row = false;
    __half* x16 = nullptr;
    int x16_b = 0;
    bool has_x16 = false;
    // x16 already holds this product's X, split by the pass that wrote X
    // with the exponents x16exp (else the product splits X first)
    bool x16_ready = false;
    const int32_t* x16exp = nullptr;
};

slq_status make_xmaps(XMaps* m, const float* base, int64_t rows, int b, bool row)
{
    if (row) SLQ_TRY(row_map(&m->row, base, rows, b));
    m->has_row = row;
    return SLQ_OK;
}


// ---------------------------------------------------------------------------
// dense FP32 operators (tensor-core product, k_dense_tc)
// ---------------------------------------------------------------------------


int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

struct DenseBufs {
    float *hi, *lo, *t_hi, *t_lo, *x_hi, *x_lo, *acc;
    int32_t* error;
    int64_t ldk, ldk_t, ldx;
};

// K parts per 128-row tile of an M x K dense product: when the row tiles
// fill at most half of the SMs, each tile's K range is split (on
// accumulation-chunk boundaries, at most 8 parts) so that more SMs work;
// the parts' FP32 totals are added by k_dense_epi.
int dense_ksplit(int64_t M, int64_t K, int sms)
{
    const int64_t ntm = (M + 127) / 128;
    const int64_t nch = ((K + DT_BK - 1) / DT_BK + DT_CHUNK - 1) / DT_CHUNK;
    if (ntm * 2 > sms) return 1;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({8, sms / ntm, nch})));
}

void dense_layout(Carver& c, int64_t rows, int64_t cols, int need_transpose, int sms,
                  DenseBufs* d)
{
    d->ldk = round_up(std::max<int64_t>(cols, 1), DT_BK);
    d->ldk_t = need_transpose ? round_up(std::max<int64_t>(rows, 1), DT_BK) : 0;
    d->ldx = std::max(d->ldk, d->ldk_t);
    d->hi = c.take<float>(static_cast<size_t>(rows) * d->ldk);
    d->lo = c.take<float>(static_cast<size_t>(rows) * d->ldk);
    d->t_hi = need_transpose ? c.take<float>(static_cast<size_t>(cols) * d->ldk_t) : nullptr;
    d->t_lo = need_transpose ? c.take<float>(static_cast<size_t>(cols) * d->ldk_t) : nullptr;
    d->x_hi = c.take<float>(static_cast<size_t>(256) * d->ldx);
    d->x_lo = c.take<float>(static_cast<size_t>(256) * d->ldx);
    // running totals of split products, for either direction
    int64_t acc_rows = dense_ksplit(rows, cols, sms) > 1 ? dense_ksplit(rows, cols, sms) * rows : 0;
    if (need_transpose && dense_ksplit(cols, rows, sms) > 1)
        acc_rows = std::max<int64_t>(acc_rows, dense_ksplit(cols, rows, sms) * cols);
    d->acc = acc_rows ? c.take<float>(static_cast<size_t>(acc_rows) * 256) : nullptr;
    d->error = c.take<int32_t>(1);
}

// K-major TF32-part tensor map: [outer][ld] FP32, box 32 x box_rows,
// SWIZZLE_128B (128-byte rows)
slq_status part_map(CUtensorMap* m, const float* base, int64_t ld, int64_t outer,
                    int box_rows)
{
    if (!g_encode_tiled)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SLQ_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess)
            return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(outer)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * sizeof(float)};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(DT_BK), static_cast<cuuint32_t>(box_rows)};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode_tiled(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base),
                                dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled (dense) failed (" +
                                      std::to_string(int(r)) + ")");
    return SLQ_OK;
}

size_t dense_smem(int NB)
{
    const size_t stage = 2 * 128 * DT_BK * 4 + 2 * static_cast<size_t>(NB) * DT_BK * 4;
    return 1023 + DT_STAGES * stage + 128 + 4 * 256 * sizeof(double);
}

// Y = A X (transpose: A^T X) on a dense operator, the SpMM epilogue fused;
// at most 256 probes per GEMM launch.  *grid_out = the partial rows.
slq_status dense_spmm(Launcher& L, const slq_op* op, int transpose, int b, const float* X,
                      const double* sx, double shift, float* Y, const float* Z,
                      const double* zc, const double* zs, int epi, double* partials,
                      int* grid_out, int32_t* error)
{
    if (transpose && !op->dt_hi)
        return fail(SLQ_ERR_BAD_ARG, "dense operator has no transpose");
    const int64_t M = transpose ? op->ncols : op->nrows;
    const int64_t K = transpose ? op->nrows : op->ncols;
    const CUtensorMap& ahi = transpose ? op->map_t_hi : op->map_hi;
    const CUtensorMap& alo = transpose ? op->map_t_lo : op->map_lo;
    const int64_t ntm = (M + 127) / 128;
    // split K when the row tiles leave most SMs idle (the same choice as the
    // scratch was sized for)
    const int ksplit = op->d_acc ? dense_ksplit(M, K, op->dense_sms) : 1;
    static bool attr = false;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(dense_smem(256))));
        attr = true;
    }
    const double bytes = double(M) * K * 8.0 + double(K) * b * 4.0 + double(M) * b * 4.0;
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    // one grid for every chunk (the finalize reads the same partial rows for
    // all columns): the first chunk's, which has the most tiles; a CTA
    // without a tile writes zero partials
    int grid_all = 0;
    // the split products' epilogue: one block per 32 rows, at most 2 per SM
    const int epi_grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>((M + 31) / 32, 2 * static_cast<int64_t>(L.sms))));
    for (int p_off = 0; p_off < b; p_off += 256)
    {
        const int nb = std::min(256, b - p_off);
        // one probe tile per chunk: narrower tiles (more CTAs for small M)
        // re-read the A tile from shared memory for less MMA work each and
        // measured slower (n = 8192: 414 vs 369 us)
        const int NB = static_cast<int>(round_up(nb, 16));
        const int ntn = 1;
        if (grid_all == 0)
            grid_all = static_cast<int>(
                std::max<int64_t>(1, std::min<int64_t>(ntm * ntn * ksplit, L.sms)));
        const int grid = grid_all;
        dim3 tg(static_cast<unsigned>((K + 31) / 32), static_cast<unsigned>((nb + 31) / 32));
        k_split_transpose<<<tg, dim3(32, 8), 0, L.st>>>(X, K, b, p_off, nb, op->ldx, op->xt_hi,
                                                        op->xt_lo);
        SLQ_LAUNCH_CK();
        ++L.launches;
        CUtensorMap xhi, xlo;
        SLQ_TRY(part_map(&xhi, op->xt_hi, op->ldx, nb, NB));
        SLQ_TRY(part_map(&xlo, op->xt_lo, op->ldx, nb, NB));
        DenseArgs d;
        d.M = M;
        d.K = K;
        d.nb = nb;
        d.NB = NB;
        d.ntn = ntn;
        d.b = b;
        d.p_off = p_off;
        // running total and chunk accumulator: two power-of-two halves
        uint32_t cols = 32;
        while (cols < static_cast<uint32_t>(NB)) cols <<= 1;
        d.tmem_cols = 2 * cols;
        d.X = X;
        d.sx = sx;
        d.shift = shift;
        d.Y = Y;
        d.Z = Z;
        d.zc = zc;
        d.zs = zs;
        d.epi = epi;
        d.partials = partials;
        d.error = error ? error : op->d_error;
        d.ksplit = ksplit;
        d.acc = op->d_acc;
        k_dense_tc<<<grid, DT_THREADS, dense_smem(NB), L.st>>>(ahi, alo, xhi, xlo, d);
        SLQ_LAUNCH_CK();
        ++L.launches;
        if (ksplit > 1)
        {
            k_dense_epi<<<epi_grid, 256, 0, L.st>>>(d);
            SLQ_LAUNCH_CK();
            ++L.launches;
        }
    }
    *grid_out = ksplit > 1 ? epi_grid : grid_all;
    return SLQ_OK;
}


template <int G, int NS>
slq_status spmm_rgt_inst(Launcher& L, const CUtensorMap* xmap, const int32_t* gptr,
                         const int32_t* gcol, const float* gval, int64_t nrows, int b,
                         const float* X, const double* sx, double shift, float* Y,
                         const float* Z, const double* zc, const double* zs, int epi,
                         double* partials, int32_t* error, int64_t nnz, int64_t xrows,
                         int* grid_out)
{
    const double bytes = nnz * 8.0 + (nrows + 1) * 4.0 + double(xrows) * b * 4.0 +
                         double(nrows) * b * 4.0 * (Z ? 2.0 : 1.0);
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    constexpr size_t smem = RgtShape<G>::SMEM;
    static bool attr = false;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_spmm_rgt<G, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
        attr = true;
    }
    const int64_t ng = (nrows + G - 1) / G;
    constexpr int GPC = RgtShape<G>::WARPS / NS;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>((ng + GPC - 1) / GPC, L.sms)));
    k_spmm_rgt<G, NS><<<grid, RgtShape<G>::WARPS * 32, smem, L.st>>>(
        *xmap, gptr, gcol, gval, nrows, ng, b, X, sx, shift, Y, Z, zc, zs, epi, partials, error);
    SLQ_LAUNCH_CK();
    ++L.launches;
    *grid_out = grid;
    return SLQ_OK;
}

// Operator product on a block: row-group SpMM where the operator has the
// format and the width suits it (32 <= b <= 256; FP64 b <= 128), else CSR.
// *grid_out receives the number of partial rows the launch writes.
template <typename VT, int LV, int G, int NS>
slq_status spmm_rg_inst(Launcher& L, const int32_t* gptr, const int32_t* gcol, const VT* gval,
                        int64_t nrows, int b, const VT* X, const double* sx, double shift, VT* Y,
                        const VT* Z, const double* zc, const double* zs, int epi,
                        double* partials, int64_t nnz, int64_t xrows, int* grid_out)
{
    const double s = sizeof(VT);
    const double bytes = nnz * (s + 4.0) + (nrows + 1) * 4.0 + double(xrows) * b * s +
                         double(nrows) * b * s * (Z ? 2.0 : 1.0);
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    const int64_t ng = (nrows + G - 1) / G;
    constexpr int GPC = 8 / NS;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>((ng + GPC - 1) / GPC, int64_t(L.sms) * 4)));
    k_spmm_rg<VT, LV, G, NS><<<grid, 256, 0, L.st>>>(gptr, gcol, gval, nrows, ng, b, X, sx, shift, Y,
                                                 Z, zc, zs, epi, partials);
    SLQ_LAUNCH_CK();
    ++L.launches;
    *grid_out = grid;
    return SLQ_OK;
}

// Tensor-core row-group SpMM (k_spmm_tc): 16-row groups, b = 128 NS, two
// CTAs per SM; X rows by TMA gathers (xmap as for k_spmm_rgt).
template <int NS>
slq_status spmm_tc_inst(Launcher& L, const CUtensorMap* xmap, const int32_t* gptr,
                        const int32_t* gcol, const float* gval, int64_t nrows, int b,
                        const float* X, const double* sx, double shift, float* Y, const float* Z,
                        const double* zc, const double* zs, int epi, double* partials,
                        int32_t* error, int64_t nnz, int64_t xrows, int* grid_out)
{
    const double bytes = nnz * 8.0 + (nrows + 1) * 4.0 + double(xrows) * b * 4.0 +
                         double(nrows) * b * 4.0 * (Z ? 2.0 : 1.0);
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    const int64_t ng = (nrows + 15) / 16;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>(ng * NS, int64_t(L.sms) * 2)));
    static bool attr = false;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_spmm_tc<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(TC_DYN_SMEM)));
        attr = true;
    }
    k_spmm_tc<NS><<<grid, TC_THREADS, TC_DYN_SMEM, L.st>>>(*xmap, gptr, gcol, gval, nrows, ng, b,
                                                          X, sx, shift, Y, Z, zc, zs, epi,
                                                          partials, error);
    SLQ_LAUNCH_CK();
    ++L.launches;
    *grid_out = grid;
    return SLQ_OK;
}

// Tensor-core block SpMM (k_spmm_blk): b = 128 or 256 probes, one CTA per
// SM over the operator's 128-row blocks.
slq_status spmm_blk_inst(Launcher& L, const slq_op* op, int transpose, int b, const float* X, const double* sx, double shift, float* Y,
                         const float* Z, const double* zc, const double* zs, int epi,
                         double* partials, int32_t* error, int64_t xrows, int* grid_out,
                         const XMaps* maps)
{
    // X split into FP16 parts first (one streaming pass) when the caller
    // gave a buffer for it and X has probe scales: the product then needs
    // no converter warps
    const bool pre = maps && maps->has_x16 && maps->x16 && maps->x16_b == b && sx;
    const int64_t rows = transpose ? op->ncols : op->nrows;
    const int64_t nblk = transpose ? op->t_nblk : op->a_nblk;
    // compulsory traffic as for the CSR kernels (the algorithm's bytes, not
    // the block format's)
    const double bytes = op->nnz * 8.0 + (rows + 1) * 4.0 + double(xrows) * b * 4.0 +
                         double(rows) * b * 4.0 * (Z ? 2.0 : 1.0);
    const bool ready = pre && maps->x16_ready && maps->x16exp;
    if (pre && !ready)
    {
        // its own profile class: one read of X and one write of its parts
        ProfScope split_prof(SLQ_K_SPLIT, double(xrows) * b * 8.0, L.st);
        k_x16_split<<<L.sms * 4, 256, 0, L.st>>>(X, sx, xrows, b, maps->x16);
        SLQ_LAUNCH_CK();
        ++L.launches;
    }
    ProfScope prof(SLQ_K_SPMM, bytes, L.st);
    const size_t smem = blk_smem_bytes(b);
    static bool attr = false;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_spmm_blk<128, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(blk_smem_bytes(128))));
        SLQ_CK(cudaFuncSetAttribute(k_spmm_blk<256, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(blk_smem_bytes(256))));
        SLQ_CK(cudaFuncSetAttribute(k_spmm_blk<128, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(blk_smem_bytes(128))));
        SLQ_CK(cudaFuncSetAttribute(k_spmm_blk<256, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(blk_smem_bytes(256))));
        attr = true;
    }

    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(nblk, L.sms)));
    // an X without probe scales: its per-probe maxima first (into the
    // partial-sum buffer past this launch's rows, or, for a product without
    // one, into the format's slot)
    unsigned int* xmax = nullptr;
    if (!sx)
    {
        xmax = partials ? reinterpret_cast<unsigned int*>(partials + int64_t(L.sms) * b)
                        : op->blk_xmax;
        if (!xmax) return fail(SLQ_ERR_BAD_ARG, "block SpMM: no room for the probe maxima");
        SLQ_CK(cudaMemsetAsync(xmax, 0, sizeof(unsigned int) * b, L.st));
        k_blk_colmax<<<dim3(static_cast<unsigned>(std::min<int64_t>((xrows + 7) / 8, L.sms * 4)),
                            static_cast<unsigned>(b / 32)),
                       256, 0, L.st>>>(X, xrows, b, xmax);
        SLQ_LAUNCH_CK();
        ++L.launches;
    }
    BlkArgs d;
    d.M = rows;
    d.nblk = nblk;
    d.NB = b;
    d.bstage = transpose ? op->t_bstage : op->a_bstage;
    d.order = transpose ? op->t_order : op->a_order;
    d.ucol = transpose ? op->t_ucol : op->a_ucol;
    d.rsc = transpose ? op->t_rsc : op->a_rsc;
    d.img = transpose ? op->t_img : op->a_img;
    d.X = X;
    d.sx = sx;
    d.xmax = xmax;
    d.shift = shift;
    d.Y = Y;
    d.Z = Z;
    d.zc = zc;
    d.zs = zs;
    d.epi = epi;
    d.partials = partials;
    d.error = error;
    d.x16 = pre ? maps->x16 : nullptr;
    d.xexp = ready ? maps->x16exp : nullptr;
    if (pre && b == 256)
        k_spmm_blk<256, true><<<grid, BLK_THREADS, smem, L.st>>>(d);
    else if (pre)
        k_spmm_blk<128, true><<<grid, BLK_THREADS, smem, L.st>>>(d);
    else if (b == 256)
        k_spmm_blk<256, false><<<grid, BLK_THREADS, smem, L.st>>>(d);
    else
        k_spmm_blk<128, false><<<grid, BLK_THREADS, smem, L.st>>>(d);
    SLQ_LAUNCH_CK();
    ++L.launches;
    *grid_out = grid;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// SpMM candidates: storage format x tile.  A row-group candidate is the tile
// of LV probes per lane and NS warps sharing one row group (b = 32 LV NS);
// the TMA candidate gathers X rows with tile::gather4 into shared memory.
// The built-in choice (op_spmm without a tuned entry) is the first of: TMA
// (FP32, G = 8, b = 128 or 256), row-group with the widest LV <= 4, CSR.
// ---------------------------------------------------------------------------

enum { CAND_CSR = 0, CAND_RG = 1, CAND_TMA = 2, CAND_TC = 3, CAND_BLK = 4 };

struct SpmmCand {
    int kind, g, lv, ns;
};

template <typename VT>
int spmm_candidates(const slq_op* op, int transpose, int b, SpmmCand* out)
{
    int n = 0;
    out[n++] = {CAND_CSR, 0, 0, 0};
    if (sizeof(VT) == 4 && (transpose ? op->t_bstage : op->a_bstage) && (b == 128 || b == 256))
        out[n++] = {CAND_BLK, BLK_ROWS, 0, b / 128};
    const int32_t* gptr = transpose ? op->t_gptr : op->a_gptr;
    const int G = op->group_rows;
    if (!G || !gptr) return n;
    // FP64 row groups: b <= 64, LV <= 2, G <= 8 (shared-memory staging);
    // 16-row groups keep LV <= 2 (16 x LV accumulators per lane)
    const int bmax = (sizeof(VT) == 8) ? 64 : 256;
    const int lvmax = (sizeof(VT) == 8 || G == 16) ? 2 : 4;
    if (b >= 32 && b <= bmax && (sizeof(VT) == 4 || G <= 8))
        for (int lv = 1; lv <= lvmax; lv *= 2)
        {
            const int ns = b / (32 * lv);
            if (ns >= 1 && ns <= 8 && 32 * lv * ns == b) out[n++] = {CAND_RG, G, lv, ns};
        }
    if (sizeof(VT) == 4 && (G == 8 || G == 16) && (b == 128 || b == 256))
        out[n++] = {CAND_TMA, G, 4, b / 128};
    if (sizeof(VT) == 4 && G == 16 && (b == 128 || b == 256))
        out[n++] = {CAND_TC, 16, 1, b / 128};
    return n;
}

template <typename VT>
slq_status spmm_cand(Launcher& L, const slq_op* op, int transpose, const SpmmCand& c, int b,
                     const VT* X, const double* sx, double shift, VT* Y, const VT* Z,
                     const double* zc, const double* zs, int epi, double* partials,
                     int* grid_out, const XMaps* maps, int32_t* error)
{
    const int64_t rows = transpose ? op->ncols : op->nrows;
    const int64_t xrows = transpose ? op->nrows : op->ncols;
    const int32_t* gptr = transpose ? op->t_gptr : op->a_gptr;
    const CUtensorMap* xmap = (maps && maps->has_row) ? &maps->row : nullptr;
    if (c.kind == CAND_BLK)
    {
        if constexpr (sizeof(VT) == 4)
        {
            if (!error) return fail(SLQ_ERR_BAD_ARG, "block SpMM needs an error word");
            return spmm_blk_inst(L, op, transpose, b, X, sx, shift, Y, Z, zc, zs, epi, partials,
                                 error, xrows, grid_out, maps);
        }
        return fail(SLQ_ERR_BAD_ARG, "block SpMM is FP32 only");
    }
    const int32_t* gcol = transpose ? op->t_gcol : op->a_gcol;
    if (c.kind == CAND_TMA)
    {
        if constexpr (sizeof(VT) == 4)
        {
            if (!xmap || !error) return fail(SLQ_ERR_BAD_ARG, "TMA SpMM needs a tensor map");
            const float* gval = static_cast<const float*>(transpose ? op->t_gval : op->a_gval);
#define SLQ_RGT_CASE(GG, NSS)                                                                  \
    if (c.g == GG && c.ns == NSS)                                                              \
        return spmm_rgt_inst<GG, NSS>(L, xmap, gptr, gcol, gval, rows, b, X, sx, shift, Y, Z, \
                                      zc, zs, epi, partials, error, op->nnz, xrows, grid_out);
            SLQ_RGT_CASE(8, 1)
            SLQ_RGT_CASE(8, 2)
            SLQ_RGT_CASE(16, 1)
            SLQ_RGT_CASE(16, 2)
#undef SLQ_RGT_CASE
            return fail(SLQ_ERR_BAD_ARG, "TMA SpMM: unsupported tile");
        }
        return fail(SLQ_ERR_BAD_ARG, "TMA SpMM is FP32 only");
    }
    if (c.kind == CAND_TC)
    {
        if constexpr (sizeof(VT) == 4)
        {
            if (!xmap || !error)
                return fail(SLQ_ERR_BAD_ARG, "tensor-core SpMM needs a tensor map and error word");
            const float* gval = static_cast<const float*>(transpose ? op->t_gval : op->a_gval);
            if (c.ns == 2)
                return spmm_tc_inst<2>(L, xmap, gptr, gcol, gval, rows, b, X, sx, shift, Y, Z, zc,
                                       zs, epi, partials, error, op->nnz, xrows, grid_out);
            return spmm_tc_inst<1>(L, xmap, gptr, gcol, gval, rows, b, X, sx, shift, Y, Z, zc, zs,
                                   epi, partials, error, op->nnz, xrows, grid_out);
        }
        return fail(SLQ_ERR_BAD_ARG, "tensor-core SpMM is FP32 only");
    }
    if (c.kind == CAND_RG)
    {
        const VT* gval = static_cast<const VT*>(transpose ? op->t_gval : op->a_gval);
#define SLQ_RG_CASE(GG, LVV, NSS)                                                            \
    if (c.g == GG && c.lv == LVV && c.ns == NSS)                                           \
        return spmm_rg_inst<VT, LVV, GG, NSS>(L, gptr, gcol, gval, rows, b, X, sx, shift, Y, \
                                              Z, zc, zs, epi, partials, op->nnz, xrows,     \
                                              grid_out);
#define SLQ_RG_ALL(GG)         \
    SLQ_RG_CASE(GG, 1, 1)      \
    SLQ_RG_CASE(GG, 1, 2)      \
    SLQ_RG_CASE(GG, 2, 1)      \
    if constexpr (sizeof(VT) == 4) \
    {                          \
        SLQ_RG_CASE(GG, 1, 4)  \
        SLQ_RG_CASE(GG, 2, 2)  \
        SLQ_RG_CASE(GG, 4, 1)  \
        SLQ_RG_CASE(GG, 1, 8)  \
        SLQ_RG_CASE(GG, 2, 4)  \
        SLQ_RG_CASE(GG, 4, 2)  \
    }
        SLQ_RG_ALL(8)
        SLQ_RG_ALL(4)
        if constexpr (sizeof(VT) == 4)
        {
            SLQ_RG_CASE(16, 1, 1)
            SLQ_RG_CASE(16, 1, 2)
            SLQ_RG_CASE(16, 2, 1)
            SLQ_RG_CASE(16, 1, 4)
            SLQ_RG_CASE(16, 2, 2)
            SLQ_RG_CASE(16, 1, 8)
            SLQ_RG_CASE(16, 2, 4)
        }
#undef SLQ_RG_ALL
#undef SLQ_RG_CASE
        return fail(SLQ_ERR_BAD_ARG, "row-group SpMM: unsupported tile");
    }
    const int32_t* ptr = transpose ? op->t_ptr : op->a_ptr;
    const int32_t* ind = transpose ? op->t_ind : op->a_ind;
    const VT* val = static_cast<const VT*>(transpose ? op->t_data : op->a_data);
    const int grid = spmm_grid<VT>(L, rows, b);
    *grid_out = grid;
    return spmm<VT>(L, grid, ptr, ind, val, rows, b, X, sx, shift, Y, Z, zc, zs, epi, partials,
                    op->nnz, xrows);
}

int log2_width(int b)
{
    int lg = 0;
    while ((1 << lg) < b) ++lg;
    return lg;
}

// Operator product on a block.  An autotuned choice (slq_operator_tune /
// slq_operator_set_variant) for this width and direction is used where one
// is set; the built-in choice otherwise (and for a tuned TMA candidate when
// the caller has no tensor map).  *grid_out receives the number of partial
// rows the launch writes.
template <typename VT>
slq_status op_spmm(Launcher& L, const slq_op* op, int transpose, int b, const VT* X,
                   const double* sx, double shift, VT* Y, const VT* Z, const double* zc,
                   const double* zs, int epi, double* partials, int* grid_out,
                   const XMaps* maps = nullptr, int32_t* error = nullptr)
{
    if (op->dense)
    {
        if constexpr (sizeof(VT) == 4)
            return dense_spmm(L, op, transpose, b, X, sx, shift, Y, Z, zc, zs, epi, partials,
                              grid_out, error);
        return fail(SLQ_ERR_BAD_ARG, "dense operators hold float32 data");
    }
    SpmmCand cands[SLQ_TUNE_MAX_CANDIDATES];
    const int nc = spmm_candidates<VT>(op, transpose, b, cands);
    const int lg = log2_width(b);
    const int ti = (lg <= 10) ? op->tuned[transpose ? 1 : 0][lg] : -1;
    const bool have_row = maps && maps->has_row && error;
    const bool have_blk = error != nullptr;
    auto usable = [&](const SpmmCand& c) {
        if (c.kind == CAND_TMA || c.kind == CAND_TC) return have_row;
        if (c.kind == CAND_BLK) return have_blk;
        return true;
    };
    if (ti >= 0 && ti < nc && usable(cands[ti]))
        return spmm_cand<VT>(L, op, transpose, cands[ti], b, X, sx, shift, Y, Z, zc, zs, epi,
                             partials, grid_out, maps, error);
    // built-in choice: the tensor-core block kernel, TMA, then the row-group
    // tile with the widest LV, then CSR
    int pick = 0;
    for (int i = 0; i < nc; ++i)
    {
        if (cands[i].kind == CAND_BLK && have_blk)
        {
            pick = i;
            break;
        }
    }
    for (int i = 0; i < nc && cands[pick].kind != CAND_BLK; ++i)
    {
        if (cands[i].kind == CAND_TC || cands[i].kind == CAND_BLK) continue;  // tuner / above
        if (cands[i].kind == CAND_TMA && !have_row) continue;
        if (cands[i].kind == CAND_TMA)
        {
            pick = i;
            break;
        }
        if (cands[i].kind == CAND_RG && (cands[pick].kind != CAND_RG || cands[i].lv > cands[pick].lv))
            pick = i;
    }
    return spmm_cand<VT>(L, op, transpose, cands[pick], b, X, sx, shift, Y, Z, zc, zs, epi,
                         partials, grid_out, maps, error);
}

// TMA-streamed pass (k_stream): MODE 0 = update + inner products,
// MODE 1 = (update +) reorthogonalisation update + norm.
template <typename VT, int MODE>
slq_status stream_pass(Launcher& L, int64_t n, int b, const VT* W, VT* Wout, int do_update,
                       const VT* Vj, const double* sj, const double* aj, const VT* Vm,
                       const double* sm, const double* bm, const VT* basis, int64_t slot_elems,
                       int bs, int last, int J, const VT* coef, int want_norm,
                       double* partials, int32_t* error, int* grid_out,
                       double* wn2_out = nullptr, const double* wn2_in = nullptr,
                       int wn2_grid = 0, __half* x16 = nullptr, int32_t* x16exp = nullptr)
{
    constexpr int R = (sizeof(VT) == 4) ? 16 : 8;
    constexpr size_t SMEM_MAX = 232448;
    const int PT = std::min(b, STREAM_CONSUMERS);
    const int T = R * (STREAM_CONSUMERS / PT);
    const size_t fixed = 256 + STREAM_CONSUMERS * sizeof(double);
    const size_t extra = (MODE == 0) ? static_cast<size_t>(J) * STREAM_CONSUMERS * 8
                                     : static_cast<size_t>(J) * PT * 8;
    if (fixed + extra + 2 * STREAM_TILE_BYTES > SMEM_MAX)
        return fail(SLQ_ERR_BAD_ARG, "stream pass: too many basis vectors per launch");
    const int S = static_cast<int>(std::min<size_t>(STREAM_MAX_STAGES,
                                                    (SMEM_MAX - fixed - extra) / STREAM_TILE_BYTES));
    const size_t smem = fixed + static_cast<size_t>(S) * STREAM_TILE_BYTES + extra;
    static bool attr = false;
    if (!attr)
    {
        SLQ_CK(cudaFuncSetAttribute(k_stream<VT, MODE, R>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(SMEM_MAX)));
        attr = true;
    }
    StreamArgs<VT> a;
    a.n = n;
    a.b = b;
    a.PT = PT;
    a.T = T;
    a.S = S;
    a.J = J;
    a.bs = bs;
    a.last = last;
    a.slot_elems = slot_elems;
    a.W = W;
    a.Wout = Wout;
    a.do_update = do_update;
    a.Vj = Vj;
    a.sj = sj;
    a.aj = aj;
    a.Vm = Vm;
    a.sm = sm;
    a.bm = bm;
    a.basis = basis;
    a.coef = coef;
    a.want_norm = want_norm;
    a.partials = partials;
    a.error = error;
    a.fail_first_wait = 0;
    a.wn2_out = wn2_out;
    a.wn2_in = wn2_in;
    a.wn2_grid = wn2_grid;
    a.x16 = x16;
    a.x16exp = x16exp;
    if (g_fail_stream_waits.load() > 0 && g_fail_stream_waits.fetch_sub(1) > 0)
        a.fail_first_wait = 1;
    const int gy = b / PT;
    const int gx = std::max(1, L.sms / gy);
    const double vb = double(n) * b * sizeof(VT);
    const int npre = 1 + (do_update ? (Vm ? 2 : 1) : 0);
    const int skip = (MODE == 0 && do_update) ? (Vm ? 2 : 1) : 0;
    const int reads = npre + std::max(0, J - skip);
    // the split parts: 2 x 2 bytes per element, one float vector's bytes
    const int writes = ((MODE == 1 || do_update) ? 1 : 0) + (x16 ? 1 : 0);
    ProfScope prof(MODE == 0 ? SLQ_K_DOTS : SLQ_K_REORTH, vb * (reads + writes), L.st);
    k_stream<VT, MODE, R><<<dim3(gx, gy), STREAM_THREADS, smem, L.st>>>(a);
    SLQ_LAUNCH_CK();
    ++L.launches;
    *grid_out = gx;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// run plan and workspace
// ---------------------------------------------------------------------------

struct RunPlan {
    int gram, orth, m, bs, b, q;
    bool x16;             // a buffer for the probe block split into FP16 parts
    int64_t nv, nu;       // probe length, U length (gram)
    int64_t wpp;          // parity words per probe
    int cw, nchunks;      // parity chunking
    size_t partial_cols;  // max partial buffer doubles
};

struct RunBufs {
    void* V;
    void* U;
    void* W;
    void* W2;
    void* T;              // normal-equations runs: A v, [nu][b]
    __half* X16;          // the SpMM's probe block split into FP16 parts, [nv][2 b]
    int32_t* X16exp;      // its per-probe exponents when a streaming pass wrote it
    double* wn2;          // |w|^2 partials of the dots pass for that split, [sms][b]
    double* negshift;     // normal-equations runs: -t per probe
    double* scale_v;
    double* scale_u;
    double* alpha;
    double* beta;
    void* coef;
    int32_t* active;
    int32_t* size;
    int32_t* status;
    int32_t* error;
    double* partials;
    double* samples;
    double* params;
    uint64_t* starts;
    uint64_t* chunk_polys;
};

int buffer_size(int gram, int orth, int m)
{
    if (gram)
    {
        if (orth == 0) return 2;
        if (orth < 0 || orth > m - 1) return m;
        return orth + 1;
    }
    if (orth == 0 || orth == 1) return 2;
    if (orth < 0 || orth > m) return m;
    return orth;
}

slq_status make_plan(const slq_op* op, const slq_params* p, int q, RunPlan* r)
{
    if (!op || !p) return fail(SLQ_ERR_BAD_ARG, "NULL operator or params");
    if (p->lanczos_degree < 1 || p->lanczos_degree > SLQ_MAX_DEGREE)
        return fail(SLQ_ERR_BAD_ARG, "lanczos_degree must be in [1, " +
                                         std::to_string(SLQ_MAX_DEGREE) + "]");
    if (p->min_num_samples < 1 || p->max_num_samples < 1 ||
        p->min_num_samples > p->max_num_samples)
        return fail(SLQ_ERR_BAD_ARG, "need 1 <= min_num_samples <= max_num_samples");
    if (p->func < SLQ_FUNC_LOG || p->func > SLQ_FUNC_SMOOTHSTEP)
        return fail(SLQ_ERR_BAD_ARG, "unknown matrix function");
    if (p->seed < 0) return fail(SLQ_ERR_BAD_ARG, "seed must be >= 0");
    if (p->first_probe < 0) return fail(SLQ_ERR_BAD_ARG, "first_probe must be >= 0");
    if (q < 1) return fail(SLQ_ERR_BAD_ARG, "num_inquiries must be >= 1");
    if (q > 1 && !op->affine)
        return fail(SLQ_ERR_BAD_ARG, "several inquiries need an affine operator");
    if (p->gram < 0 || p->gram > 2)
        return fail(SLQ_ERR_BAD_ARG, "gram must be 0, 1 or 2");
    if (q > 1 && p->gram == 1)
        return fail(SLQ_ERR_UNSUPPORTED,
                    "eigenvalue shift across inquiries is not valid for Golub-Kahn runs");
    if (p->gram != 2 && op->nrows != op->ncols && (p->gram == 0 || op->affine))
        return fail(SLQ_ERR_BAD_ARG, "this run needs a square matrix");
    if (p->gram && !(op->dense ? op->dt_hi != nullptr : op->t_ptr != nullptr))
        return fail(SLQ_ERR_BAD_ARG, "gram runs need an operator created with need_transpose");
    if (p->orthogonalize > p->lanczos_degree)
        return fail(SLQ_ERR_BAD_ARG, "orthogonalize must be at most lanczos_degree");
    if (p->rng != SLQ_RNG_PARITY && p->rng != SLQ_RNG_FAST)
        return fail(SLQ_ERR_BAD_ARG, "unknown rng mode");
    r->gram = p->gram;
    r->orth = p->orthogonalize;
    r->m = p->lanczos_degree;
    r->bs = buffer_size(r->gram == 1, r->orth, r->m);
    r->q = q;
    r->nv = r->gram ? op->ncols : op->nrows;
    r->nu = r->gram ? op->nrows : 0;
    const int bmax = (op->dtype == SLQ_F64) ? 512 : 1024;
    int b = p->block_size;
    if (b <= 0) b = std::min(next_pow2(p->max_num_samples), 256);
    b = std::min(next_pow2(b), bmax);
    b = std::min(b, next_pow2(p->max_num_samples));
    r->b = b;
    // the block SpMM of A v (a float32 block format, b = 128 or 256) takes
    // v split into FP16 parts beforehand
    r->x16 = op->dtype == SLQ_F32 && !op->dense && op->a_nblk > 0 && r->gram != 1 &&
             (b == 128 || b == 256);
    r->wpp = r->nv / 64 + 1;
    r->cw = 64;
    while ((r->wpp + r->cw - 1) / r->cw > 65535) r->cw *= 2;
    r->nchunks = static_cast<int>((r->wpp + r->cw - 1) / r->cw);
    return SLQ_OK;
}

// Elements between consecutive basis slots: the block plus 2560 bytes, so
// that slot strides are not a multiple of a large power of two (the same
// row of every slot would otherwise fall into the same DRAM channels).
template <typename VT>
int64_t slot_stride(int64_t len, int b)
{
    return ((len * b + 63) / 64) * 64 + 2560 / static_cast<int64_t>(sizeof(VT));
}

template <typename VT>
void carve(Carver& c, const RunPlan& r, int sms, RunBufs* B)
{
    const int64_t vslot = slot_stride<VT>(r.nv, r.b);
    const int64_t uslot = slot_stride<VT>(r.nu, r.b);
    B->V = c.take<VT>(static_cast<size_t>(r.bs) * vslot);
    B->U = (r.gram == 1) ? c.take<VT>(static_cast<size_t>(r.bs) * uslot) : nullptr;
    B->W = (r.gram == 1) ? nullptr : c.take<VT>(vslot);
    B->W2 = (r.gram != 1 && r.orth != 0) ? c.take<VT>(vslot) : nullptr;
    B->T = (r.gram == 2) ? c.take<VT>(static_cast<size_t>(r.nu) * r.b) : nullptr;
    B->X16 = r.x16 ? c.take<__half>(static_cast<size_t>(r.nv) * 2 * r.b) : nullptr;
    B->X16exp = r.x16 ? c.take<int32_t>(r.b) : nullptr;
    B->wn2 = r.x16 ? c.take<double>(static_cast<size_t>(sms) * r.b) : nullptr;
    B->negshift = c.take<double>(r.b);
    B->scale_v = c.take<double>(static_cast<size_t>(r.bs) * r.b);
    B->scale_u = c.take<double>(static_cast<size_t>(r.bs) * r.b);
    B->alpha = c.take<double>(static_cast<size_t>(r.m) * r.b);
    B->beta = c.take<double>(static_cast<size_t>(r.m) * r.b);
    B->coef = c.take<VT>(static_cast<size_t>(r.bs) * r.b);
    B->active = c.take<int32_t>(r.b);
    B->size = c.take<int32_t>(r.b);
    B->status = c.take<int32_t>(r.b);
    B->error = c.take<int32_t>(1);
    // partial sums: SpMM grid <= 4*sms, stream kernels <= 2*sms (x J <= MAX_J)
    const size_t pcols = std::max<size_t>(static_cast<size_t>(sms) * 4 * r.b,
                                          static_cast<size_t>(sms) * 2 * MAX_J * r.b);
    B->partials = c.take<double>(pcols);
    B->samples = c.take<double>(static_cast<size_t>(r.b) * r.q);
    B->params = c.take<double>(r.q);
    B->starts = c.take<uint64_t>(static_cast<size_t>(r.b) * 4);
    B->chunk_polys = c.take<uint64_t>(static_cast<size_t>(r.nchunks) * 4);
}

double4 func_coeff(const slq_params* p)
{
    return make_double4(p->func_coeff[0], p->func_coeff[1], p->func_coeff[2], p->func_coeff[3]);
}

template <typename VT>
slq_status launch_probes(Launcher& L, const RunPlan& r, int rng, int64_t seed, int64_t first,
                         int count, const RunBufs& B, const int32_t* inv, VT* X)
{
    dim3 grid((r.b + 127) / 128, r.nchunks);
    ProfScope prof(SLQ_K_PROBE, double(r.nv) * r.b * sizeof(VT), L.st);
    if (rng == SLQ_RNG_PARITY)
        k_probe_parity<VT><<<grid, 128, 0, L.st>>>(r.nv, r.b, count, r.wpp, r.cw, B.starts,
                                                   B.chunk_polys, inv, X);
    else
        k_probe_fast<VT><<<grid, 128, 0, L.st>>>(r.nv, r.b, count, first,
                                                 static_cast<uint64_t>(seed) * 0xd1342543de82ef95ULL,
                                                 r.wpp, r.cw, inv, X);
    SLQ_LAUNCH_CK();
    ++L.launches;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// one probe block: Lanczos (symmetric) or Golub-Kahn (gram)
// ---------------------------------------------------------------------------

template <typename VT>
slq_status krylov_block(Launcher& L, const slq_op* op, const slq_params* p, const RunPlan& r,
                        const RunBufs& B, int count, double shift)
{
    const int b = r.b;
    const int bs = r.bs;
    const int m = r.m;
    const int64_t vslot = slot_stride<VT>(r.nv, b);
    const int64_t uslot = slot_stride<VT>(r.nu, b);
    VT* V = static_cast<VT*>(B.V);
    VT* U = static_cast<VT*>(B.U);
    VT* W = static_cast<VT*>(B.W);
    VT* W2 = static_cast<VT*>(B.W2);
    VT* coef = static_cast<VT*>(B.coef);
    const double thr = p->lanczos_tol * std::sqrt(static_cast<double>(r.nv));
    auto sv_of = [&](int vec) { return B.scale_v + static_cast<int64_t>(((vec % bs) + bs) % bs) * b; };
    auto su_of = [&](int vec) { return B.scale_u + static_cast<int64_t>(((vec % bs) + bs) % bs) * b; };
    auto Vs = [&](int vec) { return V + static_cast<int64_t>(((vec % bs) + bs) % bs) * vslot; };
    auto Us = [&](int vec) { return U + static_cast<int64_t>(((vec % bs) + bs) % bs) * uslot; };

    // TMA-fed SpMM kernels: tensor maps per basis slot (V slots feed A
    // products, U slots and the normal-equations buffer T feed A^T products)
    std::vector<XMaps> vmaps, umaps;
    bool use_tma = false;
    if constexpr (sizeof(VT) == 4)
    {
        const bool wide = (b == 128 || b == 256);
        const bool row_a = wide && (op->group_rows == 8 || op->group_rows == 16);
        // the block SpMM's split probe block: one buffer, rewritten before
        // every product of A v
        const bool want_x16 = B.X16 != nullptr;
        if (row_a || want_x16)
        {
            use_tma = true;
            vmaps.resize(bs);
            for (int sl = 0; sl < bs; ++sl)
            {
                SLQ_TRY(make_xmaps(&vmaps[sl], V + static_cast<int64_t>(sl) * vslot, r.nv, b,
                                   row_a));
                if (want_x16)
                {
                    vmaps[sl].x16 = B.X16;
                    vmaps[sl].x16_b = b;
                    vmaps[sl].has_x16 = true;
                }
            }
            if (r.gram == 1 && row_a)
            {
                umaps.resize(bs);
                for (int sl = 0; sl < bs; ++sl)
                    SLQ_TRY(make_xmaps(&umaps[sl], U + static_cast<int64_t>(sl) * uslot, r.nu,
                                       b, true));
            }
        }
    }
    auto vmap_of = [&](int vec) -> const XMaps* {
        return use_tma ? &vmaps[((vec % bs) + bs) % bs] : nullptr;
    };
    auto umap_of = [&](int vec) -> const XMaps* {
        return (use_tma && r.gram == 1) ? &umaps[((vec % bs) + bs) % bs] : nullptr;
    };

    // dots + finalize(COEF) + reorth over chunks of MAX_J basis vectors;
    // returns the number of partial rows of the norm partials in *nparts.
    auto reorthogonalize = [&](int64_t n, VT* w_in_first, VT* w_work, VT* w_out, int do_update,
                               const VT* Vj, const double* sj, const double* aj, const VT* Vm,
                               const double* sm, const double* bm, const VT* basis,
                               int64_t slot_elems, const double* scales, int last, int J,
                               int* nparts, bool split) -> slq_status {
        // split: the last pass also writes w_out split into FP16 parts for
        // the block SpMM (B.X16), scaled by the norm the first dots pass
        // measures of the updated w
        split = split && B.X16 && do_update;
        int dg0 = 0;
        for (int c0 = 0; c0 < J; c0 += MAX_J)
        {
            const int Jc = std::min(MAX_J, J - c0);
            const bool first = (c0 == 0);
            int dg = 0;
            SLQ_TRY(stream_pass<VT, 0>(L, n, b, first ? w_in_first : w_work, w_work,
                                       first ? do_update : 0, Vj, sj, aj, Vm, sm, bm, basis,
                                       slot_elems, bs, last - c0, Jc, nullptr, 0, B.partials,
                                       B.error, &dg, (split && first) ? B.wn2 : nullptr));
            if (first) dg0 = dg;
            SLQ_TRY(finalize<VT>(L, B.partials, dg, Jc * b, FIN_COEF, nullptr,
                                 coef + static_cast<int64_t>(c0) * b, scales, b, bs, last - c0,
                                 nullptr, nullptr, nullptr, 0, 0.0, 0));
        }
        int rg = 0;
        for (int c0 = 0; c0 < J; c0 += MAX_J)
        {
            const int Jc = std::min(MAX_J, J - c0);
            const bool lastc = (c0 + MAX_J >= J);
            const bool sp = split && lastc;
            SLQ_TRY(stream_pass<VT, 1>(L, n, b, w_work, lastc ? w_out : w_work, 0, nullptr,
                                       nullptr, nullptr, nullptr, nullptr, nullptr, basis,
                                       slot_elems, bs, last - c0, Jc,
                                       coef + static_cast<int64_t>(c0) * b, lastc ? 1 : 0,
                                       B.partials, B.error, &rg, nullptr,
                                       sp ? B.wn2 : nullptr, sp ? dg0 : 0,
                                       sp ? B.X16 : nullptr, sp ? B.X16exp : nullptr));
        }
        *nparts = rg;
        return SLQ_OK;
    };

    if (r.gram != 1)
    {
        VT* T = static_cast<VT*>(B.T);
        // B.X16 holds v_j split into FP16 parts when the previous step's last
        // reorthogonalisation pass wrote it (else the product splits v_j)
        bool x16_ready = false;
        for (int j = 0; j < m; ++j)
        {
            VT* vj = Vs(j);
            int sg = 0;
            if (use_tma && B.X16)
            {
                XMaps& mv = vmaps[((j % bs) + bs) % bs];
                mv.x16_ready = x16_ready;
                mv.x16exp = B.X16exp;
            }
            if (r.gram == 0)
            {
                SLQ_TRY(op_spmm<VT>(L, op, 0, b, vj, sv_of(j), shift, W, nullptr, nullptr,
                                    nullptr, 1, B.partials, &sg, vmap_of(j), B.error));
            }
            else
            {
                // normal equations: T = s_j A v_j, W = A^T T + t s_j v_j,
                // alpha partials against s_j v_j
                int sg1 = 0;
                SLQ_TRY(op_spmm<VT>(L, op, 0, b, vj, sv_of(j), 0.0, T, nullptr, nullptr,
                                    nullptr, 0, B.partials, &sg1, vmap_of(j), B.error));
                SLQ_TRY(op_spmm<VT>(L, op, 1, b, T, nullptr, 0.0, W, vj, B.negshift, sv_of(j),
                                    3, B.partials, &sg, nullptr, B.error));
            }
            x16_ready = false;
            double* aj = B.alpha + static_cast<int64_t>(j) * b;
            SLQ_TRY(finalize<VT>(L, B.partials, sg, b, FIN_STORE, aj, nullptr, nullptr, b, bs, 0,
                                 nullptr, nullptr, nullptr, 0, 0.0, j));
            const VT* vm = (j > 0) ? Vs(j - 1) : nullptr;
            const double* sm = (j > 0) ? sv_of(j - 1) : nullptr;
            const double* bm = (j > 0) ? B.beta + static_cast<int64_t>(j - 1) * b : nullptr;
            int J = 0;
            if (r.orth != 0)
                J = static_cast<int>(std::min<int64_t>((j < bs) ? j + 1 : bs, r.nv));
            int nparts = 0;
            if (J == 0)
            {
                SLQ_TRY(stream_pass<VT, 1>(L, r.nv, b, W, Vs(j + 1), 1, vj, sv_of(j), aj, vm, sm,
                                           bm, V, vslot, bs, j, 0, coef, 1, B.partials, B.error,
                                           &nparts));
            }
            else
            {
                SLQ_TRY(reorthogonalize(r.nv, W, W2, Vs(j + 1), 1, vj, sv_of(j), aj, vm, sm, bm,
                                        V, vslot, B.scale_v, j, J, &nparts, true));
                x16_ready = B.X16 != nullptr;
            }
            SLQ_TRY(finalize<VT>(L, B.partials, nparts, b, FIN_NORM,
                                 B.beta + static_cast<int64_t>(j) * b, nullptr, nullptr, b, bs, 0,
                                 sv_of(j + 1), B.active, B.size, 1, thr, j));
        }
    }
    else
    {
        for (int j = 0; j < m; ++j)
        {
            int no = 0;
            if (r.orth != 0) no = (j < bs) ? j : bs - 1;
            // u_j = A v_j - beta_{j-1} u_{j-1}
            const int Ju = (j > 0) ? static_cast<int>(std::min<int64_t>(no, r.nu)) : 0;
            VT* uj = Us(j);
            int sgu = 0;
            SLQ_TRY(op_spmm<VT>(L, op, 0, b, Vs(j), sv_of(j), shift, uj,
                                (j > 0) ? Us(j - 1) : nullptr,
                                (j > 0) ? B.beta + static_cast<int64_t>(j - 1) * b : nullptr,
                                (j > 0) ? su_of(j - 1) : nullptr, Ju > 0 ? 0 : 2, B.partials,
                                &sgu, vmap_of(j), B.error));
            int nparts = sgu;
            if (Ju > 0)
                SLQ_TRY(reorthogonalize(r.nu, uj, uj, uj, 0, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, U, uslot, B.scale_u, j - 1, Ju,
                                        &nparts, false));
            double* aj = B.alpha + static_cast<int64_t>(j) * b;
            SLQ_TRY(finalize<VT>(L, B.partials, nparts, b, FIN_NORM, aj, nullptr, nullptr, b, bs,
                                 0, su_of(j), B.active, B.size, 0, 0.0, j));
            // v_{j+1} = A^T u_j - alpha_j v_j
            const int Jv = static_cast<int>(std::min<int64_t>(no, r.nv));
            VT* vn = Vs(j + 1);
            int sgv = 0;
            SLQ_TRY(op_spmm<VT>(L, op, 1, b, uj, su_of(j), shift, vn, Vs(j), aj, sv_of(j),
                                Jv > 0 ? 0 : 2, B.partials, &sgv, umap_of(j), B.error));
            nparts = sgv;
            if (Jv > 0)
                SLQ_TRY(reorthogonalize(r.nv, vn, vn, vn, 0, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, V, vslot, B.scale_v, j, Jv, &nparts,
                                        false));
            SLQ_TRY(finalize<VT>(L, B.partials, nparts, b, FIN_NORM,
                                 B.beta + static_cast<int64_t>(j) * b, nullptr, nullptr, b, bs, 0,
                                 sv_of(j + 1), B.active, B.size, 1, thr, j));
        }
    }
    return SLQ_OK;
}

// Parity stream set-up of a run: start state of its probe 0, the advance
// polynomial between consecutive probes and the per-chunk polynomials.
slq_status parity_setup(const slq_params* p, const RunPlan& r, uint64_t* cur, Poly256* advance,
                        std::vector<uint64_t>* polys)
{
    if (!self_check()) return fail(SLQ_ERR_CUDA, "xoshiro256 jump polynomial self-check failed");
    stream_state(p->seed, cur);
    jump_ahead(cur, static_cast<uint64_t>(p->first_probe) * static_cast<uint64_t>(r.wpp));
    *advance = jump_poly(static_cast<uint64_t>(r.wpp));
    polys->assign(static_cast<size_t>(r.nchunks) * 4, 0);
    const Poly256 step = jump_poly(static_cast<uint64_t>(r.cw));
    Poly256 acc = {{1, 0, 0, 0}};
    for (int cidx = 0; cidx < r.nchunks; ++cidx)
    {
        for (int k = 0; k < 4; ++k) (*polys)[static_cast<size_t>(cidx) * 4 + k] = acc.w[k];
        acc = poly_mulmod(acc, step);
    }
    return SLQ_OK;
}

template <typename VT>
slq_status run_typed(slq_op* op, const slq_params* p, const double* parameters, int q,
                     void* workspace, size_t workspace_bytes, cudaStream_t st, slq_result* res)
{
    RunPlan r;
    SLQ_TRY(make_plan(op, p, q, &r));
    Launcher L;
    L.st = st;
    SLQ_TRY(device_sms(&L.sms));
    Carver c(workspace, workspace_bytes);
    RunBufs B;
    carve<VT>(c, r, L.sms, &B);
    if (!c.fits() || !workspace)
        return fail(SLQ_ERR_WORKSPACE, "run: workspace too small (need " + std::to_string(c.off) +
                                           " bytes)");

    const int max_s = p->max_num_samples;
    const int m = r.m;
    const int b = r.b;
    std::vector<double> params(q, 0.0);
    if (op->affine && parameters)
        for (int j = 0; j < q; ++j) params[j] = parameters[j];
    const double shift = op->affine ? params[0] : 0.0;
    SLQ_CK(cudaMemcpyAsync(B.params, params.data(), sizeof(double) * q, cudaMemcpyHostToDevice, st));
    SLQ_CK(cudaMemsetAsync(B.error, 0, sizeof(int32_t), st));
    k_fill_f64<<<(b + 255) / 256, 256, 0, st>>>(B.negshift, b, -shift);
    SLQ_LAUNCH_CK();
    int32_t herr = 0;

    // parity stream set-up on the host: state of probe 0 and the per-chunk
    // advance polynomials
    uint64_t cur[4] = {0, 0, 0, 0};
    Poly256 advance = {{1, 0, 0, 0}};
    std::vector<uint64_t> polys;
    if (p->rng == SLQ_RNG_PARITY)
    {
        SLQ_TRY(parity_setup(p, r, cur, &advance, &polys));
        SLQ_CK(cudaMemcpyAsync(B.chunk_polys, polys.data(), polys.size() * sizeof(uint64_t),
                               cudaMemcpyHostToDevice, st));
    }

    // outputs
    for (int64_t i = 0; i < static_cast<int64_t>(max_s) * q; ++i) res->samples[i] = NAN;
    for (int i = 0; i < max_s; ++i)
    {
        res->processed_samples_indices[i] = 0;
        if (res->lanczos_size) res->lanczos_size[i] = 0;
        if (res->probe_status) res->probe_status[i] = -1;
    }
    for (int j = 0; j < q; ++j)
    {
        res->converged[j] = 0;
        res->num_samples_used[j] = 0;
        res->num_outliers[j] = 0;
        res->trace[j] = NAN;
        res->error[j] = NAN;
    }
    if (res->alpha)
        for (int64_t i = 0; i < static_cast<int64_t>(max_s) * m; ++i) res->alpha[i] = NAN;
    if (res->beta)
        for (int64_t i = 0; i < static_cast<int64_t>(max_s) * m; ++i) res->beta[i] = NAN;

    cudaEvent_t ev0, ev1;
    SLQ_CK(cudaEventCreate(&ev0));
    SLQ_CK(cudaEventCreate(&ev1));
    SLQ_CK(cudaEventRecord(ev0, st));

    std::vector<double> hs(static_cast<size_t>(b) * q);
    std::vector<int32_t> hsize(b), hstat(b);
    std::vector<double> ha, hb;
    if (res->alpha || res->beta)
    {
        ha.resize(static_cast<size_t>(m) * b);
        hb.resize(static_cast<size_t>(m) * b);
    }
    std::vector<uint64_t> hstarts(static_cast<size_t>(b) * 4);
    const double s0 = 1.0 / std::sqrt(static_cast<double>(r.nv));
    int nproc = 0;
    int all = 0;
    int blocks = 0;
    int64_t computed = 0;
    slq_status status = SLQ_OK;
    bool eig_failed = false;
    for (int g = 0; g < max_s && !all; g += b)
    {
        const int count = std::min(b, max_s - g);
        if (p->rng == SLQ_RNG_PARITY)
        {
            for (int pi = 0; pi < count; ++pi)
            {
                for (int k = 0; k < 4; ++k) hstarts[static_cast<size_t>(pi) * 4 + k] = cur[k];
                apply_poly(advance, cur);
            }
            SLQ_CK(cudaMemcpyAsync(B.starts, hstarts.data(),
                                   sizeof(uint64_t) * 4 * static_cast<size_t>(count),
                                   cudaMemcpyHostToDevice, st));
        }
        SLQ_TRY(launch_probes<VT>(L, r, p->rng, p->seed, p->first_probe + g, count, B,
                                  op->inv, static_cast<VT*>(B.V)));
        {
        ProfScope prof(SLQ_K_OTHER, 0.0, st);
        k_init_block<<<(b + 127) / 128, 128, 0, st>>>(count, b, m, s0, B.scale_v, B.active,
                                                     B.size);
        SLQ_LAUNCH_CK();
        ++L.launches;
        }
        SLQ_TRY(krylov_block<VT>(L, op, p, r, B, count, shift));
        {
        ProfScope prof(SLQ_K_EIG, double(m) * b * 16.0 + double(count) * q * 8.0, st);
        k_eig_quad<<<(count + 127) / 128, 128, 0, st>>>(
            count, b, m, B.alpha, B.beta, B.size, r.gram == 1, p->func, func_coeff(p),
            p->exponent, B.params, q, static_cast<double>(r.nv), B.samples, nullptr, nullptr,
            B.status);
        SLQ_LAUNCH_CK();
        ++L.launches;
        }
        SLQ_CK(cudaMemcpyAsync(hs.data(), B.samples, sizeof(double) * count * q,
                               cudaMemcpyDeviceToHost, st));
        SLQ_CK(cudaMemcpyAsync(hsize.data(), B.size, sizeof(int32_t) * count,
                               cudaMemcpyDeviceToHost, st));
        SLQ_CK(cudaMemcpyAsync(hstat.data(), B.status, sizeof(int32_t) * count,
                               cudaMemcpyDeviceToHost, st));
        if (!ha.empty())
        {
            SLQ_CK(cudaMemcpyAsync(ha.data(), B.alpha, sizeof(double) * m * b,
                                   cudaMemcpyDeviceToHost, st));
            SLQ_CK(cudaMemcpyAsync(hb.data(), B.beta, sizeof(double) * m * b,
                                   cudaMemcpyDeviceToHost, st));
        }
        SLQ_CK(cudaMemcpyAsync(&herr, B.error, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SLQ_CK(cudaStreamSynchronize(st));
        if (herr)
            return fail(SLQ_ERR_TIMEOUT, "a streaming kernel gave up waiting for its copies");
        if (res->probe_status)
            for (int pi = 0; pi < count; ++pi) res->probe_status[g + pi] = hstat[pi];
        ++blocks;
        computed += count;
        for (int pi = 0; pi < count && !all; ++pi)
        {
            const int s = g + pi;
            for (int j = 0; j < q; ++j)
                res->samples[static_cast<int64_t>(s) * q + j] = hs[static_cast<size_t>(pi) * q + j];
            if (res->lanczos_size) res->lanczos_size[s] = hsize[pi];
            if (hstat[pi] & 2) eig_failed = true;
            if (!ha.empty())
                for (int i = 0; i < m; ++i)
                {
                    if (res->alpha)
                        res->alpha[static_cast<int64_t>(s) * m + i] =
                            (i < hsize[pi]) ? ha[static_cast<size_t>(i) * b + pi] : NAN;
                    if (res->beta)
                        res->beta[static_cast<int64_t>(s) * m + i] =
                            (i < hsize[pi]) ? hb[static_cast<size_t>(i) * b + pi] : NAN;
                }
            // with a known eigenvalue relation every inquiry is refreshed by
            // each sample (c_trace_estimator.cpp:572-583)
            if (op->affine && q > 1)
                for (int j = 0; j < q; ++j) res->converged[j] = 0;
            res->processed_samples_indices[nproc++] = s;
            all = slq_check_convergence(res->samples, q, p->min_num_samples,
                                        res->processed_samples_indices, nproc,
                                        p->confidence_level, p->error_atol, p->error_rtol,
                                        res->error, res->num_samples_used, res->converged);
        }
    }
    SLQ_CK(cudaEventRecord(ev1, st));
    SLQ_CK(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    SLQ_CK(cudaEventElapsedTime(&ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);

    slq_average_estimates(p->confidence_level, p->outlier_significance_level, q, max_s,
                          res->num_samples_used, res->processed_samples_indices, res->samples,
                          res->num_outliers, res->trace, res->error);
    res->all_converged = all;
    res->num_blocks = blocks;
    res->num_probes_computed = computed;
    res->gpu_launches = L.launches;
    res->alg_wall_time = ms * 1e-3f;
    if (eig_failed) status = fail(SLQ_ERR_EIGEN, "tridiagonal eigen-solve did not converge");
    return status;
}

}  // namespace

extern "C" slq_status slq_run_workspace_bytes(const slq_op* op, const slq_params* p,
                                              int num_inquiries, size_t* bytes)
{
    if (!bytes) return fail(SLQ_ERR_BAD_ARG, "bytes is NULL");
    RunPlan r;
    SLQ_TRY(make_plan(op, p, num_inquiries, &r));
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(nullptr, 0);
    RunBufs B;
    if (op->dtype == SLQ_F64) carve<double>(c, r, sms, &B);
    else carve<float>(c, r, sms, &B);
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_run(slq_op* op, const slq_params* p, const double* parameters,
                              int num_inquiries, void* workspace, size_t workspace_bytes,
                              void* stream, slq_result* result)
{
    if (!result || !result->trace || !result->error || !result->samples ||
        !result->processed_samples_indices || !result->num_samples_used ||
        !result->num_outliers || !result->converged)
        return fail(SLQ_ERR_BAD_ARG, "run: result arrays missing");
    if (!op) return fail(SLQ_ERR_BAD_ARG, "run: operator is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (op->dtype == SLQ_F64)
        return run_typed<double>(op, p, parameters, num_inquiries, workspace, workspace_bytes, st,
                                 result);
    return run_typed<float>(op, p, parameters, num_inquiries, workspace, workspace_bytes, st,
                            result);
}

// ---------------------------------------------------------------------------
// SpMM autotuner
// ---------------------------------------------------------------------------

namespace {

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

struct TuneBufs {
    void* X;
    void* Y;
    double* sx;
    double* partials;
    int32_t* error;
};

void tune_layout(Carver& c, const slq_op* op, int width, int sms, TuneBufs* t)
{
    const size_t s = (op->dtype == SLQ_F64) ? 8 : 4;
    const size_t len = static_cast<size_t>(std::max(op->nrows, op->ncols));
    t->X = c.take<char>(len * width * s);
    t->Y = c.take<char>(len * width * s);
    t->sx = c.take<double>(width);
    t->partials = c.take<double>(static_cast<size_t>(sms) * 4 * width);
    t->error = c.take<int32_t>(1);
}

template <typename VT>
slq_status tune_typed(slq_op* op, int width, int transpose, int reps, const TuneBufs& t,
                      cudaStream_t st, slq_tune_result* res)
{
    Launcher L;
    L.st = st;
    SLQ_TRY(device_sms(&L.sms));
    SpmmCand c[SLQ_TUNE_MAX_CANDIDATES];
    const int nc = spmm_candidates<VT>(op, transpose, width, c);
    const int64_t xrows = transpose ? op->nrows : op->ncols;
    SLQ_CK(cudaMemsetAsync(t.X, 0, static_cast<size_t>(xrows) * width * sizeof(VT), st));
    SLQ_CK(cudaMemsetAsync(t.error, 0, sizeof(int32_t), st));
    k_fill_f64<<<(width + 255) / 256, 256, 0, st>>>(t.sx, width, 1.0);
    SLQ_LAUNCH_CK();
    XMaps map;
    bool have_map = false;
    if constexpr (sizeof(VT) == 4)
    {
        if (width == 128 || width == 256)
        {
            SLQ_TRY(make_xmaps(&map, static_cast<const float*>(t.X), xrows, width, true));
            have_map = true;
        }
    }
    EventPair ev;
    SLQ_CK(cudaEventCreate(&ev.a));
    SLQ_CK(cudaEventCreate(&ev.b));
    res->width = width;
    res->transpose = transpose;
    res->num_candidates = nc;
    res->chosen = 0;
    for (int i = 0; i < SLQ_TUNE_MAX_CANDIDATES; ++i)
    {
        res->kind[i] = res->group_rows[i] = res->lanes_vec[i] = res->slices[i] = 0;
        res->milliseconds[i] = 0.0;
    }
    for (int i = 0; i < nc; ++i)
    {
        int grid = 0;
        auto launch = [&]() {
            return spmm_cand<VT>(L, op, transpose, c[i], width, static_cast<const VT*>(t.X), t.sx,
                                 0.0, static_cast<VT*>(t.Y), nullptr, nullptr, nullptr, 1,
                                 t.partials, &grid, have_map ? &map : nullptr, t.error);
        };
        SLQ_TRY(launch());
        SLQ_CK(cudaEventRecord(ev.a, st));
        for (int r = 0; r < reps; ++r) SLQ_TRY(launch());
        SLQ_CK(cudaEventRecord(ev.b, st));
        SLQ_CK(cudaEventSynchronize(ev.b));
        float ms = 0.0f;
        SLQ_CK(cudaEventElapsedTime(&ms, ev.a, ev.b));
        res->kind[i] = c[i].kind;
        res->group_rows[i] = c[i].g;
        res->lanes_vec[i] = c[i].lv;
        res->slices[i] = c[i].ns;
        res->milliseconds[i] = static_cast<double>(ms) / reps;
        if (res->milliseconds[i] < res->milliseconds[res->chosen]) res->chosen = i;
    }
    int32_t herr = 0;
    SLQ_CK(cudaMemcpy(&herr, t.error, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (herr) return fail(SLQ_ERR_TIMEOUT, "tune: a TMA SpMM gave up waiting for its copies");
    op->tuned[transpose ? 1 : 0][log2_width(width)] = static_cast<int8_t>(res->chosen);
    return SLQ_OK;
}

slq_status check_width(const slq_op* op, int width)
{
    if (!op) return fail(SLQ_ERR_BAD_ARG, "operator is NULL");
    if (!is_pow2(width) || width > ((op->dtype == SLQ_F64) ? 512 : 1024))
        return fail(SLQ_ERR_BAD_ARG, "width must be a power of two <= 1024 (512 for float64)");
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_operator_tune_workspace_bytes(const slq_op* op, int width,
                                                        size_t* bytes)
{
    if (op && op->dense)
        return fail(SLQ_ERR_BAD_ARG, "dense operators have one product kernel (no tuning)");
    SLQ_TRY(check_width(op, width));
    if (!bytes) return fail(SLQ_ERR_BAD_ARG, "bytes is NULL");
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(nullptr, 0);
    TuneBufs t;
    tune_layout(c, op, width, sms, &t);
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_operator_tune(slq_op* op, int width, int transpose, int reps,
                                        void* workspace, size_t workspace_bytes, void* stream,
                                        slq_tune_result* result)
{
    if (op && op->dense)
        return fail(SLQ_ERR_BAD_ARG, "dense operators have one product kernel (no tuning)");
    SLQ_TRY(check_width(op, width));
    if (!result) return fail(SLQ_ERR_BAD_ARG, "tune: result is NULL");
    if (transpose && !op->t_ptr) return fail(SLQ_ERR_BAD_ARG, "tune: operator has no transpose");
    if (reps < 1) return fail(SLQ_ERR_BAD_ARG, "tune: reps must be positive");
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(workspace, workspace_bytes);
    TuneBufs t;
    tune_layout(c, op, width, sms, &t);
    if (!workspace || !c.fits()) return fail(SLQ_ERR_WORKSPACE, "tune: workspace too small");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (op->dtype == SLQ_F64) return tune_typed<double>(op, width, transpose, reps, t, st, result);
    return tune_typed<float>(op, width, transpose, reps, t, st, result);
}

extern "C" slq_status slq_operator_set_variant(slq_op* op, int width, int transpose,
                                               int candidate)
{
    if (op && op->dense)
        return fail(SLQ_ERR_BAD_ARG, "dense operators have one product kernel (no tuning)");
    SLQ_TRY(check_width(op, width));
    if (candidate < -1 || candidate >= SLQ_TUNE_MAX_CANDIDATES)
        return fail(SLQ_ERR_BAD_ARG, "set_variant: candidate out of range");
    if (candidate >= 0)
    {
        SpmmCand c[SLQ_TUNE_MAX_CANDIDATES];
        const int nc = (op->dtype == SLQ_F64)
                           ? spmm_candidates<double>(op, transpose, width, c)
                           : spmm_candidates<float>(op, transpose, width, c);
        if (candidate >= nc)
            return fail(SLQ_ERR_BAD_ARG, "set_variant: no such candidate for this operator");
    }
    op->tuned[transpose ? 1 : 0][log2_width(width)] = static_cast<int8_t>(candidate);
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// Batched estimator: every probe block of every run recorded into one CUDA
// graph, one branch per run, then the host stopping rule per run.
// ---------------------------------------------------------------------------

namespace {

struct BatchRun {
    slq_op* op = nullptr;
    slq_params p{};
    RunPlan r{};
    std::vector<double> params;
    double shift = 0.0;
    int nblocks = 0;
    RunBufs B{};
    // outputs (device, inside the batch's contiguous output region)
    double* samples = nullptr;  // [max][q]
    int32_t* size = nullptr;    // [max]
    int32_t* status = nullptr;  // [max]
    double* alpha = nullptr;    // [nblocks][m][b]
    double* beta = nullptr;
    int32_t* error = nullptr;
    uint64_t* starts = nullptr;  // [nblocks][b][4]
    int64_t launches = 0;
};

// Outputs of all runs first (one device-to-host copy brings them back), then
// each run's working buffers.
void batch_layout(Carver& c, std::vector<BatchRun>& runs, int sms, size_t* out_bytes)
{
    for (auto& R : runs)
    {
        const size_t mx = static_cast<size_t>(R.p.max_num_samples);
        R.samples = c.take<double>(mx * R.r.q);
        R.size = c.take<int32_t>(mx);
        R.status = c.take<int32_t>(mx);
        R.alpha = c.take<double>(static_cast<size_t>(R.nblocks) * R.r.m * R.r.b);
        R.beta = c.take<double>(static_cast<size_t>(R.nblocks) * R.r.m * R.r.b);
        R.error = c.take<int32_t>(1);
    }
    *out_bytes = (c.off + 255) & ~static_cast<size_t>(255);
    for (auto& R : runs)
    {
        if (R.op->dtype == SLQ_F64) carve<double>(c, R.r, sms, &R.B);
        else carve<float>(c, R.r, sms, &R.B);
        R.B.error = R.error;
        R.starts = c.take<uint64_t>(static_cast<size_t>(R.nblocks) * R.r.b * 4);
    }
}

template <typename VT>
slq_status batch_upload(BatchRun& R, cudaStream_t st)
{
    const RunPlan& r = R.r;
    RunBufs& B = R.B;
    SLQ_CK(cudaMemcpyAsync(B.params, R.params.data(), sizeof(double) * r.q,
                           cudaMemcpyHostToDevice, st));
    k_fill_f64<<<(r.b + 255) / 256, 256, 0, st>>>(B.negshift, r.b, -R.shift);
    SLQ_LAUNCH_CK();
    if (R.p.rng == SLQ_RNG_PARITY)
    {
        uint64_t cur[4];
        Poly256 advance;
        std::vector<uint64_t> polys;
        SLQ_TRY(parity_setup(&R.p, r, cur, &advance, &polys));
        SLQ_CK(cudaMemcpyAsync(B.chunk_polys, polys.data(), polys.size() * sizeof(uint64_t),
                               cudaMemcpyHostToDevice, st));
        std::vector<uint64_t> hs(static_cast<size_t>(R.nblocks) * r.b * 4, 0);
        for (int s = 0; s < R.p.max_num_samples; ++s)
        {
            for (int k = 0; k < 4; ++k) hs[static_cast<size_t>(s) * 4 + k] = cur[k];
            apply_poly(advance, cur);
        }
        SLQ_CK(cudaMemcpyAsync(R.starts, hs.data(), hs.size() * sizeof(uint64_t),
                               cudaMemcpyHostToDevice, st));
        // the copy reads a host vector that goes out of scope here
        SLQ_CK(cudaStreamSynchronize(st));
    }
    return SLQ_OK;
}

// All probe blocks of one run on stream st (recorded into the graph).
template <typename VT>
slq_status batch_enqueue(BatchRun& R, cudaStream_t st, int sms)
{
    Launcher L;
    L.st = st;
    L.sms = sms;
    const RunPlan& r = R.r;
    const slq_params* p = &R.p;
    const int max_s = p->max_num_samples;
    const double s0 = 1.0 / std::sqrt(static_cast<double>(r.nv));
    RunBufs B = R.B;
    SLQ_CK(cudaMemsetAsync(R.error, 0, sizeof(int32_t), st));
    for (int blk = 0; blk < R.nblocks; ++blk)
    {
        const int g = blk * r.b;
        const int count = std::min(r.b, max_s - g);
        B.starts = R.starts + static_cast<size_t>(blk) * r.b * 4;
        SLQ_TRY(launch_probes<VT>(L, r, p->rng, p->seed, p->first_probe + g, count, B,
                                  R.op->inv, static_cast<VT*>(B.V)));
        k_init_block<<<(r.b + 127) / 128, 128, 0, st>>>(count, r.b, r.m, s0, B.scale_v, B.active,
                                                        B.size);
        SLQ_LAUNCH_CK();
        ++L.launches;
        SLQ_TRY(krylov_block<VT>(L, R.op, p, r, B, count, R.shift));
        k_eig_quad<<<(count + 127) / 128, 128, 0, st>>>(
            count, r.b, r.m, B.alpha, B.beta, B.size, r.gram == 1, p->func, func_coeff(p),
            p->exponent, B.params, r.q, static_cast<double>(r.nv), R.samples + static_cast<size_t>(g) * r.q,
            nullptr, nullptr, R.status + g);
        SLQ_LAUNCH_CK();
        ++L.launches;
        const size_t ab = static_cast<size_t>(r.m) * r.b;
        SLQ_CK(cudaMemcpyAsync(R.size + g, B.size, sizeof(int32_t) * count,
                               cudaMemcpyDeviceToDevice, st));
        SLQ_CK(cudaMemcpyAsync(R.alpha + blk * ab, B.alpha, sizeof(double) * ab,
                               cudaMemcpyDeviceToDevice, st));
        SLQ_CK(cudaMemcpyAsync(R.beta + blk * ab, B.beta, sizeof(double) * ab,
                               cudaMemcpyDeviceToDevice, st));
    }
    R.launches = L.launches;
    return SLQ_OK;
}

slq_status batch_plan(int count, slq_op* const* ops, const slq_params* params,
                      const double* const* parameters, const int* num_inquiries,
                      std::vector<BatchRun>* runs)
{
    if (count < 1 || !ops || !params || !num_inquiries)
        return fail(SLQ_ERR_BAD_ARG, "batch: count, ops, params and num_inquiries are required");
    runs->resize(count);
    for (int i = 0; i < count; ++i)
    {
        BatchRun& R = (*runs)[i];
        if (!ops[i]) return fail(SLQ_ERR_BAD_ARG, "batch: operator " + std::to_string(i) + " is NULL");
        if (ops[i]->dense)
            return fail(SLQ_ERR_BAD_ARG, "batch: operator " + std::to_string(i) +
                                             " is dense (one product at a time)");
        R.op = ops[i];
        R.p = params[i];
        const int q = num_inquiries[i];
        SLQ_TRY(make_plan(R.op, &R.p, q, &R.r));
        R.params.assign(q, 0.0);
        if (R.op->affine && parameters && parameters[i])
            for (int j = 0; j < q; ++j) R.params[j] = parameters[i][j];
        R.shift = R.op->affine ? R.params[0] : 0.0;
        R.nblocks = (R.p.max_num_samples + R.r.b - 1) / R.r.b;
    }
    return SLQ_OK;
}

// Reference stopping rule over a run's samples, in probe order, into res
// (the same bookkeeping as run_typed's sample loop).
slq_status batch_replay(const BatchRun& R, const char* host, const char* dev_base, float ms,
                        slq_result* res)
{
    auto hp = [&](const void* d) { return host + (static_cast<const char*>(d) - dev_base); };
    const double* hs = reinterpret_cast<const double*>(hp(R.samples));
    const int32_t* hsize = reinterpret_cast<const int32_t*>(hp(R.size));
    const int32_t* hstat = reinterpret_cast<const int32_t*>(hp(R.status));
    const double* ha = reinterpret_cast<const double*>(hp(R.alpha));
    const double* hb = reinterpret_cast<const double*>(hp(R.beta));
    const int32_t herr = *reinterpret_cast<const int32_t*>(hp(R.error));
    const slq_params* p = &R.p;
    const int max_s = p->max_num_samples;
    const int q = R.r.q;
    const int m = R.r.m;
    const int b = R.r.b;
    if (!res->trace || !res->error || !res->samples || !res->processed_samples_indices ||
        !res->num_samples_used || !res->num_outliers || !res->converged)
        return fail(SLQ_ERR_BAD_ARG, "batch: result arrays missing");
    for (int64_t i = 0; i < static_cast<int64_t>(max_s) * q; ++i) res->samples[i] = NAN;
    for (int i = 0; i < max_s; ++i)
    {
        res->processed_samples_indices[i] = 0;
        if (res->lanczos_size) res->lanczos_size[i] = 0;
        if (res->probe_status) res->probe_status[i] = -1;
    }
    for (int j = 0; j < q; ++j)
    {
        res->converged[j] = 0;
        res->num_samples_used[j] = 0;
        res->num_outliers[j] = 0;
        res->trace[j] = NAN;
        res->error[j] = NAN;
    }
    if (res->alpha)
        for (int64_t i = 0; i < static_cast<int64_t>(max_s) * m; ++i) res->alpha[i] = NAN;
    if (res->beta)
        for (int64_t i = 0; i < static_cast<int64_t>(max_s) * m; ++i) res->beta[i] = NAN;
    res->num_blocks = R.nblocks;
    res->num_probes_computed = max_s;
    res->gpu_launches = R.launches;
    res->alg_wall_time = ms * 1e-3f;
    res->all_converged = 0;
    if (herr) return fail(SLQ_ERR_TIMEOUT, "a streaming kernel gave up waiting for its copies");

    int nproc = 0;
    int all = 0;
    bool eig_failed = false;
    for (int s = 0; s < max_s && !all; ++s)
    {
        const int blk = s / b;
        const int pi = s % b;
        for (int j = 0; j < q; ++j)
            res->samples[static_cast<int64_t>(s) * q + j] = hs[static_cast<size_t>(s) * q + j];
        if (res->lanczos_size) res->lanczos_size[s] = hsize[s];
        if (hstat[s] & 2) eig_failed = true;
        if (res->probe_status) res->probe_status[s] = hstat[s];
        const size_t base = static_cast<size_t>(blk) * m * b;
        for (int i = 0; i < m; ++i)
        {
            if (res->alpha)
                res->alpha[static_cast<int64_t>(s) * m + i] =
                    (i < hsize[s]) ? ha[base + static_cast<size_t>(i) * b + pi] : NAN;
            if (res->beta)
                res->beta[static_cast<int64_t>(s) * m + i] =
                    (i < hsize[s]) ? hb[base + static_cast<size_t>(i) * b + pi] : NAN;
        }
        if (R.op->affine && q > 1)
            for (int j = 0; j < q; ++j) res->converged[j] = 0;
        res->processed_samples_indices[nproc++] = s;
        all = slq_check_convergence(res->samples, q, p->min_num_samples,
                                    res->processed_samples_indices, nproc, p->confidence_level,
                                    p->error_atol, p->error_rtol, res->error,
                                    res->num_samples_used, res->converged);
    }
    slq_average_estimates(p->confidence_level, p->outlier_significance_level, q, max_s,
                          res->num_samples_used, res->processed_samples_indices, res->samples,
                          res->num_outliers, res->trace, res->error);
    res->all_converged = all;
    if (eig_failed) return fail(SLQ_ERR_EIGEN, "tridiagonal eigen-solve did not converge");
    return SLQ_OK;
}

}  // namespace

struct slq_batch {
    std::vector<BatchRun> runs;
    char* out_dev = nullptr;
    size_t out_bytes = 0;
    std::vector<char> out_host;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
    int64_t nodes = 0;
    ~slq_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

// Streams and events of one capture, released on every path.
struct CaptureRes {
    cudaStream_t origin = nullptr;
    std::vector<cudaStream_t> br;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    ~CaptureRes()
    {
        for (auto e : join)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (auto s : br)
            if (s) cudaStreamDestroy(s);
        if (origin) cudaStreamDestroy(origin);
    }
};

slq_status batch_capture(slq_batch* bt, int sms)
{
    const int count = static_cast<int>(bt->runs.size());
    const int nbr = std::min(count, 64);
    CaptureRes cr;
    SLQ_CK(cudaStreamCreateWithFlags(&cr.origin, cudaStreamNonBlocking));
    cr.br.assign(nbr, nullptr);
    cr.join.assign(nbr, nullptr);
    for (int k = 0; k < nbr; ++k)
    {
        SLQ_CK(cudaStreamCreateWithFlags(&cr.br[k], cudaStreamNonBlocking));
        SLQ_CK(cudaEventCreateWithFlags(&cr.join[k], cudaEventDisableTiming));
    }
    SLQ_CK(cudaEventCreateWithFlags(&cr.fork, cudaEventDisableTiming));

    const bool prof = g_prof.on;
    g_prof.on = false;  // no timing events inside the graph
    SLQ_CK(cudaStreamBeginCapture(cr.origin, cudaStreamCaptureModeRelaxed));
    slq_status st = SLQ_OK;
    if (cudaEventRecord(cr.fork, cr.origin) != cudaSuccess)
        st = fail(SLQ_ERR_CUDA, "batch: capture fork failed");
    for (int k = 0; k < nbr && st == SLQ_OK; ++k)
        if (cudaStreamWaitEvent(cr.br[k], cr.fork, 0) != cudaSuccess)
            st = fail(SLQ_ERR_CUDA, "batch: capture fork failed");
    // longest runs first so that each branch's queue is balanced
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::vector<double> cost(count);
    for (int i = 0; i < count; ++i)
    {
        const BatchRun& R = bt->runs[i];
        cost[i] = double(R.op->nnz + R.r.nv) * R.p.max_num_samples * R.r.m;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> load(nbr, 0.0);
    for (int oi = 0; oi < count && st == SLQ_OK; ++oi)
    {
        const int i = order[oi];
        const int k = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += cost[i];
        BatchRun& R = bt->runs[i];
        st = (R.op->dtype == SLQ_F64) ? batch_enqueue<double>(R, cr.br[k], sms)
                                      : batch_enqueue<float>(R, cr.br[k], sms);
    }
    // join every branch (also after an error, so that the capture ends cleanly)
    for (int k = 0; k < nbr; ++k)
    {
        cudaEventRecord(cr.join[k], cr.br[k]);
        cudaStreamWaitEvent(cr.origin, cr.join[k], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cr.origin, &graph);
    g_prof.on = prof;
    if (st != SLQ_OK)
    {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return st;
    }
    if (ee != cudaSuccess || !graph)
    {
        if (graph) cudaGraphDestroy(graph);
        return fail(SLQ_ERR_CUDA, std::string("batch: stream capture failed: ") +
                                      cudaGetErrorString(ee));
    }
    bt->graph = graph;
    size_t nn = 0;
    SLQ_CK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    SLQ_CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    int64_t kn = 0;
    for (auto nd : nodes)
    {
        cudaGraphNodeType ty;
        SLQ_CK(cudaGraphNodeGetType(nd, &ty));
        if (ty == cudaGraphNodeTypeKernel) ++kn;
    }
    bt->nodes = static_cast<int64_t>(nn);
    bt->kernels = kn;
    SLQ_CK(cudaGraphInstantiate(&bt->exec, graph, 0));
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_batch_workspace_bytes(int count, slq_op* const* ops,
                                                const slq_params* params,
                                                const int* num_inquiries, size_t* bytes)
{
    if (!bytes) return fail(SLQ_ERR_BAD_ARG, "bytes is NULL");
    std::vector<BatchRun> runs;
    SLQ_TRY(batch_plan(count, ops, params, nullptr, num_inquiries, &runs));
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(nullptr, 0);
    size_t ob = 0;
    batch_layout(c, runs, sms, &ob);
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_batch_create(int count, slq_op* const* ops, const slq_params* params,
                                       const double* const* parameters,
                                       const int* num_inquiries, void* workspace,
                                       size_t workspace_bytes, void* stream, slq_batch** out)
{
    if (!out) return fail(SLQ_ERR_BAD_ARG, "batch: out is NULL");
    *out = nullptr;
    std::unique_ptr<slq_batch> bt(new slq_batch());
    SLQ_TRY(batch_plan(count, ops, params, parameters, num_inquiries, &bt->runs));
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(workspace, workspace_bytes);
    batch_layout(c, bt->runs, sms, &bt->out_bytes);
    if (!workspace || !c.fits())
        return fail(SLQ_ERR_WORKSPACE, "batch: workspace too small (need " +
                                           std::to_string(c.off) + " bytes)");
    bt->out_dev = static_cast<char*>(workspace);
    bt->out_host.resize(bt->out_bytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (auto& R : bt->runs)
        SLQ_TRY((R.op->dtype == SLQ_F64) ? batch_upload<double>(R, st) : batch_upload<float>(R, st));
    SLQ_CK(cudaStreamSynchronize(st));
    SLQ_TRY(batch_capture(bt.get(), sms));
    *out = bt.release();
    return SLQ_OK;
}

extern "C" slq_status slq_batch_run(slq_batch* bt, void* stream, slq_result* results)
{
    if (!bt || !results) return fail(SLQ_ERR_BAD_ARG, "batch_run: NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    EventPair ev;
    SLQ_CK(cudaEventCreate(&ev.a));
    SLQ_CK(cudaEventCreate(&ev.b));
    SLQ_CK(cudaEventRecord(ev.a, st));
    SLQ_CK(cudaGraphLaunch(bt->exec, st));
    SLQ_CK(cudaEventRecord(ev.b, st));
    SLQ_CK(cudaMemcpyAsync(bt->out_host.data(), bt->out_dev, bt->out_bytes,
                           cudaMemcpyDeviceToHost, st));
    SLQ_CK(cudaStreamSynchronize(st));
    float ms = 0.0f;
    SLQ_CK(cudaEventElapsedTime(&ms, ev.a, ev.b));
    slq_status worst = SLQ_OK;
    for (size_t i = 0; i < bt->runs.size(); ++i)
    {
        const slq_status s =
            batch_replay(bt->runs[i], bt->out_host.data(), bt->out_dev, ms, &results[i]);
        if (s != SLQ_OK && (worst == SLQ_OK || worst == SLQ_ERR_EIGEN)) worst = s;
    }
    return worst;
}

extern "C" slq_status slq_batch_info(const slq_batch* bt, int64_t* kernels, int64_t* nodes)
{
    if (!bt) return fail(SLQ_ERR_BAD_ARG, "batch_info: batch is NULL");
    if (kernels) *kernels = bt->kernels;
    if (nodes) *nodes = bt->nodes;
    return SLQ_OK;
}

extern "C" slq_status slq_batch_destroy(slq_batch* bt)
{
    delete bt;
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// operator product, probes, nodes/weights, device info
// ---------------------------------------------------------------------------

extern "C" slq_status slq_operator_dot(slq_op* op, int transpose, double t, const void* x,
                                       void* y, int width, void* stream)
{
    if (!op || !x || !y) return fail(SLQ_ERR_BAD_ARG, "operator_dot: NULL argument");
    if (x == y) return fail(SLQ_ERR_BAD_ARG, "operator_dot: x and y must not alias");
    if (!is_pow2(width) || width > ((op->dtype == SLQ_F64) ? 512 : 1024))
        return fail(SLQ_ERR_BAD_ARG, "operator_dot: width must be a power of two");
    if (transpose && !(op->dense ? op->dt_hi != nullptr : op->t_ptr != nullptr))
        return fail(SLQ_ERR_BAD_ARG, "operator_dot: operator has no transpose");
    Launcher L;
    L.st = static_cast<cudaStream_t>(stream);
    SLQ_TRY(device_sms(&L.sms));
    const double shift = op->affine ? t : 0.0;
    int grid = 0;
    if (op->dtype == SLQ_F64)
        return op_spmm<double>(L, op, transpose, width, static_cast<const double*>(x), nullptr,
                               shift, static_cast<double*>(y), nullptr, nullptr, nullptr, 0,
                               nullptr, &grid);
    // an operator with the block format runs its block-wide products on the
    // block kernel, whose error word lives in the format buffer (checked
    // after the product)
    const bool blk = (transpose ? op->t_bstage : op->a_bstage) != nullptr && op->blk_error &&
                     (width == 128 || width == 256);
    if (blk) SLQ_CK(cudaMemsetAsync(op->blk_error, 0, sizeof(int32_t), L.st));
    SLQ_TRY(op_spmm<float>(L, op, transpose, width, static_cast<const float*>(x), nullptr, shift,
                           static_cast<float*>(y), nullptr, nullptr, nullptr, 0, nullptr, &grid,
                           nullptr, blk ? op->blk_error : nullptr));
    if (blk)
    {
        int32_t herr = 0;
        SLQ_CK(cudaMemcpyAsync(&herr, op->blk_error, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               L.st));
        SLQ_CK(cudaStreamSynchronize(L.st));
        if (herr) return fail(SLQ_ERR_TIMEOUT, "operator_dot: the block kernel gave up waiting");
    }
    return SLQ_OK;
}

// ---------------------------------------------------------------------------
// reverse Cuthill-McKee order on the device
// ---------------------------------------------------------------------------

namespace {

struct RcmBufs {
    int32_t* flag;      // [4]: CSR check, level count, first unvisited, max degree
    int32_t* degree;
    int32_t* rows;
    int32_t* deg_sorted;
    int32_t* by_degree;
    int32_t* pos;
    int32_t* claim;
    int32_t* out;
    uint64_t* keys;
    uint64_t* keys_alt;
    void* temp;
    size_t temp_bytes;
    RcmCoopState* coop;  // the one-launch order's level state and barrier
    int32_t* coop_err;
};

slq_status rcm_layout(Carver& c, int64_t n, RcmBufs* B)
{
    const int items = static_cast<int>(std::max<int64_t>(n, 1));
    size_t t1 = 0, t2 = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, t1, static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
        static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr), items);
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub sort sizing: ") + cudaGetErrorString(e));
    e = cub::DeviceRadixSort::SortKeys(nullptr, t2, static_cast<const uint64_t*>(nullptr),
                                       static_cast<uint64_t*>(nullptr), items);
    if (e != cudaSuccess)
        return fail(SLQ_ERR_CUDA, std::string("cub sort sizing: ") + cudaGetErrorString(e));
    B->flag = c.take<int32_t>(4);
    B->degree = c.take<int32_t>(n);
    B->rows = c.take<int32_t>(n);
    B->deg_sorted = c.take<int32_t>(n);
    B->by_degree = c.take<int32_t>(n);
    B->pos = c.take<int32_t>(n);
    B->claim = c.take<int32_t>(n);
    B->out = c.take<int32_t>(n);
    B->keys = c.take<uint64_t>(n);
    B->keys_alt = c.take<uint64_t>(n);
    B->temp_bytes = std::max(t1, t2);
    B->temp = c.take<char>(B->temp_bytes);
    B->coop = c.take<RcmCoopState>(1);
    B->coop_err = c.take<int32_t>(4);
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_rcm_order_device_workspace_bytes(int64_t n, size_t* bytes)
{
    if (!bytes || n < 0 || n > INT32_MAX) return fail(SLQ_ERR_BAD_ARG, "rcm_order_device: bad argument");
    Carver c(nullptr, 0);
    RcmBufs B;
    SLQ_TRY(rcm_layout(c, n, &B));
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_rcm_order_device(int64_t n, int64_t nnz, const int32_t* indptr,
                                           const int32_t* indices, int max_components,
                                           int32_t* order, int* done, void* workspace,
                                           size_t workspace_bytes, void* stream)
{
    if (!done || n < 0 || n > INT32_MAX || nnz < 0 || nnz > INT32_MAX || !indptr || !order ||
        (nnz > 0 && !indices) || max_components < 1)
        return fail(SLQ_ERR_BAD_ARG, "rcm_order_device: bad argument");
    *done = 0;
    size_t need = 0;
    SLQ_TRY(slq_rcm_order_device_workspace_bytes(n, &need));
    if (!workspace || workspace_bytes < need)
        return fail(SLQ_ERR_WORKSPACE, "rcm_order_device: workspace too small (need " +
                                           std::to_string(need) + " bytes)");
    if (n == 0)
    {
        *done = 1;
        return SLQ_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Carver c(workspace, workspace_bytes);
    RcmBufs B;
    SLQ_TRY(rcm_layout(c, n, &B));
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    const int grid = sms * 4;

    // the pattern must index inside [0, n) before any kernel follows it
    SLQ_CK(cudaMemsetAsync(B.flag, 0, 4 * sizeof(int32_t), st));
    k_check_csr<<<grid, 256, 0, st>>>(indptr, indices, n, n, nnz, B.flag);
    SLQ_LAUNCH_CK();
    k_rcm_init<<<grid, 256, 0, st>>>(indptr, n, B.degree, B.rows, B.pos, B.claim, B.flag + 3);
    SLQ_LAUNCH_CK();
    int32_t h[4] = {0, 0, 0, 0};
    SLQ_CK(read_back(h, B.flag, sizeof(h), st));
    if (h[0] & 1) return fail(SLQ_ERR_BAD_CSR, "rcm_order_device: index pointer must start at 0 and end at nnz");
    if (h[0] & 2) return fail(SLQ_ERR_BAD_CSR, "rcm_order_device: index pointer must be non-decreasing");
    if (h[0] & 4) return fail(SLQ_ERR_BAD_CSR, "rcm_order_device: index out of range");
    const int32_t maxdeg = h[3];
    const int nb = bits_for(n - 1);
    const int db = bits_for(maxdeg);
    if (nb + db + 1 > 64) return SLQ_OK;  // keys do not fit: *done stays 0

    // rows by increasing degree, ties by row (stable sort of (degree, row))
    {
        size_t tb = B.temp_bytes;
        cudaError_t e = cub::DeviceRadixSort::SortPairs(
            B.temp, tb, B.degree, B.deg_sorted, B.rows, B.by_degree, static_cast<int>(n), 0,
            db, st);
        if (e != cudaSuccess)
            return fail(SLQ_ERR_CUDA, std::string("cub sort: ") + cudaGetErrorString(e));
    }

    // every level in one cooperative launch when a warp's sort buffer holds
    // the widest row's children; else one host round per level (below)
    if (maxdeg <= 1024 && n <= (int64_t(1) << 30))
    {
        int cap = 32;
        while (cap < maxdeg) cap <<= 1;
        const int threads = 512;
        const size_t smem = static_cast<size_t>(threads / 32) * cap * sizeof(uint64_t);
        int per_sm = 0;
        bool coop = cudaFuncSetAttribute(k_rcm_coop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rcm_coop, threads,
                                                                  smem) == cudaSuccess &&
                    per_sm >= 1;
        cudaGetLastError();  // a refused attribute leaves the level rounds
        if (coop)
        {
            SLQ_CK(cudaMemsetAsync(B.coop, 0, sizeof(RcmCoopState), st));
            SLQ_CK(cudaMemsetAsync(B.coop_err, 0, 4 * sizeof(int32_t), st));
            int64_t n_arg = n;
            int maxc = max_components;
            // about two seconds at the boost clock
            long long spin_limit = 1LL << 32;
            int32_t* counts = B.deg_sorted;  // free after the degree sort
            void* args[] = {(void*)&indptr, (void*)&indices, (void*)&B.degree,
                            (void*)&B.by_degree, (void*)&n_arg, (void*)&maxc, (void*)&cap,
                            (void*)&B.pos, (void*)&B.claim, (void*)&B.out, (void*)&counts,
                            (void*)&B.coop, (void*)&B.coop_err, (void*)&spin_limit};
            SLQ_CK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_rcm_coop),
                                               dim3(sms), dim3(threads), args, smem, st));
            int32_t herr = 0;
            RcmCoopState hs{};
            SLQ_CK(read_back(&herr, B.coop_err, sizeof(int32_t), st));
            SLQ_CK(read_back(&hs, B.coop, sizeof(hs), st));
            if (herr & 64) return SLQ_OK;  // more components than asked for: *done stays 0
            if (herr & 16)
                return fail(SLQ_ERR_TIMEOUT, "rcm_order_device: a grid barrier wait ran out");
            if (herr != 0 || !hs.done || hs.cnt != n)
                return fail(SLQ_ERR_CUDA, "rcm_order_device: lost track of the visited rows");
            k_rcm_reverse<<<grid, 256, 0, st>>>(B.out, n, order);
            SLQ_LAUNCH_CK();
            *done = 1;
            return SLQ_OK;
        }
    }

    const int32_t first_init = static_cast<int32_t>(n);
    int64_t cnt = 0, cursor = 0;
    int components = 0;
    while (cnt < n)
    {
        if (++components > max_components) return SLQ_OK;  // *done stays 0
        SLQ_CK(cudaMemcpyAsync(B.flag + 2, &first_init, sizeof(int32_t), cudaMemcpyHostToDevice, st));
        k_rcm_first<<<grid, 256, 0, st>>>(B.by_degree, B.pos, cursor, n, B.flag + 2);
        SLQ_LAUNCH_CK();
        k_rcm_start<<<1, 1, 0, st>>>(B.by_degree, B.flag + 2, B.pos, B.out, cnt, n);
        SLQ_LAUNCH_CK();
        int32_t first = 0;
        SLQ_CK(read_back(&first, B.flag + 2, sizeof(int32_t), st));
        if (first >= n) return fail(SLQ_ERR_CUDA, "rcm_order_device: lost track of the visited rows");
        cursor = first + 1;
        int64_t lb = cnt, le = cnt + 1;
        cnt = le;
        while (lb < le)
        {
            const int pb = bits_for(le - lb - 1);
            if (pb + db + nb > 64) return SLQ_OK;  // *done stays 0
            const int64_t warps = le - lb;
            const int blocks = static_cast<int>(std::min<int64_t>((warps + 7) / 8, int64_t(sms) * 8));
            k_rcm_claim<<<blocks, 256, 0, st>>>(B.out, lb, le, indptr, indices, B.pos, B.claim,
                                                 B.flag + 1);
            SLQ_LAUNCH_CK();
            k_rcm_collect<<<blocks, 256, 0, st>>>(B.out, lb, le, indptr, indices, B.pos, B.degree,
                                                   B.claim, nb, db, B.keys, B.flag + 1);
            SLQ_LAUNCH_CK();
            int32_t m = 0;
            SLQ_CK(read_back(&m, B.flag + 1, sizeof(int32_t), st));
            if (m < 0 || cnt + m > n)
                return fail(SLQ_ERR_CUDA, "rcm_order_device: level count out of range");
            if (m > 0)
            {
                cub::DoubleBuffer<uint64_t> kb(B.keys, B.keys_alt);
                size_t tb = B.temp_bytes;
                cudaError_t e = cub::DeviceRadixSort::SortKeys(B.temp, tb, kb, static_cast<int>(m),
                                                               0, pb + db + nb, st);
                if (e != cudaSuccess)
                    return fail(SLQ_ERR_CUDA, std::string("cub sort: ") + cudaGetErrorString(e));
                const uint64_t rowmask = (uint64_t(1) << nb) - 1;
                const int ab = static_cast<int>(std::min<int64_t>((m + 255) / 256, grid));
                k_rcm_assign<<<ab, 256, 0, st>>>(kb.Current(), m, rowmask, cnt, B.out, B.pos);
                SLQ_LAUNCH_CK();
            }
            lb = le;
            le = cnt + m;
            cnt = le;
        }
    }
    k_rcm_reverse<<<grid, 256, 0, st>>>(B.out, n, order);
    SLQ_LAUNCH_CK();
    *done = 1;
    return SLQ_OK;
}


extern "C" slq_status slq_dense_operator_workspace_bytes(int64_t num_rows, int64_t num_cols,
                                                         int dtype, int need_transpose,
                                                         size_t* bytes)
{
    if (!bytes || num_rows < 1 || num_cols < 1 || num_rows > INT32_MAX || num_cols > INT32_MAX)
        return fail(SLQ_ERR_BAD_ARG, "dense_operator: bad size");
    if (dtype != SLQ_F32)
        return fail(SLQ_ERR_BAD_ARG, "dense_operator: float32 data only");
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(nullptr, 0);
    DenseBufs d;
    dense_layout(c, num_rows, num_cols, need_transpose, sms, &d);
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_dense_operator_create(const void* data, int64_t num_rows,
                                                int64_t num_cols, int dtype, int affine,
                                                int need_transpose, void* workspace,
                                                size_t workspace_bytes, void* stream,
                                                slq_op** out)
{
    if (!out || !data) return fail(SLQ_ERR_BAD_ARG, "dense_operator: NULL argument");
    size_t need = 0;
    SLQ_TRY(slq_dense_operator_workspace_bytes(num_rows, num_cols, dtype, need_transpose,
                                               &need));
    if (!workspace || workspace_bytes < need)
        return fail(SLQ_ERR_WORKSPACE, "dense_operator: workspace too small (need " +
                                           std::to_string(need) + " bytes)");
    if (affine && num_rows != num_cols)
        return fail(SLQ_ERR_BAD_ARG, "dense_operator: A + t I needs a square A");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int sms = 0;
    SLQ_TRY(device_sms(&sms));
    Carver c(workspace, workspace_bytes);
    DenseBufs d;
    dense_layout(c, num_rows, num_cols, need_transpose, sms, &d);
    // zero padding, then the parts
    SLQ_CK(cudaMemsetAsync(workspace, 0, c.off, st));
    const float* A = static_cast<const float*>(data);
    k_split_rows<<<sms * 8, 256, 0, st>>>(A, num_rows, num_cols, num_cols, d.ldk, d.hi, d.lo);
    SLQ_LAUNCH_CK();
    if (need_transpose)
    {
        dim3 tg(static_cast<unsigned>((num_rows + 31) / 32),
                static_cast<unsigned>((num_cols + 31) / 32));
        k_split_transpose<<<tg, dim3(32, 8), 0, st>>>(A, num_rows, num_cols, 0, num_cols,
                                                      d.ldk_t, d.t_hi, d.t_lo);
        SLQ_LAUNCH_CK();
    }
    slq_op* op = new slq_op();
    op->dtype = dtype;
    op->affine = affine;
    op->nrows = num_rows;
    op->ncols = num_cols;
    op->nnz = num_rows * num_cols;
    op->dense = 1;
    op->d_hi = d.hi;
    op->d_lo = d.lo;
    op->dt_hi = d.t_hi;
    op->dt_lo = d.t_lo;
    op->ldk = d.ldk;
    op->ldk_t = d.ldk_t;
    op->ldx = d.ldx;
    op->xt_hi = d.x_hi;
    op->xt_lo = d.x_lo;
    op->d_acc = d.acc;
    op->dense_sms = sms;
    op->d_error = d.error;
    slq_status s = part_map(&op->map_hi, d.hi, d.ldk, num_rows, 128);
    if (s == SLQ_OK) s = part_map(&op->map_lo, d.lo, d.ldk, num_rows, 128);
    if (s == SLQ_OK && need_transpose) s = part_map(&op->map_t_hi, d.t_hi, d.ldk_t, num_cols, 128);
    if (s == SLQ_OK && need_transpose) s = part_map(&op->map_t_lo, d.t_lo, d.ldk_t, num_cols, 128);
    if (s != SLQ_OK)
    {
        delete op;
        return s;
    }
    *out = op;
    return SLQ_OK;
}


extern "C" slq_status slq_generate_probes_workspace_bytes(int64_t len, int width,
                                                          size_t* bytes)
{
    if (!bytes || len <= 0 || width <= 0) return fail(SLQ_ERR_BAD_ARG, "bad argument");
    const int64_t wpp = len / 64 + 1;
    int cw = 64;
    while ((wpp + cw - 1) / cw > 65535) cw *= 2;
    const int64_t nchunks = (wpp + cw - 1) / cw;
    Carver c(nullptr, 0);
    c.take<uint64_t>(static_cast<size_t>(width) * 4);
    c.take<uint64_t>(static_cast<size_t>(nchunks) * 4);
    *bytes = c.off + 256;
    return SLQ_OK;
}

extern "C" slq_status slq_generate_probes(int64_t seed, int rng, int64_t len, int64_t first,
                                          int count, int width, int dtype, void* out,
                                          void* workspace, size_t workspace_bytes, void* stream)
{
    if (!out || len <= 0 || first < 0 || count < 0 || width <= 0 || count > width ||
        seed < 0 || (rng != SLQ_RNG_PARITY && rng != SLQ_RNG_FAST))
        return fail(SLQ_ERR_BAD_ARG, "generate_probes: bad argument");
    size_t need = 0;
    SLQ_TRY(slq_generate_probes_workspace_bytes(len, width, &need));
    if (!workspace || workspace_bytes < need)
        return fail(SLQ_ERR_WORKSPACE, "generate_probes: workspace too small");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RunPlan r;
    r.nv = len;
    r.b = width;
    r.wpp = len / 64 + 1;
    r.cw = 64;
    while ((r.wpp + r.cw - 1) / r.cw > 65535) r.cw *= 2;
    r.nchunks = static_cast<int>((r.wpp + r.cw - 1) / r.cw);
    Carver c(workspace, workspace_bytes);
    RunBufs B;
    B.starts = c.take<uint64_t>(static_cast<size_t>(width) * 4);
    B.chunk_polys = c.take<uint64_t>(static_cast<size_t>(r.nchunks) * 4);
    if (rng == SLQ_RNG_PARITY)
    {
        if (!self_check()) return fail(SLQ_ERR_CUDA, "jump polynomial self-check failed");
        uint64_t cur[4];
        stream_state(seed, cur);
        jump_ahead(cur, static_cast<uint64_t>(first) * static_cast<uint64_t>(r.wpp));
        const Poly256 adv = jump_poly(static_cast<uint64_t>(r.wpp));
        std::vector<uint64_t> hs(static_cast<size_t>(width) * 4, 0);
        for (int pi = 0; pi < count; ++pi)
        {
            for (int k = 0; k < 4; ++k) hs[static_cast<size_t>(pi) * 4 + k] = cur[k];
            apply_poly(adv, cur);
        }
        std::vector<uint64_t> polys(static_cast<size_t>(r.nchunks) * 4);
        const Poly256 step = jump_poly(static_cast<uint64_t>(r.cw));
        Poly256 acc = {{1, 0, 0, 0}};
        for (int ci = 0; ci < r.nchunks; ++ci)
        {
            for (int k = 0; k < 4; ++k) polys[static_cast<size_t>(ci) * 4 + k] = acc.w[k];
            acc = poly_mulmod(acc, step);
        }
        SLQ_CK(cudaMemcpyAsync(B.starts, hs.data(), hs.size() * 8, cudaMemcpyHostToDevice, st));
        SLQ_CK(cudaMemcpyAsync(B.chunk_polys, polys.data(), polys.size() * 8,
                               cudaMemcpyHostToDevice, st));
        SLQ_CK(cudaStreamSynchronize(st));  // host vectors go out of scope
    }
    Launcher L;
    L.st = st;
    SLQ_TRY(device_sms(&L.sms));
    if (dtype == SLQ_F64)
        return launch_probes<double>(L, r, rng, seed, first, count, B, nullptr,
                                     static_cast<double*>(out));
    return launch_probes<float>(L, r, rng, seed, first, count, B, nullptr,
                                static_cast<float*>(out));
}

// ---------------------------------------------------------------------------
// Probe generation that allocates nothing (slq_generate_probes_noalloc).
//
// Some callers cannot hand the engine a workspace: code whose device memory
// is wholly owned by a caching allocator or a fixed-size arena (a direct
// cudaMalloc there fails or fragments the pool), and latency-critical paths
// that cannot afford the device-wide synchronisation cudaFree may trigger.
// For them the generator keeps its scratch -- per-probe xoshiro256** start
// states and per-chunk jump polynomials -- in a file-scope device array of
// fixed size.  Every GPU that loads this library holds the array (288 KB)
// until the process exits.
// ---------------------------------------------------------------------------

namespace {
constexpr int NOALLOC_MAX_WIDTH = 1024;    // probes per call
constexpr int NOALLOC_MAX_CHUNKS = 8192;   // parallel chunks per probe
constexpr size_t NOALLOC_WORDS =
    static_cast<size_t>(NOALLOC_MAX_WIDTH + NOALLOC_MAX_CHUNKS) * 4;
constexpr int NOALLOC_MAX_DEVICES = 64;

std::mutex g_noalloc_mutex;
// device address of the scratch array, per device (host code must not use
// the array's name as a device pointer).  Resolved by the first call on a
// device and kept for the process: a cudaDeviceReset (or any reset of the
// device's primary context) reloads the module and may move the array, after
// which this cached address is stale, so this entry point must not be called
// again on a device after its context was reset.
uint64_t* g_noalloc_dev[NOALLOC_MAX_DEVICES] = {};
// host staging of the scratch contents (static storage, no heap)
uint64_t g_noalloc_host[NOALLOC_WORDS];
}  // namespace

// starts: words [0, 4*NOALLOC_MAX_WIDTH); chunk polynomials after them
static __device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_WORDS];

extern "C" slq_status slq_generate_probes_noalloc(int64_t seed, int rng, int64_t len,
                                                  int64_t first, int count, int width,
                                                  int dtype, void* out, void* stream)
{
    if (!out || len <= 0 || first < 0 || count < 0 || width <= 0 || count > width ||
        seed < 0 || (rng != SLQ_RNG_PARITY && rng != SLQ_RNG_FAST) ||
        (dtype != SLQ_F32 && dtype != SLQ_F64))
        return fail(SLQ_ERR_BAD_ARG, "generate_probes_noalloc: bad argument");
    if (width > NOALLOC_MAX_WIDTH)
        return fail(SLQ_ERR_BAD_ARG,
                    "generate_probes_noalloc: width " + std::to_string(width) +
                        " exceeds the static scratch limit of " +
                        std::to_string(NOALLOC_MAX_WIDTH) + " probes per call");
    int dev = 0;
    SLQ_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(SLQ_ERR_BAD_ARG, "generate_probes_noalloc: device index out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (rng == SLQ_RNG_PARITY)
    {
        // parity mode stages its scratch through host memory and waits for
        // the copies; both would break a capture the caller has open on this
        // stream, so refuse before touching the stream
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        SLQ_CK(cudaStreamIsCapturing(st, &cap));
        if (cap != cudaStreamCaptureStatusNone)
            return fail(SLQ_ERR_BAD_ARG,
                        "generate_probes_noalloc: the parity probe stream (rng = "
                        "SLQ_RNG_PARITY) copies host staging and synchronizes the "
                        "stream, which a stream capture does not allow");
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_dev[dev])
    {
        // first call on this device (the device is current): resolve the
        // array's device address once
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(SLQ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e));
        g_noalloc_dev[dev] = static_cast<uint64_t*>(ptr);
    }
    uint64_t* scratch = g_noalloc_dev[dev];

    RunPlan r;
    r.nv = len;
    r.b = width;
    r.wpp = len / 64 + 1;
    r.cw = 64;
    while ((r.wpp + r.cw - 1) / r.cw > NOALLOC_MAX_CHUNKS) r.cw *= 2;
    r.nchunks = static_cast<int>((r.wpp + r.cw - 1) / r.cw);
    RunBufs B;
    B.starts = scratch;
    B.chunk_polys = scratch + static_cast<size_t>(NOALLOC_MAX_WIDTH) * 4;
    if (rng == SLQ_RNG_PARITY)
    {
        if (!self_check()) return fail(SLQ_ERR_CUDA, "jump polynomial self-check failed");
        uint64_t cur[4];
        stream_state(seed, cur);
        jump_ahead(cur, static_cast<uint64_t>(first) * static_cast<uint64_t>(r.wpp));
        const Poly256 adv = jump_poly(static_cast<uint64_t>(r.wpp));
        uint64_t* hs = g_noalloc_host;
        uint64_t* hp = g_noalloc_host + static_cast<size_t>(NOALLOC_MAX_WIDTH) * 4;
        for (int pi = 0; pi < count; ++pi)
        {
            for (int k = 0; k < 4; ++k) hs[static_cast<size_t>(pi) * 4 + k] = cur[k];
            apply_poly(adv, cur);
        }
        const Poly256 step = jump_poly(static_cast<uint64_t>(r.cw));
        Poly256 acc = {{1, 0, 0, 0}};
        for (int ci = 0; ci < r.nchunks; ++ci)
        {
            for (int k = 0; k < 4; ++k) hp[static_cast<size_t>(ci) * 4 + k] = acc.w[k];
            acc = poly_mulmod(acc, step);
        }
        SLQ_CK(cudaMemcpyAsync(B.starts, hs, sizeof(uint64_t) * 4 * static_cast<size_t>(count),
                               cudaMemcpyHostToDevice, st));
        SLQ_CK(cudaMemcpyAsync(B.chunk_polys, hp,
                               sizeof(uint64_t) * 4 * static_cast<size_t>(r.nchunks),
                               cudaMemcpyHostToDevice, st));
        // the host staging is reused by the next call
        SLQ_CK(cudaStreamSynchronize(st));
    }
    Launcher L;
    L.st = st;
    SLQ_TRY(device_sms(&L.sms));
    if (dtype == SLQ_F64)
        return launch_probes<double>(L, r, rng, seed, first, count, B, nullptr,
                                     static_cast<double*>(out));
    return launch_probes<float>(L, r, rng, seed, first, count, B, nullptr,
                                static_cast<float*>(out));
}

extern "C" slq_status slq_nodes_weights(const double* alpha, const double* beta,
                                        const int32_t* sizes, int count, int m, int gram,
                                        double* theta, double* tau, int32_t* status,
                                        void* stream)
{
    if (!alpha || !beta || !sizes || !theta || !tau || !status || count <= 0 || m <= 0 ||
        m > EIG_MAX)
        return fail(SLQ_ERR_BAD_ARG, "nodes_weights: bad argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_eig_quad<<<(count + 127) / 128, 128, 0, st>>>(count, count, m, alpha, beta, sizes, gram, 0,
                                                   make_double4(0.0, 0.0, 0.0, 0.0), 1.0, nullptr,
                                                   0, 1.0, nullptr, theta, tau, status);
    SLQ_LAUNCH_CK();
    return SLQ_OK;
}

extern "C" slq_status slq_device_info(int* num_devices, int* num_sms, int* max_threads_per_sm)
{
    int n = 0;
    SLQ_CK(cudaGetDeviceCount(&n));
    if (num_devices) *num_devices = n;
    if (n > 0)
    {
        int dev = 0;
        SLQ_CK(cudaGetDevice(&dev));
        if (num_sms) SLQ_CK(cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, dev));
        if (max_threads_per_sm)
            SLQ_CK(cudaDeviceGetAttribute(max_threads_per_sm,
                                          cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    }
    return SLQ_OK;
}

extern "C" void slq_xoshiro_jump_ahead(uint64_t* state, uint64_t k) { jump_ahead(state, k); }

extern "C" const char* slq_last_error(void) { return g_error.c_str(); }

namespace slq {
void set_error(const std::string& message) { g_error = message; }
}  // namespace slq

extern "C" slq_status slq_tc_selftest(const float* a, const float* b, float* d, int mode,
                                      int32_t* error, void* stream)
{
    if (!a || !b || !d || !error) return fail(SLQ_ERR_BAD_ARG, "tc_selftest: NULL argument");
    if (mode < 0 || mode > 3) return fail(SLQ_ERR_BAD_ARG, "tc_selftest: mode must be 0..3");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SLQ_CK(cudaMemsetAsync(error, 0, sizeof(int32_t), st));
    k_tc_selftest<<<1, 128, 0, st>>>(a, b, d, mode, error);
    SLQ_LAUNCH_CK();
    int32_t herr = 0;
    SLQ_CK(cudaMemcpyAsync(&herr, error, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SLQ_CK(cudaStreamSynchronize(st));
    if (herr) return fail(SLQ_ERR_TIMEOUT, "tc_selftest: the MMA did not complete");
    return SLQ_OK;
}

extern "C" slq_status slq_tc_selftest_mn(const float* a, const float* b, float* d, int gather,
                                         int32_t* error, void* stream)
{
    if (!a || !b || !d || !error) return fail(SLQ_ERR_BAD_ARG, "tc_selftest_mn: NULL argument");
    if (gather != 0 && gather != 1)
        return fail(SLQ_ERR_BAD_ARG, "tc_selftest_mn: gather must be 0 or 1");
    if (reinterpret_cast<uintptr_t>(b) % 16 != 0)
        return fail(SLQ_ERR_BAD_ARG, "tc_selftest_mn: b must be 16-byte aligned");
    if (!g_encode_tiled)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SLQ_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess)
            return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    // B as [8][32] FP32 rows of 128 bytes, one row per box (gather4 form)
    CUtensorMap bmap;
    cuuint64_t dims[2] = {32, 8};
    cuuint64_t strides[1] = {32 * sizeof(float)};
    cuuint32_t box[2] = {32, 1};
    cuuint32_t es[2] = {1, 1};
    const CUresult r = g_encode_tiled(&bmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                      const_cast<float*>(b), dims, strides, box, es,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                                      CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(SLQ_ERR_CUDA, "cuTensorMapEncodeTiled (selftest) failed (" +
                                      std::to_string(int(r)) + ")");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SLQ_CK(cudaMemsetAsync(error, 0, sizeof(int32_t), st));
    k_tc_selftest_mn<<<1, 128, 0, st>>>(bmap, a, b, d, gather, error);
    SLQ_LAUNCH_CK();
    int32_t herr = 0;
    SLQ_CK(cudaMemcpyAsync(&herr, error, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SLQ_CK(cudaStreamSynchronize(st));
    if (herr) return fail(SLQ_ERR_TIMEOUT, "tc_selftest_mn: a wait did not complete");
    return SLQ_OK;
}

extern "C" int slq_abi_version(void) { return SLQ_ABI_VERSION; }

extern "C" slq_status slq_debug_blocks_sorted_keys(int on)
{
    if (on != 0 && on != 1) return fail(SLQ_ERR_BAD_ARG, "debug_blocks_sorted_keys: on must be 0 or 1");
    g_blk_sorted_keys.store(on);
    return SLQ_OK;
}

extern "C" slq_status slq_debug_fail_stream_waits(int count)
{
    if (count < 0) return fail(SLQ_ERR_BAD_ARG, "debug_fail_stream_waits: count < 0");
    g_fail_stream_waits.store(count);
    return SLQ_OK;
}
