// Device kernels of the B200 SLQ engine.
//
// Data layout.  A probe block is b column vectors stored row-major, [len][b]:
// element (row r, probe p) at r*b + p, so one matrix row's gather reads b
// contiguous values (one 128-byte line per 32 FP32 probes) and every vector
// kernel streams contiguous memory.  A Krylov basis is bs such blocks
// ("slots") back to back; slot (v mod bs) holds basis vector v, stored
// unnormalised together with a per-probe scale ([bs][b] doubles) so that a
// normalisation never needs its own pass over the vector.
//
// Precision.  Vector storage and SpMM accumulation use the operator's dtype
// (FP32 in mixed mode, FP64 in FP64 mode); every reduction (alpha, beta,
// reorthogonalisation inner products) accumulates in FP64, and the
// three-term update and reorthogonalisation subtraction are evaluated in
// FP64 before rounding to storage.  The tridiagonal eigen-solve and the
// quadrature run in FP64.
//
// Reductions are deterministic: each CTA writes its partial sums to a
// [grid][cols] buffer and k_finalize sums them in a fixed order.

#ifndef SLQ_KERNELS_CUH_
#define SLQ_KERNELS_CUH_

#include <cuda_fp16.h>
#include <climits>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "slq_tc.cuh"

namespace slq {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int MAX_J = 64;  // basis vectors per streaming-pass launch

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

template <typename VT, int N>
__device__ __forceinline__ void load_n(const VT* p, VT (&v)[N])
{
    constexpr int BYTES = N * static_cast<int>(sizeof(VT));
    if constexpr (BYTES % 16 == 0)
    {
        const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i)
        {
            uint4 t = q[i];
            memcpy(reinterpret_cast<char*>(v) + 16 * i, &t, 16);
        }
    }
    else if constexpr (BYTES % 8 == 0)
    {
        const uint2* q = reinterpret_cast<const uint2*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i)
        {
            uint2 t = q[i];
            memcpy(reinterpret_cast<char*>(v) + 8 * i, &t, 8);
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = p[i];
    }
}

// read-only path for gathers from a buffer no thread of the kernel writes
template <typename VT, int N>
__device__ __forceinline__ void ldg_n(const VT* p, VT (&v)[N])
{
    constexpr int BYTES = N * static_cast<int>(sizeof(VT));
    if constexpr (BYTES % 16 == 0)
    {
        const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i)
        {
            uint4 t = __ldg(q + i);
            memcpy(reinterpret_cast<char*>(v) + 16 * i, &t, 16);
        }
    }
    else if constexpr (BYTES % 8 == 0)
    {
        const uint2* q = reinterpret_cast<const uint2*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i)
        {
            uint2 t = __ldg(q + i);
            memcpy(reinterpret_cast<char*>(v) + 8 * i, &t, 8);
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = __ldg(p + i);
    }
}

template <typename VT, int N>
__device__ __forceinline__ void store_n(VT* p, const VT (&v)[N])
{
    constexpr int BYTES = N * static_cast<int>(sizeof(VT));
    if constexpr (BYTES % 16 == 0)
    {
        uint4* q = reinterpret_cast<uint4*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i)
        {
            uint4 t;
            memcpy(&t, reinterpret_cast<const char*>(v) + 16 * i, 16);
            q[i] = t;
        }
    }
    else if constexpr (BYTES % 8 == 0)
    {
        uint2* q = reinterpret_cast<uint2*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i)
        {
            uint2 t;
            memcpy(&t, reinterpret_cast<const char*>(v) + 8 * i, 8);
            q[i] = t;
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < N; ++i) p[i] = v[i];
    }
}

__device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ int ring_slot(int vec, int bs)
{
    int s = vec % bs;
    return s < 0 ? s + bs : s;
}

// ---------------------------------------------------------------------------
// CSR SpMM: Y = sx * (A X) [+ shift * sx * X] [- zc * zs * Z]
//
// One warp per matrix row; the row's b probe columns are split over the
// lanes: P = b / LV lanes, each owning LV consecutive probes, and KS = 32/P
// lane slices that walk alternate nonzeros of the row (KS > 1 only for
// b < 32).  Column indices and values are read coalesced 32 at a time and
// broadcast by shuffle; each nonzero then costs one contiguous LV-wide
// gather per lane (the whole warp reads b contiguous values of X).  The
// epilogue applies the per-probe scale and the Krylov recurrence's axpy and
// accumulates the FP64 partial of alpha (Lanczos) or of the squared norm.
//
// epi: 0 store only, 1 alpha partial <sx X[r], Y[r]>, 2 norm partial
// |Y[r]|^2, 3 alpha partial <zs Z[r], Y[r]> (normal-equations Lanczos, where
// the Krylov vector is Z and X is the intermediate A v)
// ---------------------------------------------------------------------------

// resident 256-thread blocks per SM the FP32 CSR kernel is compiled for:
// more warps keep more row gathers in flight (short rows issue few per warp)
template <typename VT, int LV>
struct SpmmOcc {
    static constexpr int MINB = (sizeof(VT) != 4) ? 1 : (LV <= 4) ? 4 : (LV == 8 ? 3 : 1);
};

template <typename VT, int LV, int KS>
__global__ void __launch_bounds__(256, SpmmOcc<VT, LV>::MINB)
k_spmm(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
       const VT* __restrict__ vals, int64_t nrows, int b,
       const VT* __restrict__ X, const double* __restrict__ sx, double shift,
       VT* __restrict__ Y, const VT* __restrict__ Z,
       const double* __restrict__ zc, const double* __restrict__ zs, int epi,
       double* __restrict__ partials)
{
    constexpr int P = 32 / KS;
    extern __shared__ double smem_spmm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int pl = lane % P;
    const int ks = lane / P;
    const int p0 = pl * LV;

    double part[LV];
#pragma unroll
    for (int v = 0; v < LV; ++v) part[v] = 0.0;

    const int64_t gw = static_cast<int64_t>(blockIdx.x) * nwarps + warp;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * nwarps;
    for (int64_t row = gw; row < nrows; row += stride)
    {
        const int k0 = indptr[row];
        const int k1 = indptr[row + 1];
        VT acc[LV];
#pragma unroll
        for (int v = 0; v < LV; ++v) acc[v] = VT(0);

        for (int base = k0; base < k1; base += 32)
        {
            const int kk = base + lane;
            int c = 0;
            VT a = VT(0);
            if (kk < k1)
            {
                c = __ldg(indices + kk);
                a = __ldg(vals + kk);
            }
            const int cnt = min(32, k1 - base);
            int t = 0;
            // four nonzeros per lane slice in flight
            for (; t + 4 * KS <= cnt; t += 4 * KS)
            {
                int cc[4];
                VT aa[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    cc[u] = __shfl_sync(FULL_MASK, c, t + u * KS + ks);
                    aa[u] = __shfl_sync(FULL_MASK, a, t + u * KS + ks);
                }
                VT x[4][LV];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    ldg_n<VT, LV>(X + static_cast<int64_t>(cc[u]) * b + p0, x[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < LV; ++v) acc[v] += aa[u] * x[u][v];
            }
            for (; t < cnt; t += KS)
            {
                const int src = t + ks;
                const int cc = __shfl_sync(FULL_MASK, c, src & 31);
                const VT aa = __shfl_sync(FULL_MASK, a, src & 31);
                if (src < cnt)
                {
                    VT x[LV];
                    ldg_n<VT, LV>(X + static_cast<int64_t>(cc) * b + p0, x);
#pragma unroll
                    for (int v = 0; v < LV; ++v) acc[v] += aa * x[v];
                }
            }
        }
        if constexpr (KS > 1)
        {
#pragma unroll
            for (int off = P; off < 32; off <<= 1)
#pragma unroll
                for (int v = 0; v < LV; ++v)
                    acc[v] += __shfl_xor_sync(FULL_MASK, acc[v], off);
        }
        if (ks == 0)
        {
            const int64_t o = row * b + p0;
            VT xr[LV], zr[LV], yr[LV];
            if (shift != 0.0 || epi == 1) ldg_n<VT, LV>(X + o, xr);
            if (Z) ldg_n<VT, LV>(Z + o, zr);
#pragma unroll
            for (int v = 0; v < LV; ++v)
            {
                // per-probe scales from L1 (not held in registers)
                const double sxv = sx ? __ldg(sx + p0 + v) : 1.0;
                double y = static_cast<double>(acc[v]) * sxv;
                if (shift != 0.0)
                    y += shift * (sxv * static_cast<double>(xr[v]));
                if (Z) y -= (__ldg(zc + p0 + v) * __ldg(zs + p0 + v)) * static_cast<double>(zr[v]);
                yr[v] = static_cast<VT>(y);
                const double ys = static_cast<double>(yr[v]);
                if (epi == 1)
                    part[v] += (sxv * static_cast<double>(xr[v])) * ys;
                else if (epi == 2)
                    part[v] += ys * ys;
                else if (epi == 3)
                    part[v] += (zs[p0 + v] * static_cast<double>(zr[v])) * ys;
            }
            store_n<VT, LV>(Y + o, yr);
        }
    }

    if (epi == 0) return;
    // CTA reduction over warps, fixed order
    if (ks == 0)
#pragma unroll
        for (int v = 0; v < LV; ++v) smem_spmm[warp * b + p0 + v] = part[v];
    __syncthreads();
    for (int p = threadIdx.x; p < b; p += blockDim.x)
    {
        double s = 0.0;
        for (int w = 0; w < nwarps; ++w) s += smem_spmm[w * b + p];
        partials[static_cast<int64_t>(blockIdx.x) * b + p] = s;
    }
}

// ---------------------------------------------------------------------------
// Deterministic column sums of a [nparts][cols] partials buffer, followed by
// the per-column finalisation of one Krylov quantity.
//   FIN_STORE : out[col] = sum                        (alpha_j, Lanczos)
//   FIN_COEF  : col = i*b + p -> coef[col] = sum * s_i(p)^2 (reorth coefs)
//   FIN_NORM  : nrm = sqrt(sum); out[p] = nrm; next_scale[p] = active ? 1/nrm
//               : 0; with check_break, probes whose nrm < thr stop at size
//               step+1 (the breakdown test of c_lanczos_tridiagonalization
//               .cpp:225-228).
// 32 x 32 threads: 32 columns per CTA, 32 partial rows per column.
// ---------------------------------------------------------------------------

enum { FIN_STORE = 0, FIN_COEF = 1, FIN_NORM = 2 };

template <typename VT>
__global__ void __launch_bounds__(1024)
k_finalize(const double* __restrict__ partials, int nparts, int cols, int mode,
           double* __restrict__ out, VT* __restrict__ coef,
           const double* __restrict__ scales, int b, int bs, int last,
           double* __restrict__ next_scale, int32_t* __restrict__ active,
           int32_t* __restrict__ size, int check_break, double thr, int step)
{
    __shared__ double red[32][33];
    const int cx = threadIdx.x & 31;
    const int cy = threadIdx.x >> 5;
    const int col = blockIdx.x * 32 + cx;
    double s = 0.0;
    if (col < cols)
        for (int q = cy; q < nparts; q += 32)
            s += partials[static_cast<int64_t>(q) * cols + col];
    red[cy][cx] = s;
    __syncthreads();
    if (cy != 0 || col >= cols) return;
    double t = 0.0;
    for (int q = 0; q < 32; ++q) t += red[q][cx];

    if (mode == FIN_STORE)
    {
        out[col] = t;
    }
    else if (mode == FIN_COEF)
    {
        const int i = col / b;
        const int p = col % b;
        const double si = scales[static_cast<int64_t>(ring_slot(last - i, bs)) * b + p];
        coef[col] = static_cast<VT>(t * si * si);
    }
    else
    {
        const int p = col;
        const double nrm = sqrt(t);
        out[p] = nrm;
        int act = active[p];
        if (act && check_break && nrm < thr)
        {
            size[p] = step + 1;
            act = 0;
            active[p] = 0;
        }
        next_scale[p] = act ? 1.0 / nrm : 0.0;
    }
}

// ---------------------------------------------------------------------------
// Nodes, weights and quadrature, one thread per probe.
//
// Implicit QL with Wilkinson shifts on the symmetric tridiagonal T (the
// Jacobi matrix of Lanczos, or B^T B for Golub-Kahn's upper bidiagonal B),
// tracking only the first row of the eigenvector matrix (Golub & Welsch):
// theta = eigenvalues, tau = first eigenvector entries.  The sample of
// inquiry j is  nscale * sum_i tau_i^2 f((theta_i - t_0 + t_j)^p)
// (c_trace_estimator.cpp:564-629).
// ---------------------------------------------------------------------------

constexpr int EIG_MAX = 256;

// f at a node (imate/functions/*.cpp; coefficients c as in slq_func)
__device__ __forceinline__ double apply_func(int func, double x, const double4& c)
{
    switch (func)
    {
        case 0: return log(x);
        case 1: return 1.0 / x;
        case 3: return exp(x * c.x);
        case 4: return (c.x * x + c.y) / (c.z * x + c.w);
        case 5: return (x < c.x || x > c.y) ? 0.0 : 1.0;
        case 6:
        {
            // 0.5 * M_SQRT1_2 * M_2_SQRTPI / sigma = 1 / (sigma sqrt(2 pi))
            const double u = (x - c.x) / c.y;
            return (0.5 * 0.70710678118654752440 * 1.12837916709551257390 / c.y) *
                   exp(-0.5 * u * u);
        }
        case 7: return 0.5 * (1.0 + tanh(c.x * x));
        default: return x;
    }
}

__device__ int ql_first_row(double* d, double* e, double* z, int k)
{
    for (int i = 0; i < k; ++i) z[i] = (i == 0) ? 1.0 : 0.0;
    if (k <= 1) return 0;
    e[k - 1] = 0.0;
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < k; ++l)
    {
        int iter = 0;
        for (;;)
        {
            int mm;
            for (mm = l; mm < k - 1; ++mm)
            {
                const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
                if (fabs(e[mm]) <= eps * dd) break;
            }
            if (mm == l) break;
            if (++iter > 60) return 1;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = mm - 1; i >= l; --i)
            {
                const double f = s * e[i];
                const double bb = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0)
                {
                    d[i + 1] -= p;
                    e[mm] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * bb;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - bb;
                const double zf = z[i + 1];
                z[i + 1] = s * z[i] + c * zf;
                z[i] = c * z[i] - s * zf;
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    return 0;
}

__global__ void __launch_bounds__(128)
k_eig_quad(int count, int b, int m, const double* __restrict__ alpha,
           const double* __restrict__ beta, const int32_t* __restrict__ size,
           int gram, int func, double4 fc, double exponent,
           const double* __restrict__ params, int q, double nscale,
           double* __restrict__ samples, double* __restrict__ theta_out,
           double* __restrict__ tau_out, int32_t* __restrict__ status)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    double d[EIG_MAX], e[EIG_MAX], z[EIG_MAX];
    const int k = size[p];
    bool bad = false;
    for (int i = 0; i < k; ++i)
    {
        const double a = alpha[static_cast<int64_t>(i) * b + p];
        const double bt = beta[static_cast<int64_t>(i) * b + p];
        if (!isfinite(a) || (i < k - 1 && !isfinite(bt))) bad = true;
        if (gram)
        {
            const double bp = (i > 0) ? beta[static_cast<int64_t>(i - 1) * b + p] : 0.0;
            d[i] = a * a + bp * bp;
            e[i] = (i < k - 1) ? a * bt : 0.0;
        }
        else
        {
            d[i] = a;
            e[i] = (i < k - 1) ? bt : 0.0;
        }
    }
    int st = ql_first_row(d, e, z, k);
    for (int i = 0; i < k; ++i)
        if (!isfinite(d[i]) || !isfinite(z[i])) bad = true;
    if (theta_out)
        for (int i = 0; i < k; ++i)
        {
            theta_out[static_cast<int64_t>(i) * b + p] = d[i];
            tau_out[static_cast<int64_t>(i) * b + p] = z[i];
        }
    const double t0 = (q > 0) ? params[0] : 0.0;
    bool node = false, nonfinite = false;
    for (int j = 0; j < q; ++j)
    {
        double acc = 0.0;
        for (int i = 0; i < k; ++i)
        {
            const double th = (j > 0) ? d[i] - t0 + params[j] : d[i];
            const double x = pow(th, exponent);
            // log of a non-positive node, 1/x of a zero node (weighted)
            if (z[i] != 0.0 && ((func == 0 && !(x > 0.0)) || (func == 1 && x == 0.0)))
                node = true;
            acc += z[i] * z[i] * apply_func(func, x, fc);
        }
        samples[static_cast<int64_t>(p) * q + j] = nscale * acc;
        if (!isfinite(nscale * acc)) nonfinite = true;
    }
    // bit mask: 1 non-finite coefficients or eigen-solve results, 2 QL did
    // not converge, 4 a non-positive node under log (zero node under 1/x),
    // 8 a non-finite sample
    status[p] = (bad ? 1 : 0) | (st ? 2 : 0) | (node ? 4 : 0) | (nonfinite ? 8 : 0);
}

// ---------------------------------------------------------------------------
// Rademacher probe generation into a [len][b] block.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t xoshiro_next_dev(uint64_t* s)
{
    const uint64_t x = s[1] * 5;
    const uint64_t result = ((x << 7) | (x >> 57)) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return result;
}

// Parity mode: probe p (0 <= p < count) is words [0, wpp) of the stream
// state starts[p]; block (x = probe tile, y = chunk) thread advances to word
// chunk*cw by the polynomial chunk_polys[chunk] (x^(chunk*cw) mod P) and
// draws cw words.  Bit j of word w gives element 64 w + j (+1 if set).
template <typename VT>
__global__ void __launch_bounds__(128)
k_probe_parity(int64_t len, int b, int count, int64_t wpp, int cw,
               const uint64_t* __restrict__ starts,
               const uint64_t* __restrict__ chunk_polys,
               const int32_t* __restrict__ inv, VT* __restrict__ X)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b) return;
    const int64_t w0 = static_cast<int64_t>(blockIdx.y) * cw;
    const int64_t w1 = min64(w0 + cw, wpp);
    if (p >= count)
    {
        for (int64_t idx = w0 * 64; idx < min64(w1 * 64, len); ++idx)
            X[static_cast<int64_t>(inv ? inv[idx] : idx) * b + p] = VT(0);
        return;
    }
    uint64_t s[4];
    for (int k = 0; k < 4; ++k) s[k] = starts[static_cast<int64_t>(p) * 4 + k];
    if (blockIdx.y > 0)
    {
        const uint64_t* q = chunk_polys + static_cast<int64_t>(blockIdx.y) * 4;
        uint64_t acc[4] = {0, 0, 0, 0};
        for (int i = 0; i < 256; ++i)
        {
            if ((q[i >> 6] >> (i & 63)) & 1ULL)
                for (int k = 0; k < 4; ++k) acc[k] ^= s[k];
            xoshiro_next_dev(s);
        }
        for (int k = 0; k < 4; ++k) s[k] = acc[k];
    }
    for (int64_t w = w0; w < w1; ++w)
    {
        const uint64_t bits = xoshiro_next_dev(s);
        const int64_t e0 = w * 64;
        const int ne = static_cast<int>(min64(64, len - e0));
        for (int j = 0; j < ne; ++j)
        {
            const int64_t row = inv ? inv[e0 + j] : e0 + j;
            X[row * b + p] = ((bits >> j) & 1ULL) ? VT(1) : VT(-1);
        }
    }
}

// Fast mode: word w of probe g is a SplitMix64 finaliser of a counter built
// from (seed, g, w); no sequential state, no host set-up.
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

template <typename VT>
__global__ void __launch_bounds__(128)
k_probe_fast(int64_t len, int b, int count, int64_t first, uint64_t key,
             int64_t wpp, int cw, const int32_t* __restrict__ inv,
             VT* __restrict__ X)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b) return;
    const int64_t w0 = static_cast<int64_t>(blockIdx.y) * cw;
    const int64_t w1 = min64(w0 + cw, wpp);
    const uint64_t g = static_cast<uint64_t>(first + p);
    for (int64_t w = w0; w < w1; ++w)
    {
        const uint64_t bits =
            mix64(key + 0x9e3779b97f4a7c15ULL * (g * 0x100000001b3ULL + static_cast<uint64_t>(w) + 1));
        const int64_t e0 = w * 64;
        const int ne = static_cast<int>(min64(64, len - e0));
        for (int j = 0; j < ne; ++j)
        {
            const int64_t row = inv ? inv[e0 + j] : e0 + j;
            X[row * b + p] = (p >= count) ? VT(0)
                             : (((bits >> j) & 1ULL) ? VT(1) : VT(-1));
        }
    }
}

// ---------------------------------------------------------------------------
// Operator set-up helpers
// ---------------------------------------------------------------------------

// flag |= 1: indptr[0] != 0 or indptr[rows] != nnz; 2: decreasing indptr;
// 4: column index out of range
__global__ void k_check_csr(const int32_t* __restrict__ indptr,
                            const int32_t* __restrict__ indices, int64_t rows,
                            int64_t cols, int64_t nnz, int32_t* flag)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    if (i == 0 && (indptr[0] != 0 || indptr[rows] != nnz)) atomicOr(flag, 1);
    for (int64_t r = i; r < rows; r += stride)
        if (indptr[r + 1] < indptr[r]) atomicOr(flag, 2);
    for (int64_t k = i; k < nnz; k += stride)
    {
        const int32_t c = indices[k];
        if (c < 0 || c >= cols) atomicOr(flag, 4);
    }
}

__global__ void k_row_ids(const int32_t* __restrict__ indptr, int64_t rows,
                          int32_t* __restrict__ row_of)
{
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
    const int lane = threadIdx.x & 31;
    for (int64_t r = r0; r < rows; r += stride)
        for (int k = indptr[r] + lane; k < indptr[r + 1]; k += 32) row_of[k] = static_cast<int32_t>(r);
}

__global__ void k_iota(int32_t* __restrict__ a, int64_t n)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        a[i] = static_cast<int32_t>(i);
}

template <typename VT>
__global__ void k_gather_transpose(const int32_t* __restrict__ perm,
                                   const int32_t* __restrict__ row_of,
                                   const VT* __restrict__ data, int64_t nnz,
                                   int32_t* __restrict__ t_indices,
                                   VT* __restrict__ t_data)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < nnz; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int32_t k = perm[i];
        t_indices[i] = row_of[k];
        t_data[i] = data[k];
    }
}

// t_indptr[c] = first position of key >= c in the sorted column keys
__global__ void k_bounds(const int32_t* __restrict__ sorted_keys, int64_t nnz,
                         int64_t ncols, int32_t* __restrict__ t_indptr)
{
    const int64_t c0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t c = c0; c <= ncols; c += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        int64_t lo = 0, hi = nnz;
        while (lo < hi)
        {
            const int64_t mid = (lo + hi) >> 1;
            if (sorted_keys[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        t_indptr[c] = static_cast<int32_t>(lo);
    }
}

// Symmetric permutation B = P A P^T of a square CSR matrix: inverse map,
// 64-bit (new row, new column) sort keys, gather of the sorted entries and
// row pointers from the sorted keys.
__global__ void k_inverse_perm(const int32_t* __restrict__ perm, int64_t n,
                               int32_t* __restrict__ inv)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        inv[perm[i]] = static_cast<int32_t>(i);
}

__global__ void k_perm_keys(const int32_t* __restrict__ indptr,
                            const int32_t* __restrict__ indices,
                            const int32_t* __restrict__ inv, int64_t rows,
                            uint64_t* __restrict__ keys, int32_t* __restrict__ pos)
{
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
    const int lane = threadIdx.x & 31;
    for (int64_t r = r0; r < rows; r += stride)
    {
        const uint64_t hi = static_cast<uint64_t>(static_cast<uint32_t>(inv[r])) << 32;
        for (int k = indptr[r] + lane; k < indptr[r + 1]; k += 32)
        {
            keys[k] = hi | static_cast<uint32_t>(inv[indices[k]]);
            pos[k] = k;
        }
    }
}

// deg[i] = row length of A's row perm[i] (deg[n] = 0, for the exclusive
// scan into B's row pointer); *maxdeg = the largest
__global__ void k_perm_deg(const int32_t* __restrict__ indptr, const int32_t* __restrict__ perm,
                           int64_t n, int32_t* __restrict__ deg, int32_t* __restrict__ maxdeg)
{
    int32_t m = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        int32_t d = 0;
        if (i < n)
        {
            const int32_t r = perm[i];
            d = indptr[r + 1] - indptr[r];
        }
        deg[i] = d;
        m = max(m, d);
    }
    atomicMax(maxdeg, m);
}

// Rows of B = P A P^T, one warp per row i of B (A's row perm[i], at most
// PERM_ROW_MAX entries): the entries relabelled (column inv[c]) and sorted by
// (new column, position in the row) with a bitonic network held in the
// warp's registers -- the order a stable sort of (row, column) keys gives,
// so B is the same bit for bit.  Key t of the row sits in lane t % 32,
// register t / 32: exchanges across lanes are shuffles, those across
// registers stay in the lane, and the loads and stores are coalesced.  Each
// row runs the smallest network (32, 64, ..., 1024 keys) that holds it.
constexpr int PERM_ROW_MAX = 1024;
constexpr int PERM_WARPS = 8;

// Bitonic sort of the warp's 32 * KPL keys into increasing order.
template <int KPL>
__device__ __forceinline__ void warp_bitonic(uint64_t (&a)[KPL], int lane)
{
    constexpr int M = 32 * KPL;
#pragma unroll
    for (int k = 2; k <= M; k <<= 1)
    {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            if (j >= 32)
            {
                const int jr = j >> 5;
#pragma unroll
                for (int r = 0; r < KPL; ++r)
                {
                    if (r & jr) continue;
                    const bool up = ((((r << 5) | lane) & k) == 0);
                    const uint64_t x = a[r], y = a[r | jr];
                    const bool sw = (x > y) == up;
                    a[r] = sw ? y : x;
                    a[r | jr] = sw ? x : y;
                }
            }
            else
            {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int r = 0; r < KPL; ++r)
                {
                    const uint64_t y = __shfl_xor_sync(0xffffffffu, a[r], j);
                    const bool up = ((((r << 5) | lane) & k) == 0);
                    const uint64_t lo = a[r] < y ? a[r] : y;
                    const uint64_t hi = a[r] < y ? y : a[r];
                    a[r] = (up == lower) ? lo : hi;
                }
            }
        }
    }
}

template <typename VT, int KPL>
__device__ __forceinline__ void perm_row(const int32_t* __restrict__ indices,
                                         const VT* __restrict__ data,
                                         const int32_t* __restrict__ inv, int32_t e0, int len,
                                         int64_t o, int lane, int32_t* __restrict__ p_ind,
                                         VT* __restrict__ p_data)
{
    uint64_t a[KPL];
#pragma unroll
    for (int r = 0; r < KPL; ++r)
    {
        const int t = (r << 5) | lane;
        a[r] = t < len ? (static_cast<uint64_t>(static_cast<uint32_t>(inv[indices[e0 + t]])) << 32) |
                             static_cast<uint32_t>(t)
                       : ~uint64_t(0);
    }
    warp_bitonic<KPL>(a, lane);
#pragma unroll
    for (int r = 0; r < KPL; ++r)
    {
        const int t = (r << 5) | lane;
        if (t < len)
        {
            p_ind[o + t] = static_cast<int32_t>(a[r] >> 32);
            p_data[o + t] = data[e0 + static_cast<int32_t>(a[r] & 0xffffffffu)];
        }
    }
}

template <typename VT>
__global__ void __launch_bounds__(PERM_WARPS * 32)
    k_perm_rows(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                const VT* __restrict__ data, const int32_t* __restrict__ perm,
                const int32_t* __restrict__ inv, const int32_t* __restrict__ p_ptr, int64_t n,
                int32_t* __restrict__ p_ind, VT* __restrict__ p_data)
{
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * PERM_WARPS + w; i < n;
         i += static_cast<int64_t>(gridDim.x) * PERM_WARPS)
    {
        const int32_t r = perm[i];
        const int32_t e0 = indptr[r];
        const int len = indptr[r + 1] - e0;
        const int64_t o = p_ptr[i];
        // len is the same in every lane: the branch is warp-uniform
        if (len <= 0) continue;
        if (len <= 32) perm_row<VT, 1>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
        else if (len <= 64) perm_row<VT, 2>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
        else if (len <= 128) perm_row<VT, 4>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
        else if (len <= 256) perm_row<VT, 8>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
        else if (len <= 512) perm_row<VT, 16>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
        else if (len <= PERM_ROW_MAX)
            perm_row<VT, 32>(indices, data, inv, e0, len, o, lane, p_ind, p_data);
    }
}

template <typename VT>
__global__ void k_perm_gather(const uint64_t* __restrict__ sorted_keys,
                              const int32_t* __restrict__ sorted_pos,
                              const VT* __restrict__ data, int64_t nnz,
                              int32_t* __restrict__ p_ind, VT* __restrict__ p_data)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < nnz; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        p_ind[i] = static_cast<int32_t>(sorted_keys[i] & 0xffffffffULL);
        p_data[i] = data[sorted_pos[i]];
    }
}

__global__ void k_bounds64(const uint64_t* __restrict__ sorted_keys, int64_t nnz,
                           int64_t rows, int32_t* __restrict__ p_ptr)
{
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t r = r0; r <= rows; r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const uint64_t key = static_cast<uint64_t>(r) << 32;
        int64_t lo = 0, hi = nnz;
        while (lo < hi)
        {
            const int64_t mid = (lo + hi) >> 1;
            if (sorted_keys[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        p_ptr[r] = static_cast<int32_t>(lo);
    }
}

// ---------------------------------------------------------------------------
// Cuthill-McKee order on the device, one breadth-first level per round.
//
// The serial order appends the not-yet-visited neighbours of each visited
// row, sorted by (degree, row), in visit order; so a row of the next level
// belongs to the earliest-visited row of the current level that lists it,
// and the next level is its rows sorted by (that parent's position, degree,
// row).  k_rcm_claim takes the parent as an atomic minimum of positions,
// k_rcm_collect lists each claimed row once (packed key: parent offset,
// degree, row), a radix sort orders the keys, k_rcm_assign places them.
// pos[r] < 0 marks an unvisited row; claim[r] holds INT_MAX until claimed.
// ---------------------------------------------------------------------------

__global__ void k_rcm_init(const int32_t* __restrict__ indptr, int64_t n,
                           int32_t* __restrict__ degree, int32_t* __restrict__ rows,
                           int32_t* __restrict__ pos, int32_t* __restrict__ claim,
                           int32_t* __restrict__ maxdeg)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    int32_t m = 0;
    for (int64_t r = i0; r < n; r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int32_t d = indptr[r + 1] - indptr[r];
        degree[r] = d;
        rows[r] = static_cast<int32_t>(r);
        pos[r] = -1;
        claim[r] = INT_MAX;
        m = max(m, d);
    }
    atomicMax(maxdeg, m);
}

// *result = the first index i >= from of by_degree whose row is unvisited
// (n if none; *result must hold n before the launch)
__global__ void k_rcm_first(const int32_t* __restrict__ by_degree,
                            const int32_t* __restrict__ pos, int64_t from, int64_t n,
                            int32_t* __restrict__ result)
{
    const int64_t i0 = from + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (pos[by_degree[i]] < 0)
        {
            atomicMin(result, static_cast<int32_t>(i));
            return;
        }
}

// the row at by_degree[*result] starts a component at position cnt
__global__ void k_rcm_start(const int32_t* __restrict__ by_degree,
                            const int32_t* __restrict__ result, int32_t* __restrict__ pos,
                            int32_t* __restrict__ out, int64_t cnt, int64_t n)
{
    if (*result < 0 || *result >= n || cnt >= n) return;  // host reports it
    const int32_t r = by_degree[*result];
    pos[r] = static_cast<int32_t>(cnt);
    out[cnt] = r;
}

// warp per frontier row k in [lb, le): claim[c] = min(claim[c], k) for its
// unvisited neighbours c; also clears the level's row count
__global__ void k_rcm_claim(const int32_t* __restrict__ out, int64_t lb, int64_t le,
                            const int32_t* __restrict__ indptr,
                            const int32_t* __restrict__ indices,
                            const int32_t* __restrict__ pos, int32_t* __restrict__ claim,
                            int32_t* __restrict__ count)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = 0;
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t k = lb + w0; k < le; k += ws)
    {
        const int32_t r = out[k];
        const int32_t e1 = indptr[r + 1];
        for (int32_t e = indptr[r] + lane; e < e1; e += 32)
        {
            const int32_t c = indices[e];
            if (pos[c] < 0) atomicMin(&claim[c], static_cast<int32_t>(k));
        }
    }
}

// warp per frontier row k: each unvisited neighbour whose claim is k is
// listed once, key = (k - lb) << (db + nb) | degree << nb | row
__global__ void k_rcm_collect(const int32_t* __restrict__ out, int64_t lb, int64_t le,
                              const int32_t* __restrict__ indptr,
                              const int32_t* __restrict__ indices,
                              const int32_t* __restrict__ pos,
                              const int32_t* __restrict__ degree, int32_t* __restrict__ claim,
                              int nb, int db, uint64_t* __restrict__ keys,
                              int32_t* __restrict__ count)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t k = lb + w0; k < le; k += ws)
    {
        const int32_t r = out[k];
        const int32_t kk = static_cast<int32_t>(k);
        const int32_t e1 = indptr[r + 1];
        for (int32_t e = indptr[r] + lane; e < e1; e += 32)
        {
            const int32_t c = indices[e];
            if (pos[c] >= 0 || claim[c] != kk) continue;
            // once per row, also when r lists c twice
            if (atomicCAS(&claim[c], kk, -1) != kk) continue;
            const int32_t i = atomicAdd(count, 1);
            keys[i] = (static_cast<uint64_t>(k - lb) << (db + nb)) |
                      (static_cast<uint64_t>(degree[c]) << nb) | static_cast<uint64_t>(c);
        }
    }
}

// sorted keys -> positions cnt .. cnt + m - 1
__global__ void k_rcm_assign(const uint64_t* __restrict__ keys, int64_t m, uint64_t rowmask,
                             int64_t cnt, int32_t* __restrict__ out, int32_t* __restrict__ pos)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < m; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int32_t c = static_cast<int32_t>(keys[i] & rowmask);
        out[cnt + i] = c;
        pos[c] = static_cast<int32_t>(cnt + i);
    }
}

__global__ void k_rcm_reverse(const int32_t* __restrict__ out, int64_t n,
                              int32_t* __restrict__ order)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t k = i0; k < n; k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        order[k] = out[n - 1 - k];
}

// ---------------------------------------------------------------------------
// Cuthill-McKee order in one cooperative launch: the same levels, parents
// and (degree, row) order as the round-per-level kernels above, with every
// level done inside the kernel between grid barriers instead of by host
// rounds (a memcpy, a synchronisation and a radix sort per level).  Per
// level:
//   A  claim: claim[c] = min(claim[c], k) over the unvisited neighbours c of
//      every frontier row k (as k_rcm_claim);
//   B  count: each claimed neighbour is taken once by its parent k
//      (claim k -> -2 - k) and counted, counts[k - lb];
//   C  block 0 scans the counts into offsets, sets the next level
//      [le, le + m) -- or, when the level has no children, starts the next
//      component at the first unvisited row of the (degree, row) order;
//   D  each parent lists its children again (claim -2 - k -> INT_MIN), ranks
//      them by (degree, row) inside its warp and places them at
//      le + offset + rank.
// A warp lists at most `cap` children (cap >= the largest row degree, which
// the host checks).  The grid barrier is a counter and a generation word
// whose waits give up after `spin_limit` clock cycles (error bit 16), so the
// kernel always ends.
// ---------------------------------------------------------------------------

struct RcmCoopState {
    int64_t lb, le, cnt, cursor;
    int32_t components, done;
    uint32_t bar_count, bar_gen;
};

__device__ __forceinline__ int32_t ldcg_i32(const int32_t* p) { return __ldcg(p); }

// the error word as one value for the whole block (thread 0 reads it)
__device__ __forceinline__ int32_t rcm_block_err(const int32_t* err, int32_t* slot)
{
    __syncthreads();
    if (threadIdx.x == 0) *slot = *reinterpret_cast<const volatile int32_t*>(err);
    __syncthreads();
    return *slot;
}

__device__ __forceinline__ void rcm_grid_sync(RcmCoopState* st, int32_t* err,
                                              long long spin_limit)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile uint32_t* gen = &st->bar_gen;
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1)
        {
            atomicExch(&st->bar_count, 0u);
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        }
        else
        {
            const long long t0 = clock64();
            while (*gen == g)
            {
                if (clock64() - t0 > spin_limit)
                {
                    atomicOr(err, 16);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// block-wide exclusive scan of a[0 .. len) in place (block 0 only); returns
// the total to every thread of the block
__device__ int64_t rcm_block_scan(int32_t* a, int64_t len, int32_t* warp_sums)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int64_t carry = 0;
    for (int64_t base = 0; base < len; base += blockDim.x)
    {
        const int64_t i = base + threadIdx.x;
        const int32_t v = i < len ? ldcg_i32(a + i) : 0;
        int32_t x = v;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0)
        {
            int32_t s = lane < nw ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1)
            {
                const int32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            if (lane < nw) warp_sums[lane] = s;  // inclusive warp prefix
        }
        __syncthreads();
        const int32_t before = (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
        if (i < len) a[i] = static_cast<int32_t>(carry + before);
        carry += warp_sums[nw - 1];
        __syncthreads();
    }
    return carry;
}

// block 0: the first unvisited row of by_degree at or after the cursor
// starts a component at position cnt
__device__ void rcm_start_component(RcmCoopState* st, const int32_t* __restrict__ by_degree,
                                    int32_t* __restrict__ pos, int32_t* __restrict__ out,
                                    int64_t n, int max_components, int32_t* err, int32_t* sh)
{
    if (threadIdx.x == 0) sh[0] = INT_MAX;
    __syncthreads();
    int64_t cursor = st->cursor;
    for (;;)
    {
        const int64_t i = cursor + threadIdx.x;
        if (i < n && ldcg_i32(pos + by_degree[i]) < 0) atomicMin(sh, static_cast<int32_t>(i));
        __syncthreads();
        const int32_t found = sh[0];
        if (found != INT_MAX || cursor + blockDim.x >= n) break;
        cursor += blockDim.x;
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        const int32_t found = sh[0];
        if (found == INT_MAX || st->cnt >= n)
            atomicOr(err, 32);  // lost track of the unvisited rows
        else if (st->components + 1 > max_components)
            atomicOr(err, 64);  // more components than asked for
        else
        {
            const int32_t r = by_degree[found];
            pos[r] = static_cast<int32_t>(st->cnt);
            out[st->cnt] = r;
            st->cursor = found + 1;
            st->lb = st->cnt;
            st->le = st->cnt + 1;
            st->cnt += 1;
            st->components += 1;
        }
        __threadfence();
    }
    __syncthreads();
}

__global__ void __launch_bounds__(512, 1)
    k_rcm_coop(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
               const int32_t* __restrict__ degree, const int32_t* __restrict__ by_degree,
               int64_t n, int max_components, int cap, int32_t* __restrict__ pos,
               int32_t* __restrict__ claim, int32_t* __restrict__ out,
               int32_t* __restrict__ counts, RcmCoopState* st, int32_t* err,
               long long spin_limit)
{
    extern __shared__ uint64_t rcm_sh[];
    __shared__ int32_t small[40];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    uint64_t* buf = rcm_sh + static_cast<int64_t>(wid) * cap;
    const int64_t gw = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + wid;
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);

    if (blockIdx.x == 0) rcm_start_component(st, by_degree, pos, out, n, max_components, err, small);
    rcm_grid_sync(st, err, spin_limit);
    for (;;)
    {
        if (rcm_block_err(err, small + 32) != 0) return;
        const int64_t lb = *reinterpret_cast<volatile int64_t*>(&st->lb);
        const int64_t le = *reinterpret_cast<volatile int64_t*>(&st->le);
        if (*reinterpret_cast<volatile int32_t*>(&st->done)) return;

        // A: claims
        for (int64_t k = lb + gw; k < le; k += nwarps)
        {
            const int32_t r = ldcg_i32(out + k);
            const int32_t e1 = __ldg(indptr + r + 1);
            for (int32_t e = __ldg(indptr + r) + lane; e < e1; e += 32)
            {
                const int32_t c = __ldg(indices + e);
                if (ldcg_i32(pos + c) < 0) atomicMin(claim + c, static_cast<int32_t>(k));
            }
        }
        rcm_grid_sync(st, err, spin_limit);
        // B: each child taken once by its parent, counted
        for (int64_t k = lb + gw; k < le; k += nwarps)
        {
            const int32_t r = ldcg_i32(out + k);
            const int32_t kk = static_cast<int32_t>(k);
            const int32_t e1 = __ldg(indptr + r + 1);
            int32_t m = 0;
            for (int32_t e = __ldg(indptr + r) + lane; e < e1; e += 32)
            {
                const int32_t c = __ldg(indices + e);
                if (ldcg_i32(claim + c) == kk && atomicCAS(claim + c, kk, -2 - kk) == kk) ++m;
            }
            for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
            if (lane == 0)
            {
                if (m > cap) atomicOr(err, 128);
                counts[k - lb] = m;
            }
        }
        rcm_grid_sync(st, err, spin_limit);
        // C: offsets and the next level (block 0)
        if (blockIdx.x == 0 && rcm_block_err(err, small + 32) == 0)
        {
            const int64_t m = rcm_block_scan(counts, le - lb, small);
            if (threadIdx.x == 0)
            {
                st->lb = le;
                st->le = le + m;
                st->cnt = le + m;
                if (m == 0 && st->cnt >= n) st->done = 1;
                __threadfence();
            }
            __syncthreads();
            if (m == 0 && le < n)
                rcm_start_component(st, by_degree, pos, out, n, max_components, err, small);
        }
        rcm_grid_sync(st, err, spin_limit);
        if (rcm_block_err(err, small + 32) != 0) return;
        // D: children placed at le + offset + rank of (degree, row)
        for (int64_t k = lb + gw; k < le; k += nwarps)
        {
            const int32_t r = ldcg_i32(out + k);
            const int32_t mark = -2 - static_cast<int32_t>(k);
            const int32_t e0 = __ldg(indptr + r), e1 = __ldg(indptr + r + 1);
            int count = 0;
            for (int32_t eb = e0; eb < e1; eb += 32)
            {
                const int32_t e = eb + lane;
                bool take = false;
                int32_t c = 0;
                if (e < e1)
                {
                    c = __ldg(indices + e);
                    take = ldcg_i32(claim + c) == mark && atomicCAS(claim + c, mark, INT_MIN) == mark;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, take);
                if (take)
                {
                    const int slot = count + __popc(bal & ((1u << lane) - 1u));
                    if (slot < cap)
                        buf[slot] = (static_cast<uint64_t>(__ldg(degree + c)) << 32) |
                                    static_cast<uint32_t>(c);
                }
                count += __popc(bal);
            }
            __syncwarp();
            if (count > cap)
            {
                if (lane == 0) atomicOr(err, 128);
                continue;
            }
            const int64_t base = le + ldcg_i32(counts + (k - lb));
            for (int i = lane; i < count; i += 32)
            {
                const uint64_t key = buf[i];
                int rank = 0;
                for (int j = 0; j < count; ++j) rank += buf[j] < key ? 1 : 0;
                const int32_t c = static_cast<int32_t>(key & 0xffffffffu);
                out[base + rank] = c;
                pos[c] = static_cast<int32_t>(base + rank);
            }
            __syncwarp();
        }
        rcm_grid_sync(st, err, spin_limit);
    }
}

__global__ void k_fill_f64(double* __restrict__ a, int64_t n, double v)
{
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x) a[i] = v;
}

__global__ void k_init_block(int count, int b, int m, double s0,
                             double* __restrict__ scale0,
                             int32_t* __restrict__ active,
                             int32_t* __restrict__ size)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b) return;
    const bool real = p < count;
    scale0[p] = real ? s0 : 0.0;
    active[p] = real ? 1 : 0;
    size[p] = m;
}


// ===========================================================================
// TMA-streamed reorthogonalisation passes (sm_100a).
//
// One CTA per SM: a producer warp moves tiles of T rows x PT probes of every
// vector the pass reads into a ring of S shared-memory stages with
// cp.async.bulk (completion counted on an mbarrier per stage); eight
// consumer warps compute from the stages and release them through a second
// mbarrier per stage.  The copy engine keeps S x 16 KB in flight per SM, so
// the pass streams at HBM rate without registers spent on loads in flight.
//
// Work per row tile, in item order:
//   dots   : W [, v_j, v_{j-1} (three-term update; written to Wout)],
//            then the basis vectors last-i (skipping v_j, v_{j-1}, whose
//            products come from the update registers) -> FP64 partials of
//            <v_i, w> per (i, probe);
//   reorth : Win, then the basis vectors last-i: w -= c_i v_i, written to
//            Wout, FP64 partials of |w|^2.
// Rows past the last whole tile are done by the last CTA with plain loads.
//
// Every mbarrier wait is bounded; a wait that runs out sets *error and the
// CTA skips the remaining work (it still waits, bounded, for the copies it
// issued before it leaves).
// ===========================================================================

constexpr int STREAM_CONSUMERS = 256;            // 8 consumer warps
constexpr int STREAM_THREADS = STREAM_CONSUMERS + 32;
constexpr int STREAM_TILE_BYTES = 16384;
constexpr int STREAM_MAX_STAGES = 8;
constexpr long long STREAM_SPIN_LIMIT = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false if the phase did not complete within the limit or
// another thread of the CTA gave up (abort flag)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          const int* abort_flag)
{
    for (long long i = 0; i < STREAM_SPIN_LIMIT; ++i)
    {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023) == 1023 && *reinterpret_cast<const volatile int*>(abort_flag))
            return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// The same copy with an L2 eviction policy (a createpolicy value) on the
// lines it reads.
__device__ __forceinline__ void bulk_copy_g2s_hint(void* dst, const void* src, uint32_t bytes,
                                                   uint64_t* bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// L2 policy: lines read once go first when L2 needs room
__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// The exponent e_p that scales a probe of norm 1 / s into FP16 range for
// the block SpMM (every scaled |x| <= 2^14); 0 without a usable scale.
__device__ __forceinline__ int x16_exp(double s)
{
    return (s > 0.0 && isfinite(s)) ? min(max(ilogb(s) + 13, -120), 120) : 0;
}

// hi = rn_f16(v), lo = rn_f16(v - hi) of one scaled element of the split
// block X16[row] = hi[b] | lo[b]
__device__ __forceinline__ void x16_store(__half* x16, int64_t row, int b, int p, float v)
{
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    x16[row * 2 * b + p] = h;
    x16[row * 2 * b + b + p] = l;
}

template <typename VT>
struct StreamArgs {
    int64_t n;            // rows
    int b;                // block width (row stride)
    int PT;               // probes per CTA tile (grid.y = b / PT)
    int T;                // rows per tile
    int S;                // stages
    int J;                // basis vectors (last, last-1, ...)
    int bs;               // ring slots
    int last;             // newest basis vector index
    int64_t slot_elems;   // stride between ring slots (elements)
    const VT* W;          // dots: input w (pre-update); reorth: input w
    VT* Wout;             // updated / reorthogonalised w
    int do_update;        // dots: three-term update first
    const VT* Vj;
    const double* sj;
    const double* aj;
    const VT* Vm;
    const double* sm;
    const double* bm;
    const VT* basis;
    const VT* coef;       // reorth: [J][b] coefficients c_i = h_i s_i
    int want_norm;
    double* partials;     // dots: [grid.x][J][b]; reorth: [grid.x][b]
    int32_t* error;       // set to 1 when a wait runs out
    int fail_first_wait;  // test hook: the consumers' first wait runs out at once
    // the block SpMM's split probe block, written by the pass that writes the
    // next Krylov vector (float only): dots with do_update write the partial
    // sums of |w|^2 of the updated w, [grid.x][b] (wn2_out); the last reorth
    // pass reduces them (wn2_in, wn2_grid rows), takes 2^e_p with e_p from
    // that norm (an upper bound of the final one, so every scaled element
    // fits), and writes x16[row] = hi | lo of 2^e_p w and x16exp[p] = e_p
    double* wn2_out;
    const double* wn2_in;
    int wn2_grid;
    __half* x16;
    int32_t* x16exp;
};

// MODE 0: dots, MODE 1: reorth.  R = rows per consumer thread per tile.
template <typename VT, int MODE, int R>
__global__ void __launch_bounds__(STREAM_THREADS, 1) k_stream(const StreamArgs<VT> a)
{
    // shared memory: barriers (256 B) | norm partials (256 doubles) |
    // S stages of 16 KB | dots: acc[J][256] doubles, reorth: coef[J][PT]
    extern __shared__ __align__(128) unsigned char smem_stream[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_stream);
    uint64_t* empty = full + STREAM_MAX_STAGES;
    int* abort_flag = reinterpret_cast<int*>(empty + STREAM_MAX_STAGES);
    double* red = reinterpret_cast<double*>(smem_stream + 256);
    VT* stages = reinterpret_cast<VT*>(smem_stream + 256 + STREAM_CONSUMERS * 8);
    const int tile_elems = a.T * a.PT;
    double* extra = reinterpret_cast<double*>(smem_stream + 256 + STREAM_CONSUMERS * 8 +
                                              static_cast<size_t>(a.S) * STREAM_TILE_BYTES);

    const int tid = threadIdx.x;
    const bool producer = tid >= STREAM_CONSUMERS;
    const int PT = a.PT;
    const int RSTEP = STREAM_CONSUMERS / PT;
    const int pl = tid % PT;
    const int roff = tid / PT;
    const int p0 = blockIdx.y * PT;
    const int b = a.b;
    const int J = a.J;

    // items per tile
    const bool upd = a.do_update != 0;
    const int npre = 1 + (upd ? (a.Vm ? 2 : 1) : 0);
    // dots: basis vectors v_j, v_{j-1} are served from the update registers
    const int skip = (MODE == 0 && upd) ? (a.Vm ? 2 : 1) : 0;
    const int nbasis = (J > skip) ? J - skip : 0;
    const int nitems = npre + nbasis;

    if (tid == 0)
    {
        for (int s = 0; s < a.S; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], STREAM_CONSUMERS / 32);
        }
        abort_flag[0] = 0;
        abort_flag[1] = 0;  // stays 0: bounded waits on the way out
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (MODE == 0)
    {
        for (int i = tid; i < J * STREAM_CONSUMERS; i += STREAM_THREADS) extra[i] = 0.0;
    }
    else
    {
        for (int i = tid; i < J * PT; i += STREAM_THREADS)
            extra[i] = static_cast<double>(a.coef[static_cast<int64_t>(i / PT) * b + p0 + i % PT]);
    }
    __syncthreads();

    const int64_t ntiles = a.n / a.T;
    const bool contiguous = (PT == b);
    const uint32_t tile_bytes = static_cast<uint32_t>(tile_elems * sizeof(VT));
    auto item_ptr = [&](int item) -> const VT* {
        if (item == 0) return a.W;
        if (upd && item == 1) return a.Vj;
        if (upd && item == 2 && a.Vm) return a.Vm;
        const int i = skip + (item - npre);
        return a.basis + static_cast<int64_t>(ring_slot(a.last - i, a.bs)) * a.slot_elems;
    };

    if (producer)
    {
        if ((tid & 31) == 0)
        {
            int s = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            bool ok = true;
            for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x)
            {
                const int64_t row0 = tile * a.T;
                for (int item = 0; item < nitems; ++item)
                {
                    if (*reinterpret_cast<volatile int*>(abort_flag)) { ok = false; break; }
                    if (!mbar_wait(&empty[s], phase ^ 1, abort_flag))
                    {
                        *abort_flag = 1;
                        atomicExch(a.error, 1);
                        ok = false;
                        break;
                    }
                    VT* dst = stages + static_cast<size_t>(s) * (STREAM_TILE_BYTES / sizeof(VT));
                    const VT* src = item_ptr(item) + row0 * b + p0;
                    mbar_expect_tx(&full[s], tile_bytes);
                    if (contiguous)
                    {
                        bulk_copy_g2s(dst, src, tile_bytes, &full[s]);
                    }
                    else
                    {
                        const uint32_t rb = static_cast<uint32_t>(PT * sizeof(VT));
                        for (int r = 0; r < a.T; ++r)
                            bulk_copy_g2s(dst + r * PT, src + static_cast<int64_t>(r) * b, rb,
                                          &full[s]);
                    }
                    ++issued;
                    if (++s == a.S) { s = 0; phase ^= 1; }
                }
            }
            if (!ok)
            {
                // let the copies already issued land before the CTA leaves
                int s2 = 0;
                uint32_t ph2 = 0;
                for (int64_t k = 0; k < issued; ++k)
                {
                    if (k + a.S >= issued) mbar_wait(&full[s2], ph2, abort_flag + 1);
                    if (++s2 == a.S) { s2 = 0; ph2 ^= 1; }
                }
            }
        }
    }
    else
    {
        int s = 0;
        uint32_t phase = 0;
        double cj = 0.0, cm = 0.0;
        if (upd)
        {
            cj = a.aj[p0 + pl] * a.sj[p0 + pl];
            cm = a.Vm ? a.bm[p0 + pl] * a.sm[p0 + pl] : 0.0;
        }
        double nacc = 0.0;
        bool ok = true;
        // the split probe block (MODE 1 with x16): this probe's 2^e_p from
        // the reduced |w|^2 partials of the dots pass (a fixed order)
        bool x16_on = false;
        float x16_scale = 1.0f;
        if constexpr (MODE == 1 && sizeof(VT) == 4)
        {
            if (a.x16 && a.wn2_in)
            {
                double n2 = 0.0;
                for (int g = 0; g < a.wn2_grid; ++g)
                    n2 += a.wn2_in[static_cast<int64_t>(g) * b + p0 + pl];
                const int e = (n2 > 0.0 && isfinite(n2)) ? x16_exp(1.0 / sqrt(n2)) : 0;
                x16_scale = ldexpf(1.0f, e);
                x16_on = true;
                if (roff == 0 && blockIdx.x == 0) a.x16exp[p0 + pl] = e;
            }
        }
        const int lane = tid & 31;
        auto release = [&](int st) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
        };
        for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x)
        {
            const int64_t row0 = tile * a.T;
            // 9 warps put 3 on one scheduler: at most 168 registers/thread
            double w[R], vj[R];
            for (int item = 0; item < nitems; ++item)
            {
                if (*reinterpret_cast<volatile int*>(abort_flag)) { ok = false; break; }
                if (MODE == 0 && item >= npre && item + 1 < nitems)
                {
                    // dots: two basis tiles per turn, four FMA chains each, so
                    // the two load -> convert -> FMA -> add-tree chains overlap
                    // (two warps per scheduler leave little else to hide them)
                    const int ib = skip + (item - npre);
                    const double prev0 = extra[ib * STREAM_CONSUMERS + tid];
                    const double prev1 = extra[(ib + 1) * STREAM_CONSUMERS + tid];
                    int s1 = s + 1;
                    uint32_t ph1 = phase;
                    if (s1 == a.S) { s1 = 0; ph1 ^= 1; }
                    if (!mbar_wait(&full[s], phase, abort_flag) ||
                        !mbar_wait(&full[s1], ph1, abort_flag))
                    {
                        *abort_flag = 1;
                        atomicExch(a.error, 1);
                        ok = false;
                        break;
                    }
                    const VT* t0 = stages + static_cast<size_t>(s) * (STREAM_TILE_BYTES / sizeof(VT));
                    const VT* t1 = stages + static_cast<size_t>(s1) * (STREAM_TILE_BYTES / sizeof(VT));
                    double l0[4] = {0.0, 0.0, 0.0, 0.0}, l1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                    for (int k = 0; k < R; ++k)
                    {
                        const int e = (roff + k * RSTEP) * PT + pl;
                        l0[k & 3] += static_cast<double>(t0[e]) * w[k];
                        l1[k & 3] += static_cast<double>(t1[e]) * w[k];
                    }
                    extra[ib * STREAM_CONSUMERS + tid] = prev0 + ((l0[0] + l0[1]) + (l0[2] + l0[3]));
                    extra[(ib + 1) * STREAM_CONSUMERS + tid] =
                        prev1 + ((l1[0] + l1[1]) + (l1[2] + l1[3]));
                    release(s);
                    release(s1);
                    s = s1 + 1;
                    phase = ph1;
                    if (s == a.S) { s = 0; phase ^= 1; }
                    ++item;
                    continue;
                }
                // dots: fetch this thread's running sum before the wait so the
                // shared-memory latency overlaps it
                const int ib = skip + (item - npre);
                double prev = 0.0;
                if (MODE == 0 && item >= npre) prev = extra[ib * STREAM_CONSUMERS + tid];
                // the test hook makes the first wait of the launch run out
                // (the simulated timeout takes the abort path below)
                const bool first = tile == blockIdx.x && item == 0;
                if ((a.fail_first_wait && first) || !mbar_wait(&full[s], phase, abort_flag))
                {
                    *abort_flag = 1;
                    atomicExch(a.error, 1);
                    ok = false;
                    break;
                }
                const VT* st = stages + static_cast<size_t>(s) * (STREAM_TILE_BYTES / sizeof(VT));
                if (item == 0)
                {
#pragma unroll
                    for (int k = 0; k < R; ++k)
                        w[k] = static_cast<double>(st[(roff + k * RSTEP) * PT + pl]);
                }
                else if (upd && item == 1)
                {
#pragma unroll
                    for (int k = 0; k < R; ++k)
                    {
                        vj[k] = static_cast<double>(st[(roff + k * RSTEP) * PT + pl]);
                        w[k] -= cj * vj[k];
                    }
                }
                else if (upd && item == 2 && a.Vm)
                {
#pragma unroll
                    for (int k = 0; k < R; ++k)
                        w[k] -= cm * static_cast<double>(st[(roff + k * RSTEP) * PT + pl]);
                }
                else
                {
                    const int i = ib;
                    if (MODE == 0)
                    {
                        // eight independent FMA chains: the pass is bound by
                        // the latency of this reduction (two warps per
                        // scheduler), not by FP64 throughput
                        double l[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                        for (int k = 0; k < R; ++k)
                            l[k & 7] += static_cast<double>(st[(roff + k * RSTEP) * PT + pl]) * w[k];
                        extra[i * STREAM_CONSUMERS + tid] =
                            prev + (((l[0] + l[1]) + (l[2] + l[3])) + ((l[4] + l[5]) + (l[6] + l[7])));
                    }
                    else
                    {
                        const double c = extra[i * PT + pl];
#pragma unroll
                        for (int k = 0; k < R; ++k)
                            w[k] -= c * static_cast<double>(st[(roff + k * RSTEP) * PT + pl]);
                    }
                }
                if (MODE == 0 && upd && item == npre - 1)
                {
                    // updated w: round to storage, store, and serve the
                    // products with v_j (registers) and v_{j-1} (still in
                    // this item's stage) without reading them again
                    double lj = 0.0, lm = 0.0;
#pragma unroll
                    for (int k = 0; k < R; ++k)
                    {
                        const VT wr = static_cast<VT>(w[k]);
                        w[k] = static_cast<double>(wr);
                        a.Wout[(row0 + roff + k * RSTEP) * b + p0 + pl] = wr;
                        nacc += w[k] * w[k];
                        lj += vj[k] * w[k];
                        if (a.Vm)
                            lm += static_cast<double>(st[(roff + k * RSTEP) * PT + pl]) * w[k];
                    }
                    if (J > 0) extra[0 * STREAM_CONSUMERS + tid] += lj;
                    if (a.Vm && J > 1) extra[1 * STREAM_CONSUMERS + tid] += lm;
                }
                release(s);
                if (++s == a.S) { s = 0; phase ^= 1; }
            }
            if (MODE == 1 && ok)
            {
#pragma unroll
                for (int k = 0; k < R; ++k)
                {
                    const VT wr = static_cast<VT>(w[k]);
                    const double d = static_cast<double>(wr);
                    nacc += d * d;
                    const int64_t row = row0 + roff + k * RSTEP;
                    a.Wout[row * b + p0 + pl] = wr;
                    if (x16_on)
                        x16_store(a.x16, row, b, p0 + pl, static_cast<float>(wr) * x16_scale);
                }
            }
        }

        // rows past the last whole tile: plain loads, last CTA only
        const int64_t tail0 = ntiles * a.T;
        if (ok && blockIdx.x == gridDim.x - 1 && tail0 < a.n)
        {
            for (int64_t r = tail0 + roff; r < a.n; r += RSTEP)
            {
                const int64_t o = r * b + p0 + pl;
                double wv = static_cast<double>(a.W[o]);
                if (upd)
                {
                    const double x = static_cast<double>(a.Vj[o]);
                    wv -= cj * x;
                    double y = 0.0;
                    if (a.Vm)
                    {
                        y = static_cast<double>(a.Vm[o]);
                        wv -= cm * y;
                    }
                    if (MODE == 0)
                    {
                        const VT wr = static_cast<VT>(wv);
                        wv = static_cast<double>(wr);
                        a.Wout[o] = wr;
                        nacc += wv * wv;
                        if (J > 0) extra[tid] += x * wv;
                        if (a.Vm && J > 1) extra[STREAM_CONSUMERS + tid] += y * wv;
                    }
                }
                for (int i = skip; i < J; ++i)
                {
                    const VT* vp = a.basis + static_cast<int64_t>(ring_slot(a.last - i, a.bs)) * a.slot_elems;
                    const double v = static_cast<double>(vp[o]);
                    if (MODE == 0) extra[i * STREAM_CONSUMERS + tid] += v * wv;
                    else wv -= extra[i * PT + pl] * v;
                }
                if (MODE == 1)
                {
                    const VT wr = static_cast<VT>(wv);
                    const double d = static_cast<double>(wr);
                    nacc += d * d;
                    a.Wout[o] = wr;
                    if (x16_on) x16_store(a.x16, r, b, p0 + pl, static_cast<float>(wr) * x16_scale);
                }
            }
        }
        red[tid] = nacc;
    }
    __syncthreads();

    if (producer) return;
    if (MODE == 0)
    {
        for (int idx = tid; idx < J * PT; idx += STREAM_CONSUMERS)
        {
            const int i = idx / PT;
            const int q = idx % PT;
            double sum = 0.0;
            for (int r = 0; r < RSTEP; ++r) sum += extra[i * STREAM_CONSUMERS + r * PT + q];
            a.partials[(static_cast<int64_t>(blockIdx.x) * J + i) * b + p0 + q] = sum;
        }
    }
    else if (a.want_norm)
    {
        for (int q = tid; q < PT; q += STREAM_CONSUMERS)
        {
            double sum = 0.0;
            for (int r = 0; r < RSTEP; ++r) sum += red[r * PT + q];
            a.partials[static_cast<int64_t>(blockIdx.x) * b + p0 + q] = sum;
        }
    }
    if (MODE == 0 && a.wn2_out)
    {
        for (int q = tid; q < PT; q += STREAM_CONSUMERS)
        {
            double sum = 0.0;
            for (int r = 0; r < RSTEP; ++r) sum += red[r * PT + q];
            a.wn2_out[static_cast<int64_t>(blockIdx.x) * b + p0 + q] = sum;
        }
    }
}


// ===========================================================================
// Row-group SpMM.
//
// Groups of G consecutive rows (after the locality order, neighbours) share
// most of their columns.  The row-group format stores, per group, the sorted
// union of the group's column indices and a dense G-wide value column per
// union entry (zero where a row lacks the column):
//   grp_ptr[g] .. grp_ptr[g+1]  union entries of group g
//   grp_col[u]                  column of entry u
//   grp_val[u*G + r]            value of row g*G+r at that column
// One X row gathered from L1/L2 then feeds G rows' FMAs from registers, so
// the gather traffic per useful FMA drops by ~G x fill.  Row sums run over
// the same ascending column order as CSR and the padding adds exact zeros,
// so results are bit-identical to k_spmm.
// ===========================================================================

// Union size of each group (warp per group; lanes < G hold the row cursors).
__global__ void k_rg_count(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ind,
                           int64_t nrows, int G, int32_t* __restrict__ counts, int64_t ngroups)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t ws = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t g = w0; g < ngroups; g += ws)
    {
        const int64_t row = g * G + lane;
        int k = 0, kend = 0;
        if (lane < G && row < nrows)
        {
            k = ptr[row];
            kend = ptr[row + 1];
        }
        int count = 0;
        for (;;)
        {
            const int head = (k < kend) ? ind[k] : INT_MAX;
            int mn = head;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                mn = min(mn, __shfl_xor_sync(FULL_MASK, mn, off));
            if (mn == INT_MAX) break;
            ++count;
            if (head == mn) ++k;
        }
        if (lane == 0) counts[g] = count;
    }
}

template <typename VT>
__global__ void k_rg_fill(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ind,
                          const VT* __restrict__ val, int64_t nrows, int G,
                          const int32_t* __restrict__ gptr, int32_t* __restrict__ gcol,
                          VT* __restrict__ gval, int64_t ngroups)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t ws = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t g = w0; g < ngroups; g += ws)
    {
        const int64_t row = g * G + lane;
        int k = 0, kend = 0;
        if (lane < G && row < nrows)
        {
            k = ptr[row];
            kend = ptr[row + 1];
        }
        int64_t u = gptr[g];
        for (;;)
        {
            const int head = (k < kend) ? ind[k] : INT_MAX;
            int mn = head;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                mn = min(mn, __shfl_xor_sync(FULL_MASK, mn, off));
            if (mn == INT_MAX) break;
            if (lane == 0) gcol[u] = mn;
            if (lane < G) gval[u * G + lane] = (head == mn) ? val[k] : VT(0);
            if (head == mn) ++k;
            ++u;
        }
    }
}

// Epilogue of one output row (lanes own LV consecutive probes each).
template <typename VT, int LV>
__device__ __forceinline__ void spmm_row_epilogue(int64_t row, int b, int p0, const VT (&acc)[LV],
                                                  const double (&sxr)[LV],
                                                  const double (&zcr)[LV], double shift,
                                                  const VT* __restrict__ X, VT* __restrict__ Y,
                                                  const VT* __restrict__ Z,
                                                  const double* __restrict__ zs, int epi,
                                                  double (&part)[LV])
{
    const int64_t o = row * b + p0;
    VT xr[LV], zr[LV], yr[LV];
    if (shift != 0.0 || epi == 1) ldg_n<VT, LV>(X + o, xr);
    if (Z) ldg_n<VT, LV>(Z + o, zr);
#pragma unroll
    for (int v = 0; v < LV; ++v)
    {
        double y = static_cast<double>(acc[v]) * sxr[v];
        if (shift != 0.0) y += shift * (sxr[v] * static_cast<double>(xr[v]));
        if (Z) y -= zcr[v] * static_cast<double>(zr[v]);
        yr[v] = static_cast<VT>(y);
        const double ys = static_cast<double>(yr[v]);
        if (epi == 1)
            part[v] += (sxr[v] * static_cast<double>(xr[v])) * ys;
        else if (epi == 2)
            part[v] += ys * ys;
        else if (epi == 3)
            part[v] += (zs[p0 + v] * static_cast<double>(zr[v])) * ys;
    }
    store_n<VT, LV>(Y + o, yr);
}

// b = 32 * LV * NS probes: NS warps share a row group, each owning a slice
// of 32 * LV probes (LV <= 4 keeps the G x LV accumulators and two gathers in
// flight within 128 registers, two CTAs per SM).  8 warps per CTA.
template <typename VT, int LV, int G, int NS>
__global__ void __launch_bounds__(256, 2)
k_spmm_rg(const int32_t* __restrict__ gptr, const int32_t* __restrict__ gcol,
          const VT* __restrict__ gval, int64_t nrows, int64_t ngroups, int b,
          const VT* __restrict__ X, const double* __restrict__ sx, double shift,
          VT* __restrict__ Y, const VT* __restrict__ Z, const double* __restrict__ zc,
          const double* __restrict__ zs, int epi, double* __restrict__ partials)
{
    __shared__ int32_t s_col[8][32];
    __shared__ __align__(16) VT s_val[8][32][G];
    __shared__ double s_red[8][256];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int slice = warp % NS;
    const int p0 = (slice * 32 + lane) * LV;
    constexpr int GPC = 8 / NS;  // row groups in flight per CTA

    double sxr[LV], zcr[LV], part[LV];
#pragma unroll
    for (int v = 0; v < LV; ++v)
    {
        sxr[v] = sx ? sx[p0 + v] : 1.0;
        zcr[v] = Z ? zc[p0 + v] * zs[p0 + v] : 0.0;
        part[v] = 0.0;
    }

    const int64_t gw = static_cast<int64_t>(blockIdx.x) * GPC + warp / NS;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * GPC;
    for (int64_t g = gw; g < ngroups; g += stride)
    {
        VT acc[G][LV];
#pragma unroll
        for (int r = 0; r < G; ++r)
#pragma unroll
            for (int v = 0; v < LV; ++v) acc[r][v] = VT(0);
        const int u0 = gptr[g];
        const int u1 = gptr[g + 1];
        for (int base = u0; base < u1; base += 32)
        {
            const int cnt = min(32, u1 - base);
            if (lane < cnt)
            {
                s_col[warp][lane] = __ldg(gcol + base + lane);
                VT tmp[G];
                ldg_n<VT, G>(gval + static_cast<int64_t>(base + lane) * G, tmp);
                store_n<VT, G>(&s_val[warp][lane][0], tmp);
            }
            __syncwarp();
            int t = 0;
            for (; t + 2 <= cnt; t += 2)
            {
                const int c0 = s_col[warp][t];
                const int c1 = s_col[warp][t + 1];
                VT x0[LV], x1[LV];
                ldg_n<VT, LV>(X + static_cast<int64_t>(c0) * b + p0, x0);
                ldg_n<VT, LV>(X + static_cast<int64_t>(c1) * b + p0, x1);
                VT a0[G], a1[G];
                load_n<VT, G>(&s_val[warp][t][0], a0);
                load_n<VT, G>(&s_val[warp][t + 1][0], a1);
#pragma unroll
                for (int r = 0; r < G; ++r)
#pragma unroll
                    for (int v = 0; v < LV; ++v)
                    {
                        acc[r][v] += a0[r] * x0[v];
                        acc[r][v] += a1[r] * x1[v];
                    }
            }
            if (t < cnt)
            {
                const int c0 = s_col[warp][t];
                VT x0[LV];
                ldg_n<VT, LV>(X + static_cast<int64_t>(c0) * b + p0, x0);
                VT a0[G];
                load_n<VT, G>(&s_val[warp][t][0], a0);
#pragma unroll
                for (int r = 0; r < G; ++r)
#pragma unroll
                    for (int v = 0; v < LV; ++v) acc[r][v] += a0[r] * x0[v];
            }
            __syncwarp();
        }
#pragma unroll
        for (int r = 0; r < G; ++r)
        {
            const int64_t row = g * G + r;
            if (row < nrows)
                spmm_row_epilogue<VT, LV>(row, b, p0, acc[r], sxr, zcr, shift, X, Y, Z, zs, epi,
                                          part);
        }
    }

    if (epi == 0) return;
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&s_red[0][0])[i] = 0.0;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < LV; ++v) s_red[warp][p0 + v] = part[v];
    __syncthreads();
    for (int p = threadIdx.x; p < b; p += blockDim.x)
    {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += s_red[w][p];
        partials[static_cast<int64_t>(blockIdx.x) * b + p] = s;
    }
}


// ===========================================================================
// Row-group SpMM with TMA gathers (FP32, b = 128 or 256).
//
// Same row-group format as k_spmm_rg, but the union columns' X rows are
// brought into shared memory by the copy engine (cp.async.bulk.tensor
// tile::gather4: four rows of the [len][b] block per instruction) together
// with the group's dense values (cp.async.bulk), STAGES - 1 stages ahead per
// warp.  Each warp owns its ring (no cross-warp waits); the FMAs read X from
// shared memory, so the gather latency no longer stalls the warp.
//
// A warp's row groups (slice = warp % NS, groups gw, gw + gstride, ...: the
// whole grid works through the groups in order, so the gather window stays
// inside L2) form one stage stream: the stages of the next group are issued
// while the current one is finished, and each group's offsets and first 32
// column ids are loaded a group ahead, so no global-load latency sits between
// stages.  FMAs are packed (fma.rn.f32x2: two rows of one probe), which
// rounds exactly as the scalar FMA, so results are bit-identical to k_spmm.
//
// Lane l owns probes slice*128 + 4l .. 4l + 3, so every shared-memory read
// of a stage row is a contiguous 512-byte span.
// ===========================================================================

constexpr int RGT_ROWS = 8;  // union columns per stage (two gather4)

// warps and ring stages per CTA: 16-row groups hold 64 accumulators per
// thread (12 warps, up to 168 registers), 8-row groups 32 (16 warps)
template <int G>
struct RgtShape {
    static constexpr int WARPS = (G == 16) ? 12 : 16;
    static constexpr int STAGES = (G == 16) ? 4 : 3;
    static constexpr int STAGE = RGT_ROWS * 128 * 4 + RGT_ROWS * G * 4;
    static constexpr size_t RING = static_cast<size_t>(WARPS) * STAGES * STAGE;
    static constexpr size_t SMEM =
        1024 + (RING > static_cast<size_t>(WARPS) * 256 * 8 ? RING : static_cast<size_t>(WARPS) * 256 * 8);
};

__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, int col,
                                            int r0, int r1, int r2, int r3, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(col), "r"(r0), "r"(r1),
          "r"(r2), "r"(r3), "r"(smem_u32(bar))
        : "memory");
}

// b = 128 * NS probes; NS warps share a row group, each owning a 128-probe
// slice.  The tensor map's box is one row of 128 values.
template <int G, int NS>
__global__ void __launch_bounds__(RgtShape<G>::WARPS * 32, 1)
k_spmm_rgt(const __grid_constant__ CUtensorMap xmap, const int32_t* __restrict__ gptr,
           const int32_t* __restrict__ gcol, const float* __restrict__ gval, int64_t nrows,
           int64_t ngroups, int b, const float* __restrict__ X, const double* __restrict__ sx,
           double shift, float* __restrict__ Y, const float* __restrict__ Z,
           const double* __restrict__ zc, const double* __restrict__ zs, int epi,
           double* __restrict__ partials, int32_t* __restrict__ error)
{
    constexpr int WARPS = RgtShape<G>::WARPS;
    constexpr int STAGES = RgtShape<G>::STAGES;
    constexpr int STAGE = RgtShape<G>::STAGE;
    constexpr int LV = 4;
    constexpr int ROWB = 128 * 4;                    // bytes of one row slice
    constexpr int STAGE_X = RGT_ROWS * ROWB;
    constexpr int GPC = WARPS / NS;                  // groups in flight per CTA
    static_assert(WARPS * STAGES * 8 <= 1024, "barrier area");
    extern __shared__ __align__(128) unsigned char smem_rgt[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_rgt);              // [warps][stages]
    unsigned char* ring0 = smem_rgt + 1024;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int slice = warp % NS;
    unsigned char* ring = ring0 + static_cast<size_t>(warp) * STAGES * STAGE;
    uint64_t* wbar = bars + warp * STAGES;

    if (lane == 0)
        for (int st = 0; st < STAGES; ++st) mbar_init(&wbar[st], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();

    const int pbase = slice * 128 + lane * 4;        // this lane's 4 probes
    double part[LV];
#pragma unroll
    for (int v = 0; v < LV; ++v) part[v] = 0.0;

    // group sequence of this warp; groups i1 (offsets + first id chunk
    // loaded), i2 (offsets loaded) and i3 come after the one being issued
    const int64_t gstride = static_cast<int64_t>(gridDim.x) * GPC;
    int64_t snext = static_cast<int64_t>(blockIdx.x) * GPC + warp / NS;
    auto fetch = [&]() {
        const int64_t g = snext;
        snext += gstride;
        return g;
    };
    int64_t i1 = fetch(), i2 = fetch(), i3 = fetch();
    int u1 = 0, e1 = 0, c1 = 0, u2 = 0, e2 = 0;
    if (i1 < ngroups)
    {
        u1 = __ldg(gptr + i1);
        e1 = __ldg(gptr + i1 + 1);
        c1 = (u1 + lane < e1) ? __ldg(gcol + u1 + lane) : 0;
    }
    if (i2 < ngroups)
    {
        u2 = __ldg(gptr + i2);
        e2 = __ldg(gptr + i2 + 1);
    }

    // producer cursor: group pg (-1: none left), next entry pe of [.., pend),
    // ids of entries cb .. cb + 63 in cur / nxt (one per lane)
    int64_t pg = -1;
    int pe = 0, pend = 0, cb = 0, cur = 0, nxt = 0;
    bool pfirst = true;
    auto advance = [&]() {
        pg = (i1 < ngroups) ? i1 : -1;
        pe = u1;
        pend = e1;
        cb = u1;
        cur = c1;
        nxt = (pg >= 0 && u1 + 32 + lane < e1) ? __ldg(gcol + u1 + 32 + lane) : 0;
        pfirst = true;
        i1 = i2;
        u1 = u2;
        e1 = e2;
        c1 = (i2 < ngroups && u2 + lane < e2) ? __ldg(gcol + u2 + lane) : 0;
        i2 = i3;
        if (i3 < ngroups)
        {
            u2 = __ldg(gptr + i3);
            e2 = __ldg(gptr + i3 + 1);
            i3 = fetch();
        }
    };
    advance();

    // stage metadata, oldest first: group (-1: none), cnt | first << 8 | last << 9
    int64_t qg[STAGES];
    int qf[STAGES];
    auto issue = [&](int st, int64_t& og, int& of) {
        if (pg < 0)
        {
            og = -1;
            of = 0;
            return;
        }
        const int cnt = min(RGT_ROWS, pend - pe);
        unsigned char* dst = ring + static_cast<size_t>(st) * STAGE;
        int id[RGT_ROWS];
#pragma unroll
        for (int i = 0; i < RGT_ROWS; ++i)
        {
            // entries past the group's end repeat its last one (copied, unused)
            const int off = pe + min(i, max(cnt - 1, 0)) - cb;
            id[i] = __shfl_sync(FULL_MASK, off < 32 ? cur : nxt, off & 31);
        }
        if (lane == 0)
        {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (cnt > 0)
            {
                mbar_expect_tx(&wbar[st], static_cast<uint32_t>(STAGE_X + cnt * G * 4));
                tma_gather4(dst, &xmap, slice * 128, id[0], id[1], id[2], id[3], &wbar[st]);
                tma_gather4(dst + 4 * ROWB, &xmap, slice * 128, id[4], id[5], id[6], id[7],
                            &wbar[st]);
                bulk_copy_g2s(dst + STAGE_X, gval + static_cast<int64_t>(pe) * G,
                              static_cast<uint32_t>(cnt * G * 4), &wbar[st]);
            }
            else
            {
                mbar_expect_tx(&wbar[st], 0u);  // a group without entries
            }
        }
        const bool last = (pe + cnt == pend);
        og = pg;
        of = cnt | (pfirst ? 256 : 0) | (last ? 512 : 0);
        pfirst = false;
        pe += cnt;
        if (pe - cb >= 32)
        {
            cb += 32;
            cur = nxt;
            nxt = (cb + 32 + lane < pend) ? __ldg(gcol + cb + 32 + lane) : 0;
        }
        if (last) advance();
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) issue(s, qg[s], qf[s]);

    float2 acc[G / 2][LV];  // (row 2q, row 2q + 1) of probe v
    uint32_t phases = 0;    // bit st = parity of stage st's next completion
    bool ok = true;
    const int dummy_flag = 0;
    int st = 0;             // slot of the stage consumed now
    for (;;)
    {
        {
            int nst = st + STAGES - 1;
            if (nst >= STAGES) nst -= STAGES;
            issue(nst, qg[STAGES - 1], qf[STAGES - 1]);
        }
        if (qg[0] < 0) break;
        if (!mbar_wait(&wbar[st], (phases >> st) & 1u, &dummy_flag))
        {
            ok = false;
            if (lane == 0) atomicExch(error, 1);
            break;
        }
        phases ^= (1u << st);
        const int cnt = qf[0] & 255;
        if (qf[0] & 256)
        {
#pragma unroll
            for (int q = 0; q < G / 2; ++q)
#pragma unroll
                for (int v = 0; v < LV; ++v) acc[q][v] = make_float2(0.0f, 0.0f);
        }
        const unsigned char* src = ring + static_cast<size_t>(st) * STAGE;
        const float* avals = reinterpret_cast<const float*>(src + STAGE_X);
        for (int c = 0; c < cnt; ++c)
        {
            const float4 xv = *reinterpret_cast<const float4*>(src + c * ROWB + lane * 16);
            const float x[4] = {xv.x, xv.y, xv.z, xv.w};
            float2 a2[G / 2];
#pragma unroll
            for (int q = 0; q < G; q += 4)
            {
                const float4 t = *reinterpret_cast<const float4*>(avals + c * G + q);
                a2[q / 2] = make_float2(t.x, t.y);
                a2[q / 2 + 1] = make_float2(t.z, t.w);
            }
#pragma unroll
            for (int v = 0; v < LV; ++v)
            {
                const float2 xx = make_float2(x[v], x[v]);
#pragma unroll
                for (int q = 0; q < G / 2; ++q) acc[q][v] = __ffma2_rn(a2[q], xx, acc[q][v]);
            }
        }
        __syncwarp();
        if (qf[0] & 512)
        {
            const int64_t g = qg[0];
            double sxr[LV], zcr[LV];
#pragma unroll
            for (int v = 0; v < LV; ++v)
            {
                sxr[v] = sx ? sx[pbase + v] : 1.0;
                zcr[v] = Z ? zc[pbase + v] * zs[pbase + v] : 0.0;
            }
#pragma unroll
            for (int r = 0; r < G; ++r)
            {
                const int64_t row = g * G + r;
                if (row >= nrows) continue;
                const int64_t o = row * b + pbase;
                float4 xr = make_float4(0.f, 0.f, 0.f, 0.f), zr = xr;
                if (shift != 0.0 || epi == 1) xr = __ldg(reinterpret_cast<const float4*>(X + o));
                if (Z) zr = __ldg(reinterpret_cast<const float4*>(Z + o));
                const float xs[4] = {xr.x, xr.y, xr.z, xr.w};
                const float zsv[4] = {zr.x, zr.y, zr.z, zr.w};
                float yr[4];
#pragma unroll
                for (int v = 0; v < LV; ++v)
                {
                    const float av = (r & 1) ? acc[r / 2][v].y : acc[r / 2][v].x;
                    double y = static_cast<double>(av) * sxr[v];
                    if (shift != 0.0) y += shift * (sxr[v] * static_cast<double>(xs[v]));
                    if (Z) y -= zcr[v] * static_cast<double>(zsv[v]);
                    yr[v] = static_cast<float>(y);
                    const double ys = static_cast<double>(yr[v]);
                    if (epi == 1) part[v] += (sxr[v] * static_cast<double>(xs[v])) * ys;
                    else if (epi == 2) part[v] += ys * ys;
                    else if (epi == 3)
                        part[v] += (zs[pbase + v] * static_cast<double>(zsv[v])) * ys;
                }
                *reinterpret_cast<float4*>(Y + o) = make_float4(yr[0], yr[1], yr[2], yr[3]);
            }
        }
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s)
        {
            qg[s] = qg[s + 1];
            qf[s] = qf[s + 1];
        }
        if (++st == STAGES) st = 0;
    }
    if (!ok)
    {
        // let this warp's copies in flight land before leaving
        int s2 = st;
#pragma unroll
        for (int s = 0; s < STAGES; ++s)
        {
            if (qg[s] >= 0) mbar_wait(&wbar[s2], (phases >> s2) & 1u, &dummy_flag);
            if (++s2 == STAGES) s2 = 0;
        }
    }

    if (epi == 0) return;
    // all copies have landed (every issued stage was waited on), so the ring
    // memory can hold the CTA reduction: red[warp][256]
    __syncthreads();
    double* red = reinterpret_cast<double*>(ring0);
    for (int i = threadIdx.x; i < WARPS * 256; i += blockDim.x) red[i] = 0.0;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < LV; ++v) red[warp * 256 + pbase + v] = part[v];
    __syncthreads();
    for (int p = threadIdx.x; p < b; p += blockDim.x)
    {
        double sum = 0.0;
        for (int w = 0; w < WARPS; ++w) sum += red[w * 256 + p];
        partials[static_cast<int64_t>(blockIdx.x) * b + p] = sum;
    }
}


// ===========================================================================
// Tensor-core row-group SpMM (FP32, 16-row groups, b = 128 NS probes).
//
// Per work item (row group g, 128-probe slice) and K step of 8 union columns
// the tile D[128 probes][16 rows] += X^T[128][8] A_g^T[8][16] runs on the
// tensor cores as three kind::tf32 MMAs on TF32 hi/lo splits (slq_tc.cuh):
//   warp 9     copy producer: the step's 8 X rows (two TMA tile::gather4
//              of 128 probes) and the group's 8 x 16 values (bulk copy)
//              into a 20-stage shared-memory ring, the union column ids
//              read 32 at a time across the warp, one chunk ahead;
//   warps 0-3  converters (thread = probe): read their X values and one
//              group value each from the ring, free the ring stage, split
//              into TF32 hi/lo, store A to a tensor-memory stage (their own
//              lane quarter) and B as K-major tiles in shared memory;
//   warp 8     MMA issuer (one thread) and tensor-memory owner;
//   warps 4-7  epilogue: read the finished accumulator (16 rows of their
//              lane quarter's probes), apply the SpMM epilogue (scale, shift,
//              three-term subtraction, alpha / norm partials) and store Y.
// Barriers: ring (sfull / sempty), tensor-memory stages (tfull / tempty, 4
// stages), accumulator double buffer (acc_full / acc_empty).  Tensor memory
// per CTA: stage s A hi at column 16 s, A lo at 16 s + 8, accumulator i at
// 64 + 16 i (128 columns allocated).  Every wait is bounded; a wait that
// runs out sets *error and the abort flag and every role leaves; the copy
// thread waits (bounded) for its copies in flight and the MMA thread drains
// its MMAs before the tensor memory is freed.  Each probe's partial sum
// belongs to one epilogue thread, so partials[block][p] is written without a
// CTA reduction.  Sums run in the tensor core's order, so results agree with
// the CUDA-core kernels to FP32 rounding, not bitwise.
// ===========================================================================

constexpr int TC_XSTAGES = 20;
constexpr size_t TC_DYN_SMEM = TC_XSTAGES * (8 * 128 + 8 * 16) * sizeof(float);
constexpr int TC_TSTAGES = 4;
constexpr int TC_THREADS = 320;
constexpr uint32_t TC_COLS = 128;

template <int NS>
__global__ void __launch_bounds__(TC_THREADS, 2)
k_spmm_tc(const __grid_constant__ CUtensorMap xmap, const int32_t* __restrict__ gptr,
          const int32_t* __restrict__ gcol, const float* __restrict__ gval, int64_t nrows,
          int64_t ngroups, int b, const float* __restrict__ X, const double* __restrict__ sx,
          double shift, float* __restrict__ Y, const float* __restrict__ Z,
          const double* __restrict__ zc, const double* __restrict__ zs, int epi,
          double* __restrict__ partials, int32_t* __restrict__ error)
{
    // dynamic shared memory: X rows of a step [TC_XSTAGES][8 * 128], group
    // values of a step [TC_XSTAGES][8 * 16]; static: B tiles
    extern __shared__ __align__(1024) unsigned char smem_tc[];
    float (*xst)[8 * 128] = reinterpret_cast<float (*)[8 * 128]>(smem_tc);
    float (*vst)[8 * 16] =
        reinterpret_cast<float (*)[8 * 16]>(smem_tc + TC_XSTAGES * 8 * 128 * sizeof(float));
    __shared__ __align__(1024) unsigned char bst[TC_TSTAGES][2][512];  // B hi / lo, K-major
    __shared__ __align__(8) uint64_t sfull[TC_XSTAGES];
    __shared__ __align__(8) uint64_t sempty[TC_XSTAGES];
    __shared__ __align__(8) uint64_t tfull[TC_TSTAGES];
    __shared__ __align__(8) uint64_t tempty[TC_TSTAGES];
    __shared__ __align__(8) uint64_t acc_full[2];
    __shared__ __align__(8) uint64_t acc_empty[2];
    __shared__ __align__(8) uint64_t drain;
    __shared__ uint32_t tbase;
    __shared__ int abort_flag[2];  // [1] stays 0: bounded waits on the way out

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int64_t nitems = ngroups * NS;

    if (warp == 8)
    {
        tc::tmem_alloc(&tbase, TC_COLS);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        for (int s = 0; s < TC_XSTAGES; ++s)
        {
            mbar_init(&sfull[s], 1);
            mbar_init(&sempty[s], 4);
        }
        for (int s = 0; s < TC_TSTAGES; ++s)
        {
            mbar_init(&tfull[s], 4);
            mbar_init(&tempty[s], 1);
        }
        for (int i = 0; i < 2; ++i)
        {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 4);
        }
        mbar_init(&drain, 1);
        abort_flag[0] = 0;
        abort_flag[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tb = tbase;
    auto give_up = [&]() {
        *reinterpret_cast<volatile int*>(abort_flag) = 1;
        atomicExch(error, 1);
    };

    if (warp == 9)
    {
        // copy producer: the whole warp walks the steps (lane l holds union
        // column id l of the current 32-entry chunk, the next chunk is
        // loaded one chunk ahead); lane 0 issues the copies
        int64_t kstep = 0;
        bool ok = true;
        for (int64_t item = blockIdx.x; item < nitems && ok; item += gridDim.x)
        {
            const int64_t g = item / NS;
            const int sl = static_cast<int>(item % NS);
            const int u0 = gptr[g];
            const int nu = gptr[g + 1] - u0;
            const int T = max(1, (nu + 7) / 8);
            const int last = (nu > 0) ? gcol[u0 + nu - 1] : 0;
            int cur = (lane < nu) ? gcol[u0 + lane] : last;
            int nxt = (32 + lane < nu) ? gcol[u0 + 32 + lane] : last;
            for (int t = 0; t < T; ++t, ++kstep)
            {
                const int e0 = t * 8;
                if (t > 0 && (e0 & 31) == 0)
                {
                    cur = nxt;
                    const int e = e0 + 32 + lane;
                    nxt = (e < nu) ? gcol[u0 + e] : last;
                }
                const int s = static_cast<int>(kstep % TC_XSTAGES);
                const int64_t use = kstep / TC_XSTAGES;
                const int cnt = min(8, nu - e0);  // <= 0 only for an empty group
                int id[8];
#pragma unroll
                for (int k = 0; k < 8; ++k)
                {
                    const int v = __shfl_sync(FULL_MASK, cur, (e0 + k) & 31);
                    id[k] = (k < cnt) ? v : last;
                }
                bool good = true;
                if (lane == 0)
                {
                    good = *reinterpret_cast<volatile int*>(abort_flag) == 0;
                    if (good && use > 0) good = mbar_wait(&sempty[s], (use - 1) & 1, abort_flag);
                    if (!good)
                    {
                        give_up();
                    }
                    else
                    {
                        const uint32_t vbytes = cnt > 0 ? static_cast<uint32_t>(cnt * 64) : 0u;
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        mbar_expect_tx(&sfull[s], 8u * 512u + vbytes);
                        tma_gather4(&xst[s][0], &xmap, sl * 128, id[0], id[1], id[2], id[3],
                                    &sfull[s]);
                        tma_gather4(&xst[s][4 * 128], &xmap, sl * 128, id[4], id[5], id[6],
                                    id[7], &sfull[s]);
                        if (vbytes)
                            bulk_copy_g2s(&vst[s][0], gval + static_cast<int64_t>(u0 + e0) * 16,
                                          vbytes, &sfull[s]);
                    }
                }
                if (!__shfl_sync(FULL_MASK, good ? 1 : 0, 0))
                {
                    ok = false;
                    break;
                }
            }
        }
        // the copies in flight land before the CTA leaves
        if (lane == 0)
            for (int64_t k = (kstep > TC_XSTAGES ? kstep - TC_XSTAGES : 0); k < kstep; ++k)
                mbar_wait(&sfull[k % TC_XSTAGES], (k / TC_XSTAGES) & 1, abort_flag + 1);
        __syncwarp();
    }
    else if (warp < 4)
    {
        // converters
        const int cq = warp;
        const uint32_t lanes = static_cast<uint32_t>(32 * cq) << 16;
        const int kb = tid >> 4;  // this thread's group value: K row kb, group row nb
        const int nb = tid & 15;
        int64_t kstep = 0;
        bool ok = true;
        for (int64_t item = blockIdx.x; item < nitems && ok; item += gridDim.x)
        {
            const int64_t g = item / NS;
            const int nu = gptr[g + 1] - gptr[g];
            const int T = max(1, (nu + 7) / 8);
            for (int t = 0; t < T; ++t, ++kstep)
            {
                const int s = static_cast<int>(kstep % TC_XSTAGES);
                const int64_t use = kstep / TC_XSTAGES;
                const int ts = static_cast<int>(kstep % TC_TSTAGES);
                const int64_t tuse = kstep / TC_TSTAGES;
                const int cnt = min(8, nu - t * 8);
                if (!__all_sync(FULL_MASK, mbar_wait(&sfull[s], use & 1, abort_flag)))
                {
                    if (lane == 0) give_up();
                    ok = false;
                    break;
                }
                uint32_t hi[8], lo[8];
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    tc::split_tf32(k < cnt ? xst[s][k * 128 + cq * 32 + lane] : 0.0f, hi[k],
                                   lo[k]);
                uint32_t bh, bl;
                tc::split_tf32(kb < cnt ? vst[s][kb * 16 + nb] : 0.0f, bh, bl);
                // the split consumed the ring values: the stage can be refilled
                __syncwarp();
                if (lane == 0) mbar_arrive(&sempty[s]);
                bool good = true;
                if (tuse > 0) good = mbar_wait(&tempty[ts], (tuse - 1) & 1, abort_flag);
                if (!__all_sync(FULL_MASK, good))
                {
                    if (lane == 0) give_up();
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                tc::st_x8(tb + lanes + 16 * ts, hi);
                tc::st_x8(tb + lanes + 16 * ts + 8, lo);
                *reinterpret_cast<uint32_t*>(bst[ts][0] + tc::kmajor_offset(nb, kb)) = bh;
                *reinterpret_cast<uint32_t*>(bst[ts][1] + tc::kmajor_offset(nb, kb)) = bl;
                tc::fence_proxy_async_smem();
                tc::wait_st();
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tfull[ts]);
            }
        }
    }
    else if (warp == 8)
    {
        // MMA issuer
        if (lane == 0)
        {
            int64_t kstep = 0;
            int64_t it = 0;
            bool ok = true;
            for (int64_t item = blockIdx.x; item < nitems && ok; item += gridDim.x, ++it)
            {
                const int64_t g = item / NS;
                const int nu = gptr[g + 1] - gptr[g];
                const int T = max(1, (nu + 7) / 8);
                const int db = static_cast<int>(it & 1);
                const int64_t duse = it >> 1;
                if (duse > 0 && !mbar_wait(&acc_empty[db], (duse - 1) & 1, abort_flag))
                {
                    give_up();
                    break;
                }
                tc::fence_after_sync();
                const uint32_t dcol = tb + 64 + 16 * db;
                for (int t = 0; t < T; ++t, ++kstep)
                {
                    const int ts = static_cast<int>(kstep % TC_TSTAGES);
                    const int64_t tuse = kstep / TC_TSTAGES;
                    if (!mbar_wait(&tfull[ts], tuse & 1, abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint64_t bh = tc::smem_desc(bst[ts][0], 128, 256);
                    const uint64_t bl = tc::smem_desc(bst[ts][1], 128, 256);
                    const uint32_t ahi = tb + 16 * ts;
                    const uint32_t alo = ahi + 8;
                    tc::mma_tf32_ts(dcol, alo, bh, tc::IDESC_TF32_M128_N16, t > 0 ? 1u : 0u);
                    tc::mma_tf32_ts(dcol, ahi, bl, tc::IDESC_TF32_M128_N16, 1u);
                    tc::mma_tf32_ts(dcol, ahi, bh, tc::IDESC_TF32_M128_N16, 1u);
                    tc::commit(&tempty[ts]);
                }
                if (ok) tc::commit(&acc_full[db]);
            }
            // every issued MMA completes before the tensor memory is freed
            tc::commit(&drain);
            mbar_wait(&drain, 0, abort_flag + 1);
        }
        __syncwarp();
    }
    else
    {
        // epilogue
        const int q = warp - 4;
        const uint32_t lanes = static_cast<uint32_t>(32 * q) << 16;
        double part[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) part[i] = 0.0;
        int64_t it = 0;
        for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x, ++it)
        {
            const int64_t g = item / NS;
            const int sl = static_cast<int>(item % NS);
            const int db = static_cast<int>(it & 1);
            const int64_t duse = it >> 1;
            if (!__all_sync(FULL_MASK, mbar_wait(&acc_full[db], duse & 1, abort_flag)))
            {
                if (lane == 0) give_up();
                break;
            }
            tc::fence_after_sync();
            uint32_t v[16];
            tc::ld_x16(tb + lanes + 64 + 16 * db, v);
            tc::wait_ld();
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[db]);
            const int p = sl * 128 + q * 32 + lane;
            const double sxp = sx ? sx[p] : 1.0;
            const double zcp = Z ? zc[p] * zs[p] : 0.0;
#pragma unroll
            for (int r = 0; r < 16; ++r)
            {
                const int64_t row = g * 16 + r;
                if (row >= nrows) continue;
                const int64_t o = row * b + p;
                const float xr = (shift != 0.0 || epi == 1) ? __ldg(X + o) : 0.0f;
                const float zr = Z ? __ldg(Z + o) : 0.0f;
                double y = static_cast<double>(__uint_as_float(v[r])) * sxp;
                if (shift != 0.0) y += shift * (sxp * static_cast<double>(xr));
                if (Z) y -= zcp * static_cast<double>(zr);
                const float yf = static_cast<float>(y);
                Y[o] = yf;
                const double ys = static_cast<double>(yf);
                double add = 0.0;
                if (epi == 1)
                    add = (sxp * static_cast<double>(xr)) * ys;
                else if (epi == 2)
                    add = ys * ys;
                else if (epi == 3)
                    add = (zs[p] * static_cast<double>(zr)) * ys;
#pragma unroll
                for (int i = 0; i < NS; ++i)
                    if (i == sl) part[i] += add;
            }
        }
        if (epi != 0)
        {
#pragma unroll
            for (int i = 0; i < NS; ++i)
                partials[static_cast<int64_t>(blockIdx.x) * b + i * 128 + q * 32 + lane] = part[i];
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (warp == 8)
    {
        tc::fence_after_sync();
        tc::tmem_dealloc(tb, TC_COLS);
    }
}

// ===========================================================================
// Dense operator product on the tensor cores (FP32 data, three TF32 terms).
//
// Y[M][b] = A[M][K] X[K][b] for a dense row-major A.  A is split once into
// TF32 parts, hi = rn_tf32(a), lo = rn_tf32(a - hi), stored K-major with a
// row pitch ldk (a multiple of 32, zero-padded); each product splits and
// transposes the probe block likewise (XT[p][k], k contiguous), at most 256
// probes at a time.  A CTA computes 128-row tiles of Y (persistent over the
// tiles): TMA loads 32-value K slices of A_hi, A_lo, XT_hi, XT_lo
// (128-byte rows, SWIZZLE_128B) into a two-stage ring, one thread issues
// per K step of 8 the three kind::tf32 MMAs A_hi XT_hi + A_hi XT_lo +
// A_lo XT_hi into an FP32 accumulator in tensor memory (D[128][N], lane =
// row, column = probe).  The tensor core's FP32 accumulation does not round
// to nearest: its error is biased towards zero and grows with the number of
// MMAs into one accumulator.  So each 128-value K chunk goes to a fresh
// accumulator that four warps add into a running total (also in tensor
// memory) with round-to-nearest FP32 adds, and then apply the SpMM epilogue
// to it (thread t = row t of the tile).  Measured bias of Y (mean signed
// error over mean |Y|, exponential-kernel matrices, n = 4096..16384):
// 1.4e-6 with one accumulator per 512 values, 3.5e-7 per 128 at the same
// speed for n >= 16384 (10 % slower at n = 4096), 1.7e-7 per 64 (25 %
// slower at n = 4096).  The dropped lo*lo term and the rounding of the lo
// parts leave ~2^-21 relative error per product.  Probe partial sums are
// reduced across the tile's rows in a fixed order.
// ===========================================================================

constexpr int DT_BK = 32;       // K values per stage (one 128-byte row)
constexpr int DT_STAGES = 2;
#ifndef SLQ_DT_CHUNK
#define SLQ_DT_CHUNK 4
#endif
constexpr int DT_CHUNK = SLQ_DT_CHUNK;  // stages per accumulation chunk (128 K values)
constexpr int DT_THREADS = 192; // warps 0-3 accumulate, 4 loads, 5 issues MMAs
#ifndef SLQ_DT_PREFETCH
#define SLQ_DT_PREFETCH 4
#endif
constexpr int DT_PREFETCH = SLQ_DT_PREFETCH;  // A stages prefetched into L2 ahead (0: none; 4 measured 3 % faster at n = 16384, no change at 4096-8192)

__device__ __forceinline__ void split_tf32_f(float x, float& hi, float& lo)
{
    uint32_t h, l;
    tc::split_tf32(x, h, l);
    hi = __uint_as_float(h);
    lo = __uint_as_float(l);
}

// out[r * ldo + c] = parts of src[r * lds + c] for r < rows, c < cols
__global__ void k_split_rows(const float* __restrict__ src, int64_t rows, int64_t cols,
                             int64_t lds, int64_t ldo, float* __restrict__ hi,
                             float* __restrict__ lo)
{
    const int64_t total = rows * cols;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t r = i / cols, c = i % cols;
        float h, l;
        split_tf32_f(src[r * lds + c], h, l);
        hi[r * ldo + c] = h;
        lo[r * ldo + c] = l;
    }
}

// out[j * ldo + r] = parts of src[r * lds + col0 + j] for r < rows, j < ncols
// (32 x 32 tiles through shared memory; block 32 x 8)
__global__ void k_split_transpose(const float* __restrict__ src, int64_t rows, int64_t lds,
                                  int64_t col0, int64_t ncols, int64_t ldo,
                                  float* __restrict__ hi, float* __restrict__ lo)
{
    __shared__ float t[32][33];
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * 32;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * 32;
    for (int j = threadIdx.y; j < 32; j += 8)
    {
        const int64_t r = r0 + j, c = c0 + threadIdx.x;
        t[j][threadIdx.x] = (r < rows && c < ncols) ? src[r * lds + col0 + c] : 0.0f;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8)
    {
        const int64_t c = c0 + j, r = r0 + threadIdx.x;
        if (c < ncols && r < rows)
        {
            float h, l;
            split_tf32_f(t[threadIdx.x][j], h, l);
            hi[c * ldo + r] = h;
            lo[c * ldo + r] = l;
        }
    }
}

struct DenseArgs {
    int64_t M, K;        // rows of Y, inner dimension
    int nb, NB, ntn;     // probes in this chunk; probes per tile (a multiple
                         // of 16); probe tiles per row tile
    int b, p_off;        // block width (row pitch of X, Y, Z) and chunk offset
    uint32_t tmem_cols;  // power of two >= max(32, NB)
    const float* X;
    const double* sx;
    double shift;
    float* Y;
    const float* Z;
    const double* zc;
    const double* zs;
    int epi;
    double* partials;    // [grid][b]
    int32_t* error;
    int ksplit;          // K parts per tile (1: the epilogue runs here)
    float* acc;          // ksplit > 1: running totals [ksplit][M][NB]
};

__global__ void __launch_bounds__(DT_THREADS, 1)
k_dense_tc(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
           const __grid_constant__ CUtensorMap x_hi, const __grid_constant__ CUtensorMap x_lo,
           const DenseArgs d)
{
    extern __shared__ __align__(1024) unsigned char smem_dense[];
    // [stages][A_hi 16 KB | A_lo 16 KB | B_hi NB*128 | B_lo NB*128] at a
    // 1024-aligned base, then barriers, tensor-memory address, reduction
    const uint32_t a_bytes = 128 * DT_BK * 4;
    const uint32_t b_bytes = static_cast<uint32_t>(d.NB) * DT_BK * 4;
    const uint32_t stage_bytes = 2 * a_bytes + 2 * b_bytes;
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_dense) + 1023) & ~uintptr_t(1023));
    unsigned char* tail = base + DT_STAGES * stage_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(tail);
    uint64_t* empty = full + DT_STAGES;
    uint64_t* chunk_full = empty + DT_STAGES;
    uint64_t* chunk_empty = chunk_full + 1;
    uint64_t* drain = chunk_empty + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 2);  // [2]
    double* red = reinterpret_cast<double*>(tail + 128);     // [4][256]

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    if (tid == 0)
    {
        for (int s = 0; s < DT_STAGES; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(chunk_full, 1);
        mbar_init(chunk_empty, 4);  // one arrival per accumulating warp
        mbar_init(drain, 1);
        abort_flag[0] = 0;
        abort_flag[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 4 * 256; i += DT_THREADS) red[i] = 0.0;
    if (warp == 0)
    {
        tc::tmem_alloc(tmem_slot, d.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    // running total in columns [0, NB), the chunk accumulator after it
    const uint32_t d_chunk = tmem + d.tmem_cols / 2;

    // units: 128 rows x NB probes x one of ksplit K parts, the probe tiles of
    // a row tile adjacent (they share the A stream through L2); part p of a
    // tile takes the accumulation chunks [p nch / ksplit, (p + 1) nch / ksplit)
    const int64_t ntiles = (d.M + 127) / 128 * d.ntn * d.ksplit;
    const int64_t nk = (d.K + DT_BK - 1) / DT_BK;
    const int64_t nch = (nk + DT_CHUNK - 1) / DT_CHUNK;  // chunks per tile
    auto k_range = [&](int64_t unit, int64_t& k0, int64_t& k1) {
        const int64_t part = unit % d.ksplit;
        k0 = part * nch / d.ksplit * DT_CHUNK;
        k1 = std::min<int64_t>(nk, (part + 1) * nch / d.ksplit * DT_CHUNK);
    };
    const uint32_t idesc = tc::idesc_tf32_m128(static_cast<uint32_t>(d.NB));
    auto give_up = [&]() {
        abort_flag[0] = 1;
        atomicExch(d.error, 1);
    };

    if (warp == 4)
    {
        // producer: the A and probe-block parts of every stage of every tile
        int64_t it = 0;
        if (lane == 0)
        {
            bool ok = true;
            for (int64_t unit = blockIdx.x; unit < ntiles && ok; unit += gridDim.x)
            {
                const int64_t tile = unit / d.ksplit;
                const int row0 = static_cast<int>(tile / d.ntn * 128);
                const int col0 = static_cast<int>(tile % d.ntn) * d.NB;
                int64_t k0, k1;
                k_range(unit, k0, k1);
                for (int64_t k = k0; k < k1; ++k, ++it)
                {
                    const int s = static_cast<int>(it % DT_STAGES);
                    const uint32_t ph = static_cast<uint32_t>((it / DT_STAGES) & 1);
                    if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    unsigned char* st = base + static_cast<size_t>(s) * stage_bytes;
                    mbar_expect_tx(&full[s], stage_bytes);
                    const int kx = static_cast<int>(k * DT_BK);
                    if (DT_PREFETCH > 0 && k + DT_PREFETCH < k1)
                    {
                        const int kp = static_cast<int>((k + DT_PREFETCH) * DT_BK);
                        tc::tma_prefetch_2d(&a_hi, kp, row0);
                        tc::tma_prefetch_2d(&a_lo, kp, row0);
                    }
                    tc::tma_load_2d(st, &a_hi, kx, row0, &full[s]);
                    tc::tma_load_2d(st + a_bytes, &a_lo, kx, row0, &full[s]);
                    tc::tma_load_2d(st + 2 * a_bytes, &x_hi, kx, col0, &full[s]);
                    tc::tma_load_2d(st + 2 * a_bytes + b_bytes, &x_lo, kx, col0, &full[s]);
                }
            }
            // the copies in flight land before the CTA leaves
            for (int64_t k = it - DT_STAGES; k < it; ++k)
            {
                if (k < 0) continue;
                mbar_wait(&full[k % DT_STAGES], static_cast<uint32_t>((k / DT_STAGES) & 1),
                          abort_flag + 1);
            }
        }
        __syncwarp();
    }
    else if (warp == 5)
    {
        // MMA issuer: one chunk accumulator per DT_CHUNK stages
        if (lane == 0)
        {
            int64_t it = 0, cc = 0;
            bool ok = true;
            for (int64_t unit = blockIdx.x; unit < ntiles && ok; unit += gridDim.x)
            {
                int64_t k0, k1;
                k_range(unit, k0, k1);
                for (int64_t k = k0; k < k1 && ok; ++k, ++it)
                {
                    const int64_t kc = (k - k0) % DT_CHUNK;
                    if (kc == 0 && cc > 0 &&
                        !mbar_wait(chunk_empty, static_cast<uint32_t>((cc - 1) & 1), abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    const int s = static_cast<int>(it % DT_STAGES);
                    const uint32_t ph = static_cast<uint32_t>((it / DT_STAGES) & 1);
                    if (!mbar_wait(&full[s], ph, abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    unsigned char* st = base + static_cast<size_t>(s) * stage_bytes;
                    const uint64_t ah = tc::smem_desc_sw128(st);
                    const uint64_t al = tc::smem_desc_sw128(st + a_bytes);
                    const uint64_t bh = tc::smem_desc_sw128(st + 2 * a_bytes);
                    const uint64_t bl = tc::smem_desc_sw128(st + 2 * a_bytes + b_bytes);
#pragma unroll
                    for (int kk = 0; kk < DT_BK / 8; ++kk)
                    {
                        // K step kk: 8 TF32 values = 32 bytes further into each row
                        const uint64_t o = static_cast<uint64_t>(kk * 32) >> 4;
                        const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                        tc::mma_tf32_ss(d_chunk, al + o, bh + o, idesc, acc);
                        tc::mma_tf32_ss(d_chunk, ah + o, bl + o, idesc, 1u);
                        tc::mma_tf32_ss(d_chunk, ah + o, bh + o, idesc, 1u);
                    }
                    tc::commit(&empty[s]);
                    if (kc == DT_CHUNK - 1 || k == k1 - 1)
                    {
                        tc::commit(chunk_full);
                        ++cc;
                    }
                }
            }
            // every issued MMA completes before the tensor memory is freed
            tc::commit(drain);
            mbar_wait(drain, 0, abort_flag + 1);
        }
        __syncwarp();
    }
    else
    {
        // warps 0-3: add each chunk into the running total (round to
        // nearest), then the epilogue; thread tid owns tile row tid
        int64_t cc = 0;
        bool ok = true;
        const uint32_t lanes = static_cast<uint32_t>(32 * warp) << 16;
        for (int64_t unit = blockIdx.x; unit < ntiles && ok; unit += gridDim.x)
        {
            const int64_t tile = unit / d.ksplit;
            int64_t k0, k1;
            k_range(unit, k0, k1);
            const int64_t nch_u = (k1 - k0 + DT_CHUNK - 1) / DT_CHUNK;
            for (int64_t ch = 0; ch < nch_u; ++ch, ++cc)
            {
                if (!__all_sync(FULL_MASK,
                                mbar_wait(chunk_full, static_cast<uint32_t>(cc & 1), abort_flag)))
                {
                    if (lane == 0) give_up();
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                for (int c0 = 0; c0 < d.NB; c0 += 16)
                {
                    uint32_t v[16], t[16];
                    tc::ld_x16(d_chunk + lanes + c0, v);
                    if (ch > 0) tc::ld_x16(tmem + lanes + c0, t);
                    tc::wait_ld();
                    if (ch > 0)
                    {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            v[j] = __float_as_uint(__uint_as_float(t[j]) + __uint_as_float(v[j]));
                    }
                    tc::st_x16(tmem + lanes + c0, v);
                }
                tc::wait_st();
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(chunk_empty);
            }
            if (!ok) break;
            tc::fence_after_sync();
            const int64_t row = tile / d.ntn * 128 + tid;
            const int col0 = static_cast<int>(tile % d.ntn) * d.NB;
            const bool live = row < d.M;
            if (d.ksplit > 1)
            {
                // this part's running total; k_dense_epi adds the parts
                float* dst = d.acc + ((unit % d.ksplit) * d.M + row) * d.NB + col0;
                for (int c0 = 0; c0 < d.NB; c0 += 16)
                {
                    uint32_t v[16];
                    tc::ld_x16(tmem + lanes + c0, v);
                    tc::wait_ld();
                    if (live)
                    {
#pragma unroll
                        for (int j = 0; j < 16; ++j) dst[c0 + j] = __uint_as_float(v[j]);
                    }
                }
                tc::fence_before_sync();
                continue;
            }
            for (int c0 = 0; c0 < d.NB; c0 += 16)
            {
                uint32_t v[16];
                tc::ld_x16(tmem + lanes + c0, v);
                tc::wait_ld();
                double add[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    add[j] = 0.0;
                    const int q = col0 + c0 + j;
                    if (!live || q >= d.nb) continue;
                    const int p = d.p_off + q;
                    const int64_t o = row * d.b + p;
                    const double sxv = d.sx ? d.sx[p] : 1.0;
                    const float xv = (d.shift != 0.0 || d.epi == 1) ? d.X[o] : 0.0f;
                    const float zv = d.Z ? d.Z[o] : 0.0f;
                    double y = static_cast<double>(__uint_as_float(v[j])) * sxv;
                    if (d.shift != 0.0) y += d.shift * (sxv * static_cast<double>(xv));
                    if (d.Z) y -= (d.zc[p] * d.zs[p]) * static_cast<double>(zv);
                    const float yr = static_cast<float>(y);
                    d.Y[o] = yr;
                    const double ys = static_cast<double>(yr);
                    if (d.epi == 1) add[j] = (sxv * static_cast<double>(xv)) * ys;
                    else if (d.epi == 2) add[j] = ys * ys;
                    else if (d.epi == 3) add[j] = (d.zs[p] * static_cast<double>(zv)) * ys;
                }
                if (d.epi != 0)
                {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                    {
                        double a = add[j];
#pragma unroll
                        for (int off = 16; off > 0; off >>= 1)
                            a += __shfl_xor_sync(FULL_MASK, a, off);
                        if (lane == 0 && col0 + c0 + j < d.nb)
                            red[warp * 256 + col0 + c0 + j] += a;
                    }
                }
            }
            tc::fence_before_sync();
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
    {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, d.tmem_cols);
    }
    if (d.epi != 0 && d.ksplit == 1)
        for (int q = tid; q < d.nb; q += DT_THREADS)
            d.partials[static_cast<int64_t>(blockIdx.x) * d.b + d.p_off + q] =
                ((red[q] + red[256 + q]) + red[512 + q]) + red[768 + q];
}

// The K parts of a split dense product: Y[r][p] from the ksplit running
// totals (FP32 adds in part order), then the SpMM epilogue of k_dense_tc.
// Block = 256 threads, thread q = probe column q of the chunk; block i takes
// rows [i M / grid, (i + 1) M / grid) in order, so partials[i][p] is a
// fixed-order sum over its rows.
__global__ void __launch_bounds__(256)
k_dense_epi(const DenseArgs d)
{
    const int q = threadIdx.x;
    if (q >= d.nb) return;
    const int p = d.p_off + q;
    const int64_t r0 = d.M * blockIdx.x / gridDim.x;
    const int64_t r1 = d.M * (blockIdx.x + 1) / gridDim.x;
    const double sxv = d.sx ? d.sx[p] : 1.0;
    const double zcs = d.Z ? d.zc[p] * d.zs[p] : 0.0;
    double sum = 0.0;
    for (int64_t row = r0; row < r1; ++row)
    {
        float t = d.acc[row * d.NB + q];
        for (int k = 1; k < d.ksplit; ++k) t += d.acc[(k * d.M + row) * d.NB + q];
        const int64_t o = row * d.b + p;
        const float xv = (d.shift != 0.0 || d.epi == 1) ? d.X[o] : 0.0f;
        const float zv = d.Z ? d.Z[o] : 0.0f;
        double y = static_cast<double>(t) * sxv;
        if (d.shift != 0.0) y += d.shift * (sxv * static_cast<double>(xv));
        if (d.Z) y -= zcs * static_cast<double>(zv);
        const float yr = static_cast<float>(y);
        d.Y[o] = yr;
        const double ys = static_cast<double>(yr);
        if (d.epi == 1) sum += (sxv * static_cast<double>(xv)) * ys;
        else if (d.epi == 2) sum += ys * ys;
        else if (d.epi == 3) sum += (d.zs[p] * static_cast<double>(zv)) * ys;
    }
    if (d.epi != 0) d.partials[static_cast<int64_t>(blockIdx.x) * d.b + p] = sum;
}

// ===========================================================================
// Tensor-core self-test: D[128][16] = A[128][8] B[8][16] for one tile
// through tcgen05 (one CTA of 128 threads; thread m owns row m).  mode:
//   0  A in tensor memory (written by its owning warps), B in shared
//      memory, one kind::tf32 MMA (the tensor-core SpMM's form);
//   1  as 0 with both operands split into TF32 hi/lo, three MMAs;
//   2  tensor-memory round trip: D[m][0..7] / [8..15] = the stored A hi / lo;
//   3  A and B in shared memory, one MMA.
// ===========================================================================

__global__ void __launch_bounds__(128, 1)
k_tc_selftest(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ d,
              int mode, int32_t* __restrict__ error)
{
    __shared__ __align__(1024) unsigned char atile[4096];
    __shared__ __align__(1024) unsigned char btile[2][512];  // B hi, B lo
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ int abort_none;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    if (warp == 0)
    {
        tc::tmem_alloc(&tbase, 64);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        mbar_init(&bar, 1);
        abort_none = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t base = tbase;
    const uint32_t lanes = static_cast<uint32_t>(32 * warp) << 16;
    // tensor-memory columns: A hi 0..7, A lo 8..15, D 32..47
    uint32_t hi[8], lo[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        tc::split_tf32(a[tid * 8 + k], hi[k], lo[k]);
        if (mode == 0 || mode == 3) lo[k] = 0u;
        *reinterpret_cast<uint32_t*>(atile + tc::kmajor_offset(tid, k)) = hi[k];
    }
    tc::st_x8(base + lanes + 0, hi);
    tc::st_x8(base + lanes + 8, lo);
    {
        const int k = tid >> 4;
        const int n = tid & 15;
        uint32_t h, l;
        tc::split_tf32(b[k * 16 + n], h, l);
        *reinterpret_cast<uint32_t*>(btile[0] + tc::kmajor_offset(n, k)) = h;
        *reinterpret_cast<uint32_t*>(btile[1] + tc::kmajor_offset(n, k)) = (mode == 1) ? l : 0u;
    }
    tc::fence_proxy_async_smem();
    tc::wait_st();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t dcol = (mode == 2) ? base : base + 32;
    if (tid == 0)
    {
        const uint64_t bh = tc::smem_desc(btile[0], 128, 256);
        const uint64_t bl = tc::smem_desc(btile[1], 128, 256);
        if (mode == 1)
        {
            tc::mma_tf32_ts(dcol, base + 8, bh, tc::IDESC_TF32_M128_N16, 0);
            tc::mma_tf32_ts(dcol, base + 0, bl, tc::IDESC_TF32_M128_N16, 1);
            tc::mma_tf32_ts(dcol, base + 0, bh, tc::IDESC_TF32_M128_N16, 1);
        }
        else if (mode == 0)
        {
            tc::mma_tf32_ts(dcol, base + 0, bh, tc::IDESC_TF32_M128_N16, 0);
        }
        else if (mode == 3)
        {
            const uint64_t ad = tc::smem_desc(atile, 128, 256);
            tc::mma_tf32_ss(dcol, ad, bh, tc::IDESC_TF32_M128_N16, 0);
        }
        tc::commit(&bar);  // with no MMA issued it arrives at once
    }
    const bool ok = __all_sync(FULL_MASK, mbar_wait(&bar, 0, &abort_none));
    tc::fence_after_sync();
    if (ok)
    {
        uint32_t v[16];
        tc::ld_x16(dcol + lanes, v);
        tc::wait_ld();
#pragma unroll
        for (int n = 0; n < 16; ++n) d[tid * 16 + n] = __uint_as_float(v[n]);
    }
    else if ((tid & 31) == 0)
    {
        atomicExch(error, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(base, 64);
}

// ===========================================================================
// MN-major operand self-test: D[128][32] = A[128][8] B'[8][32] through one
// kind::tf32 MMA with B' MN-major in shared memory.  A TF32 MN-major operand
// takes the 128-byte swizzle with 32-byte atoms (descriptor layout type 1,
// SWIZZLE_128B_BASE32B): atoms of 4 K rows x 128 bytes (32 N values), the
// 32-byte chunk c of row k stored at chunk c ^ (k % 4); the leading byte
// offset is the stride between 32-value N atoms, the stride byte offset the
// stride between 4-row K atoms (here 512: K rows 0-3, then 4-7).  The plain
// 128-byte swizzle (layout type 2) reads an MN-major TF32 operand as zeros.
// gather == 0: the threads write B' = B; gather == 1: two TMA tile::gather4
// loads bring B' rows k = B rows perm[k] (perm = 3 0 7 1 6 2 5 4) through
// bmap (B as [8][32] FP32, box 32 x 1, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
// which writes exactly this layout), the load form of a block SpMM's probe
// rows.  A is K-major without swizzling (as k_tc_selftest mode 3).  One CTA
// of 128 threads; thread m owns row m.
// ===========================================================================

__global__ void __launch_bounds__(128, 1)
k_tc_selftest_mn(const __grid_constant__ CUtensorMap bmap, const float* __restrict__ a,
                 const float* __restrict__ b, float* __restrict__ d, int gather,
                 int32_t* __restrict__ error)
{
    __shared__ __align__(1024) unsigned char atile[4096];
    __shared__ __align__(1024) unsigned char btile[1024];
    __shared__ __align__(8) uint64_t bars[2];  // [0] B loaded, [1] MMA done
    __shared__ uint32_t tbase;
    __shared__ int abort_none;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    if (warp == 0)
    {
        tc::tmem_alloc(&tbase, 32);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        abort_none = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t base = tbase;
    const uint32_t lanes = static_cast<uint32_t>(32 * warp) << 16;
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        uint32_t h, l;
        tc::split_tf32(a[tid * 8 + k], h, l);
        *reinterpret_cast<uint32_t*>(atile + tc::kmajor_offset(tid, k)) = h;
    }
    if (!gather)
    {
        // 256 values, two per thread: (k, n) at (k / 4) * 512 + (k % 4) * 128 +
        // ((n / 8) ^ (k % 4)) * 32 + (n % 8) * 4
        for (int e = tid; e < 256; e += 128)
        {
            const int k = e >> 5, n = e & 31;
            uint32_t h, l;
            tc::split_tf32(b[k * 32 + n], h, l);
            *reinterpret_cast<uint32_t*>(btile + (k >> 2) * 512 + (k & 3) * 128 +
                                         (((n >> 3) ^ (k & 3)) << 5) + (n & 7) * 4) = h;
        }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    bool ok = true;
    if (gather)
    {
        if (tid == 0)
        {
            mbar_expect_tx(&bars[0], 1024u);
            tma_gather4(btile, &bmap, 0, 3, 0, 7, 1, &bars[0]);
            tma_gather4(btile + 512, &bmap, 0, 6, 2, 5, 4, &bars[0]);
        }
        ok = __all_sync(FULL_MASK, mbar_wait(&bars[0], 0, &abort_none));
        ok = __syncthreads_and(ok);
    }
    tc::fence_after_sync();
    if (tid == 0 && ok)
    {
        const uint64_t ad = tc::smem_desc(atile, 128, 256);
        // MN-major, 128-byte swizzle with 32-byte atoms (layout type 1): one
        // N atom, K atoms 512 bytes apart
        const uint64_t bd = tc::smem_desc(btile, 1024, 512) | (uint64_t(1) << 61);
        tc::mma_tf32_ss(base, ad, bd, tc::idesc_tf32_m128(32) | (1u << 16), 0);
    }
    if (tid == 0) tc::commit(&bars[1]);  // with no MMA issued it arrives at once
    ok = __all_sync(FULL_MASK, mbar_wait(&bars[1], 0, &abort_none)) && ok;
    tc::fence_after_sync();
    if (ok)
    {
        uint32_t v[16];
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            tc::ld_x16(base + lanes + 16 * h, v);
            tc::wait_ld();
#pragma unroll
            for (int n = 0; n < 16; ++n) d[tid * 32 + 16 * h + n] = __uint_as_float(v[n]);
        }
    }
    else if ((tid & 31) == 0)
    {
        atomicExch(error, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(base, 32);
}

}  // namespace slq

#endif  // SLQ_KERNELS_CUH_
