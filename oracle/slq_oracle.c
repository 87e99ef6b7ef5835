/*
 * slq_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain-C, single-threaded restatement of the reference CPU stochastic
 * Lanczos quadrature (ameli/imate v0.25.2, imate/_c_trace_estimator/) used as
 * the oracle of the CUDA engine.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg load it.  Each function names the reference
 * file:line it follows.  Arithmetic follows the reference: FP64 data, long
 * double accumulators in inner products, norms and CSR row sums
 * (imate/_c_basic_algebra/c_vector_operations.cpp:223,297,
 * c_matrix_operations.cpp:480).  Probes are drawn exactly as the reference
 * estimator with num_threads=1 draws them, probe i from words
 * [i*(n/64+1), (i+1)*(n/64+1)) of one xoshiro256** stream.
 *
 * Differences from the reference, by design:
 *   - the tridiagonal eigenproblem (LAPACK ?stev in the reference,
 *     diagonalization.cpp:89-118) is solved here by implicit QL in long
 *     double, tracking only the first row of the eigenvector matrix;
 *   - the bidiagonal SVD (?bdsdc, diagonalization.cpp:190-231) is replaced by
 *     the same QL on B^T B, whose eigenvalues are sigma^2 and whose
 *     eigenvectors are the right singular vectors;
 *   - for gram=1 on a rectangular matrix the probe length and the trace scale
 *     are the number of columns (the reference uses the number of rows,
 *     c_trace_estimator.cpp:220,620, which is only right for square A);
 *   - gram=2 (no counterpart in the reference) runs Lanczos on A^T A (+ t I
 *     for affine operators), the operator of the engine's normal-equations
 *     mode.
 * The first two are pinned against the reference's LAPACK results by the
 * tests; the third only changes rectangular inputs, which the reference
 * cannot run.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef long double ld;

/* ------------------------------------------------------------------------ */
/* Random numbers: SplitMix64 seeding and xoshiro256** (Blackman & Vigna),
 * as imate/_random_generator/split_mix_64.cpp:28-64 and
 * xoshiro_256_star_star.cpp:73-133 use them.                               */
/* ------------------------------------------------------------------------ */

typedef struct { uint64_t s[4]; } xoshiro_t;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* split_mix_64.cpp:28-48: state = (seed << 32) | seed; negative seeds use
 * the clock. */
static uint64_t splitmix_next(uint64_t* state)
{
    uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static uint64_t xoshiro_next(xoshiro_t* x)
{
    uint64_t* s = x->s;
    const uint64_t result = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

/* The published 2^128-step jump polynomial of xoshiro256**. */
static void xoshiro_jump(xoshiro_t* x)
{
    static const uint64_t J[4] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL,
                                  0xa9582618e03fc9aaULL, 0x39abdc4529b1661cULL};
    uint64_t acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i)
        for (int b = 0; b < 64; ++b)
        {
            if (J[i] & (1ULL << b))
                for (int k = 0; k < 4; ++k) acc[k] ^= x->s[k];
            xoshiro_next(x);
        }
    memcpy(x->s, acc, sizeof(acc));
}

/* random_number_generator.cpp:120-137 with num_threads = 1: one stream,
 * seeded through SplitMix64 and jumped once. */
static void stream_init(xoshiro_t* x, int64_t seed)
{
    uint64_t s = (seed >= 0) ? (uint64_t)seed : (uint64_t)time(NULL);
    uint64_t st = (s << 32) | s;
    for (int i = 0; i < 4; ++i) x->s[i] = splitmix_next(&st);
    xoshiro_jump(x);
}

/* random_array_generator.cpp:63-165: bit j of word i sets element 64 i + j
 * to +1 (else -1); the tail takes one more word, drawn even when n % 64 == 0. */
static void rademacher_fill(xoshiro_t* x, double* v, int64_t n)
{
    int64_t chunks = n / 64;
    for (int64_t i = 0; i < chunks; ++i)
    {
        uint64_t bits = xoshiro_next(x);
        for (int j = 0; j < 64; ++j)
            v[i * 64 + j] = (bits >> j) & 1ULL ? 1.0 : -1.0;
    }
    uint64_t bits = xoshiro_next(x);
    for (int64_t i = chunks * 64, j = 0; i < n; ++i, ++j)
        v[i] = (bits >> j) & 1ULL ? 1.0 : -1.0;
}

/* ------------------------------------------------------------------------ */
/* Vector kernels (c_vector_operations.cpp)                                 */
/* ------------------------------------------------------------------------ */

static double dot(const double* a, const double* b, int64_t n)
{   /* c_vector_operations.cpp:204-244 (long double accumulator) */
    ld s = 0.0L;
    for (int64_t i = 0; i < n; ++i) s += (ld)a[i] * b[i];
    return (double)s;
}

static double nrm2(const double* a, int64_t n)
{   /* c_vector_operations.cpp:281-321 */
    ld s = 0.0L;
    for (int64_t i = 0; i < n; ++i) s += (ld)a[i] * a[i];
    return sqrt((double)s);
}

static void axmy(const double* x, int64_t n, double scale, double* y)
{   /* subtract_scaled_vector, c_vector_operations.cpp:135-170 */
    if (scale == 0.0) return;
    for (int64_t i = 0; i < n; ++i) y[i] -= scale * x[i];
}

/* ------------------------------------------------------------------------ */
/* Operator: CSR or CSC matrix, optionally A + t I                          */
/* (c_csr_matrix.cpp:138-211, c_matrix_operations.cpp:469-637,             */
/*  c_csr_affine_matrix_function.cpp, c_affine_matrix_function.cpp:136)     */
/* ------------------------------------------------------------------------ */

typedef struct {
    const double* data;
    const int* indices;
    const int* indptr;
    int64_t nrows, ncols;
    int fmt;        /* 0 CSR, 1 CSC */
    int affine;     /* adds t * x */
    double t;
    int normal;     /* operator is A^T A (+ t I): x -> A^T (A x) + t x */
    double* tmp;    /* nrows scratch for the normal operator */
} op_t;

static void op_tdot(const op_t* A, const double* x, double* y);

/* y = A x (+ t x); for the normal operator y = A^T (A x) + t x */
static void op_dot(const op_t* A, const double* x, double* y)
{
    if (A->normal)
    {
        op_t B = *A;
        B.normal = 0;
        B.affine = 0;
        op_dot(&B, x, A->tmp);
        op_tdot(&B, A->tmp, y);
        if (A->affine && A->t != 0.0)
            for (int64_t c = 0; c < A->ncols; ++c) y[c] += A->t * x[c];
        return;
    }
    if (A->fmt == 0)
    {
        for (int64_t r = 0; r < A->nrows; ++r)
        {
            ld s = 0.0L;
            for (int k = A->indptr[r]; k < A->indptr[r + 1]; ++k)
                s += (ld)A->data[k] * x[A->indices[k]];
            y[r] = (double)s;
        }
    }
    else
    {   /* CSC: scatter over columns, c_matrix_operations.cpp csc_matvec */
        for (int64_t r = 0; r < A->nrows; ++r) y[r] = 0.0;
        for (int64_t c = 0; c < A->ncols; ++c)
            for (int k = A->indptr[c]; k < A->indptr[c + 1]; ++k)
                y[A->indices[k]] += A->data[k] * x[c];
    }
    if (A->affine && A->t != 0.0)
        for (int64_t r = 0; r < A->nrows; ++r) y[r] += A->t * x[r];
}

/* y = A^T x (+ t x) */
static void op_tdot(const op_t* A, const double* x, double* y)
{
    if (A->fmt == 0)
    {
        for (int64_t c = 0; c < A->ncols; ++c) y[c] = 0.0;
        for (int64_t r = 0; r < A->nrows; ++r)
            for (int k = A->indptr[r]; k < A->indptr[r + 1]; ++k)
                y[A->indices[k]] += A->data[k] * x[r];
    }
    else
    {
        for (int64_t c = 0; c < A->ncols; ++c)
        {
            ld s = 0.0L;
            for (int k = A->indptr[c]; k < A->indptr[c + 1]; ++k)
                s += (ld)A->data[k] * x[A->indices[k]];
            y[c] = (double)s;
        }
    }
    if (A->affine && A->t != 0.0)
        for (int64_t c = 0; c < A->ncols; ++c) y[c] += A->t * x[c];
}

/* ------------------------------------------------------------------------ */
/* Gram-Schmidt against a ring buffer (c_orthogonalization.cpp:125-224)     */
/* ------------------------------------------------------------------------ */

static void gram_schmidt(const double* V, int64_t n, int num_vectors,
                         int last_vector, int num_ortho, double* v)
{
    int num_steps;
    if (num_ortho == 0 || num_vectors < 2) return;
    if (num_ortho < 0 || num_ortho > num_vectors) num_steps = num_vectors;
    else num_steps = num_ortho;
    if ((int64_t)num_steps > n) num_steps = (int)n;
    const double eps = 2.220446049250313e-16;
    for (int step = 0; step < num_steps; ++step)
    {
        int lv = last_vector % num_vectors;
        int i = (lv >= step) ? lv - step : lv - step + num_vectors;
        const double* Vi = V + (int64_t)i * n;
        double norm = nrm2(Vi, n);
        if (norm < eps * sqrt((double)n)) continue;
        double ip = dot(Vi, v, n);
        double scale = ip / (norm * norm);
        if (fabs(fabs(scale) - 1.0) <= 2.0 * eps)
        {
            double nv = nrm2(v, n);
            double d2 = nv * nv - 2.0 * ip + norm * norm;
            if (d2 < 2.0 * eps * n) continue;
        }
        axmy(Vi, n, scale, v);
    }
}

/* ------------------------------------------------------------------------ */
/* Lanczos tridiagonalization (c_lanczos_tridiagonalization.cpp:117-236)    */
/* ------------------------------------------------------------------------ */

static int lanczos(const op_t* A, const double* v, int64_t n, int m,
                   double tol, int orthogonalize, double* alpha, double* beta)
{
    int bs;
    if (orthogonalize == 0 || orthogonalize == 1) bs = 2;
    else if (orthogonalize < 0 || orthogonalize > m) bs = m;
    else bs = orthogonalize;
    double* V = (double*)malloc(sizeof(double) * n * bs);
    double* r = (double*)malloc(sizeof(double) * n);
    memcpy(r, v, sizeof(double) * n);
    double beta0 = nrm2(r, n);
    int size = 0;
    for (int j = 0; j < m; ++j)
    {
        ++size;
        double* Vj = V + (int64_t)(j % bs) * n;
        double s = 1.0 / (j == 0 ? beta0 : beta[j - 1]);
        for (int64_t i = 0; i < n; ++i) Vj[i] = s * r[i];
        op_dot(A, Vj, r);
        alpha[j] = dot(Vj, r, n);
        axmy(Vj, n, alpha[j], r);
        if (j > 0) axmy(V + (int64_t)((j - 1) % bs) * n, n, beta[j - 1], r);
        if (orthogonalize != 0)
        {
            int no = (j < bs) ? j + 1 : bs;
            gram_schmidt(V, n, bs, j % bs, no, r);
        }
        beta[j] = nrm2(r, n);
        if (beta[j] < tol * sqrt((double)n)) break;
    }
    free(V);
    free(r);
    return size;
}

/* ------------------------------------------------------------------------ */
/* Golub-Kahn bidiagonalization (c_golub_kahn_bidiagonalization.cpp:        */
/* 111-232), on an nr x nc operator with a start vector of length nc.       */
/* ------------------------------------------------------------------------ */

static double normalize(double* x, int64_t n)
{   /* normalize_vector_in_place, c_vector_operations.cpp:330-360 */
    double nr = nrm2(x, n);
    for (int64_t i = 0; i < n; ++i) x[i] /= nr;
    return nr;
}

static int golub_kahn(const op_t* A, const double* v, int m, double tol,
                      int orthogonalize, double* alpha, double* beta)
{
    int64_t nr = A->nrows, nc = A->ncols;
    int bs;
    if (orthogonalize == 0) bs = 2;
    else if (orthogonalize < 0 || orthogonalize > m - 1) bs = m;
    else bs = orthogonalize + 1;
    double* U = (double*)malloc(sizeof(double) * nr * bs);
    double* V = (double*)malloc(sizeof(double) * nc * bs);
    double nv = nrm2(v, nc);
    for (int64_t i = 0; i < nc; ++i) V[i] = v[i] / nv;
    int size = 0;
    int no = 0;
    for (int j = 0; j < m; ++j)
    {
        ++size;
        double* Uj = U + (int64_t)(j % bs) * nr;
        double* Vj = V + (int64_t)(j % bs) * nc;
        double* Vn = V + (int64_t)((j + 1) % bs) * nc;
        op_dot(A, Vj, Uj);
        if (j > 0) axmy(U + (int64_t)((j - 1) % bs) * nr, nr, beta[j - 1], Uj);
        if (orthogonalize != 0)
        {
            no = (j < bs) ? j : bs - 1;
            if (j > 0) gram_schmidt(U, nr, bs, (j - 1) % bs, no, Uj);
        }
        alpha[j] = normalize(Uj, nr);
        op_tdot(A, Uj, Vn);
        axmy(Vj, nc, alpha[j], Vn);
        if (orthogonalize != 0) gram_schmidt(V, nc, bs, j % bs, no, Vn);
        beta[j] = normalize(Vn, nc);
        if (beta[j] < tol * sqrt((double)nc)) break;
    }
    free(U);
    free(V);
    return size;
}

/* ------------------------------------------------------------------------ */
/* Symmetric tridiagonal eigenproblem by implicit QL with Wilkinson shifts   */
/* (Wilkinson & Reinsch / Golub & Van Loan 8.3), tracking only the first    */
/* row of the eigenvector matrix.  d[0..k-1] diagonal, e[0..k-2] off-       */
/* diagonal; on return d holds the eigenvalues and z[i] the first component */
/* of the i-th unit eigenvector.  Returns 0, or 1 if a QL sweep did not     */
/* converge in 60 iterations.                                               */
/* ------------------------------------------------------------------------ */

static int tridiag_ql(ld* d, ld* e, ld* z, int k)
{
    for (int i = 0; i < k; ++i) z[i] = (i == 0) ? 1.0L : 0.0L;
    if (k <= 1) return 0;
    e[k - 1] = 0.0L;
    const ld eps = 1.0842021724855044e-19L; /* 2^-63 */
    for (int l = 0; l < k; ++l)
    {
        int iter = 0;
        for (;;)
        {
            int mm;
            for (mm = l; mm < k - 1; ++mm)
            {
                ld dd = fabsl(d[mm]) + fabsl(d[mm + 1]);
                if (fabsl(e[mm]) <= eps * dd) break;
            }
            if (mm == l) break;
            if (++iter > 60) return 1;
            ld g = (d[l + 1] - d[l]) / (2.0L * e[l]);
            ld r = hypotl(g, 1.0L);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            ld s = 1.0L, c = 1.0L, p = 0.0L;
            int i;
            int deflated = 0;
            for (i = mm - 1; i >= l; --i)
            {
                ld f = s * e[i];
                ld b = c * e[i];
                r = hypotl(f, g);
                e[i + 1] = r;
                if (r == 0.0L)
                {
                    d[i + 1] -= p;
                    e[mm] = 0.0L;
                    deflated = 1;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0L * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                ld zf = z[i + 1];
                z[i + 1] = s * z[i] + c * zf;
                z[i] = c * z[i] - s * zf;
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0L;
        }
    }
    return 0;
}

/* Nodes and weights of one sample (c_trace_estimator.cpp:511-555):
 * Lanczos: theta = eig(T), tau = first eigenvector entries.
 * Golub-Kahn: theta = sigma^2 of upper-bidiagonal B(alpha, beta),
 * tau = first entries of the right singular vectors. */
static int nodes_weights(const double* alpha, const double* beta, int k,
                         int gram, double* theta, double* tau)
{
    ld* d = (ld*)malloc(sizeof(ld) * (k + 1));
    ld* e = (ld*)malloc(sizeof(ld) * (k + 1));
    ld* z = (ld*)malloc(sizeof(ld) * (k + 1));
    for (int i = 0; i < k; ++i)
    {
        if (gram)
        {   /* B^T B for B = diag(alpha) + superdiag(beta[0..k-2]) */
            ld a = alpha[i];
            ld bp = (i > 0) ? (ld)beta[i - 1] : 0.0L;
            d[i] = a * a + bp * bp;
            e[i] = (i < k - 1) ? a * (ld)beta[i] : 0.0L;
        }
        else
        {
            d[i] = alpha[i];
            e[i] = (i < k - 1) ? (ld)beta[i] : 0.0L;
        }
    }
    int info = tridiag_ql(d, e, z, k);
    for (int i = 0; i < k; ++i)
    {
        theta[i] = (double)d[i];
        tau[i] = (double)z[i];
    }
    free(d);
    free(e);
    free(z);
    return info;
}

/* ------------------------------------------------------------------------ */
/* Inverse error function.  Initial guess from Winitzki's closed form       */
/* (S. Winitzki, "A handy approximation for the error function and its      */
/* inverse", 2008, a = 0.147), refined by Newton steps on erf.              */
/* ------------------------------------------------------------------------ */

double oracle_erfinv(double x)
{
    if (x >= 1.0) return INFINITY;
    if (x <= -1.0) return -INFINITY;
    if (x == 0.0) return 0.0;
    const double a = 0.147;
    const double pi = 3.14159265358979323846;
    double ln = log(1.0 - x * x);
    double t = 2.0 / (pi * a) + ln / 2.0;
    double y = sqrt(sqrt(t * t - ln / a) - t);
    if (x < 0) y = -y;
    for (int it = 0; it < 8; ++it)
    {
        double step = (erf(y) - x) / (2.0 / sqrt(pi) * exp(-y * y));
        y -= step;
        if (fabs(step) <= 1e-17 * fabs(y)) break;
    }
    return y;
}

/* ------------------------------------------------------------------------ */
/* Convergence test after each processed sample (convergence_tools.cpp:     */
/* 95-194).  samples is [max][q] row-major; order lists processed rows.     */
/* ------------------------------------------------------------------------ */

static int check_convergence(const double* samples, int q, int min_s,
                             const int* order, int nproc, double conf,
                             double atol, double rtol, double* error,
                             int* used, int* converged)
{
    if (nproc < min_s)
    {
        for (int j = 0; j < q; ++j)
        {
            error[j] = INFINITY;
            converged[j] = 0;
            used[j] = nproc;
        }
        return 0;
    }
    double z = sqrt(2.0) * oracle_erfinv(conf);
    for (int j = 0; j < q; ++j)
    {
        if (converged[j]) continue;
        double sum = 0.0;
        for (int i = 0; i < nproc; ++i) sum += samples[(int64_t)order[i] * q + j];
        double mean = sum / nproc;
        double sd;
        if (nproc > 1)
        {
            sum = 0.0;
            for (int i = 0; i < nproc; ++i)
            {
                double dv = samples[(int64_t)order[i] * q + j] - mean;
                sum += dv * dv;
            }
            sd = sqrt(sum / (nproc - 1.0));
        }
        else
            sd = INFINITY;
        error[j] = z * sd / sqrt((double)nproc);
        double thr = rtol * mean;
        if (atol > thr) thr = atol;
        if (error[j] < thr) converged[j] = 1;
        used[j] = nproc;
    }
    for (int j = 0; j < q; ++j)
        if (!converged[j]) return 0;
    return 1;
}

/* Outlier removal and final mean/error (convergence_tools.cpp:256-376). */
static void average_estimates(double conf, double outlier_sig, int q,
                              int max_s, const int* used, const int* order,
                              const double* samples, int* num_outliers,
                              double* trace, double* error)
{
    char* out = (char*)malloc(max_s > 0 ? max_s : 1);
    double ez = sqrt(2.0) * oracle_erfinv(conf);
    double oz = sqrt(2.0) * oracle_erfinv(1.0 - outlier_sig);
    for (int j = 0; j < q; ++j)
    {
        memset(out, 0, max_s > 0 ? max_s : 1);
        num_outliers[j] = 0;
        int nu = used[j];
        double sum = 0.0;
        for (int i = 0; i < nu; ++i) sum += samples[(int64_t)order[i] * q + j];
        double mean = sum / nu;
        double sd;
        if (nu > 1)
        {
            sum = 0.0;
            for (int i = 0; i < nu; ++i)
            {
                double dv = samples[(int64_t)order[i] * q + j] - mean;
                sum += dv * dv;
            }
            sd = sqrt(sum / (nu - 1.0));
        }
        else
            sd = INFINITY;
        double half = oz * sd;
        for (int i = 0; i < nu; ++i)
        {
            double dv = samples[(int64_t)order[i] * q + j] - mean;
            if (fabs(dv) > half)
            {
                out[i] = 1;
                num_outliers[j] += 1;
            }
        }
        sum = 0.0;
        for (int i = 0; i < nu; ++i)
            if (!out[i]) sum += samples[(int64_t)order[i] * q + j];
        mean = sum / (nu - num_outliers[j]);
        if (nu > 1 + num_outliers[j])
        {
            sum = 0.0;
            for (int i = 0; i < nu; ++i)
                if (!out[i])
                {
                    double dv = samples[(int64_t)order[i] * q + j] - mean;
                    sum += dv * dv;
                }
            sd = sqrt(sum / (nu - num_outliers[j] - 1.0));
        }
        else
            sd = INFINITY;
        trace[j] = mean;
        error[j] = ez * sd / sqrt((double)(nu - num_outliers[j]));
    }
    free(out);
}

static double apply_function(int func_id, double x, const double* c)
{   /* functions/logarithm.cpp, inverse.cpp:41, identity.cpp:41,
     * exponential.cpp:55-58, homographic.cpp:63-75, indicator.cpp:62-72,
     * gaussian.cpp:65-69, smoothstep.cpp:55-58 */
    switch (func_id)
    {
        case 0: return log(x);
        case 1: return 1.0 / x;
        case 3: return exp(x * c[0]);
        case 4: return (c[0] * x + c[1]) / (c[2] * x + c[3]);
        case 5: return (x < c[0] || x > c[1]) ? 0.0 : 1.0;
        case 6:
        {
            double u = (x - c[0]) / c[1];
            /* 0.5 * M_SQRT1_2 * M_2_SQRTPI / sigma = 1 / (sigma sqrt(2 pi)) */
            return (0.5 * 0.70710678118654752440 * 1.12837916709551257390 /
                    c[1]) * exp(-0.5 * u * u);
        }
        case 7: return 0.5 * (1.0 + tanh(c[0] * x));
        default: return x;
    }
}

/* ------------------------------------------------------------------------ */
/* Exported entry points (ctypes)                                           */
/* ------------------------------------------------------------------------ */

/* Probe vectors of the single-thread reference estimator, in order. */
void oracle_random_probes(int64_t seed, int64_t n, int num_probes, double* out)
{
    xoshiro_t x;
    stream_init(&x, seed);
    for (int p = 0; p < num_probes; ++p) rademacher_fill(&x, out + (int64_t)p * n, n);
}

/* Raw xoshiro256** words of the stream (after the single jump). */
void oracle_stream_words(int64_t seed, int64_t count, uint64_t* out)
{
    xoshiro_t x;
    stream_init(&x, seed);
    for (int64_t i = 0; i < count; ++i) out[i] = xoshiro_next(&x);
}

/* gram: 0 Lanczos on A, 1 Golub-Kahn on A, 2 Lanczos on A^T A (+ t I). */
int oracle_krylov(const double* data, const int* indices, const int* indptr,
                  int64_t nrows, int64_t ncols, int fmt, int affine, double t,
                  int gram, const double* v, int m, double tol,
                  int orthogonalize, double* alpha, double* beta)
{
    op_t A = {data, indices, indptr, nrows, ncols, fmt, affine, t, 0, NULL};
    if (gram == 1) return golub_kahn(&A, v, m, tol, orthogonalize, alpha, beta);
    if (gram == 2)
    {
        A.normal = 1;
        A.tmp = (double*)malloc(sizeof(double) * nrows);
        int k = lanczos(&A, v, ncols, m, tol, orthogonalize, alpha, beta);
        free(A.tmp);
        return k;
    }
    return lanczos(&A, v, nrows, m, tol, orthogonalize, alpha, beta);
}

int oracle_nodes_weights(const double* alpha, const double* beta, int k,
                         int gram, double* theta, double* tau)
{
    return nodes_weights(alpha, beta, k, gram, theta, tau);
}

int oracle_check_convergence(const double* samples, int q, int min_s,
                             const int* order, int nproc, double conf,
                             double atol, double rtol, double* error,
                             int* used, int* converged)
{
    return check_convergence(samples, q, min_s, order, nproc, conf, atol,
                             rtol, error, used, converged);
}

void oracle_average_estimates(double conf, double outlier_sig, int q,
                              int max_s, const int* used, const int* order,
                              const double* samples, int* num_outliers,
                              double* trace, double* error)
{
    average_estimates(conf, outlier_sig, q, max_s, used, order, samples,
                      num_outliers, trace, error);
}

/* Whole estimator, single thread, samples processed in order
 * (c_trace_estimator.cpp:192-307 with num_threads = 1, and
 * _c_stochastic_lanczos_quadrature :411-654).  With affine = 1 the operator
 * is A + t I, run once at t = params[0] and shifted to the other inquiries
 * (c_trace_estimator.cpp:564-593, c_affine_matrix_function.cpp:98-113).
 * lanczos_sizes (optional) receives each processed sample's Krylov size;
 * alphas / betas (optional, [max_s][m]) the per-sample coefficients. */
int oracle_trace_estimator(
        const double* data, const int* indices, const int* indptr,
        int64_t nrows, int64_t ncols, int fmt, int affine,
        const double* params, int q, int func_id, const double* func_coeff,
        int gram, double exponent, int orthogonalize, int64_t seed, int m,
        double tol, int min_s,
        int max_s, double atol, double rtol, double conf, double outlier_sig,
        double* trace, double* error, double* samples, int* order, int* used,
        int* num_outliers, int* converged, int* lanczos_sizes,
        double* alphas, double* betas)
{
    int64_t n = gram ? ncols : nrows;
    op_t A = {data, indices, indptr, nrows, ncols, fmt, affine,
              affine ? params[0] : 0.0, gram == 2, NULL};
    if (gram == 2) A.tmp = (double*)malloc(sizeof(double) * nrows);
    xoshiro_t x;
    stream_init(&x, seed);
    double* v = (double*)malloc(sizeof(double) * n);
    double* alpha = (double*)malloc(sizeof(double) * m);
    double* beta = (double*)malloc(sizeof(double) * m);
    double* theta = (double*)malloc(sizeof(double) * m);
    double* tau = (double*)malloc(sizeof(double) * m);
    for (int64_t i = 0; i < (int64_t)max_s * q; ++i) samples[i] = NAN;
    for (int j = 0; j < q; ++j)
    {
        converged[j] = 0;
        used[j] = 0;
        num_outliers[j] = 0;
    }
    int nproc = 0, all = 0, status = 0;
    for (int s = 0; s < max_s && !all; ++s)
    {
        rademacher_fill(&x, v, n);
        int k;
        if (gram == 1) k = golub_kahn(&A, v, m, tol, orthogonalize, alpha, beta);
        else k = lanczos(&A, v, n, m, tol, orthogonalize, alpha, beta);
        if (lanczos_sizes) lanczos_sizes[s] = k;
        if (alphas) memcpy(alphas + (int64_t)s * m, alpha, sizeof(double) * k);
        if (betas) memcpy(betas + (int64_t)s * m, beta, sizeof(double) * k);
        if (nodes_weights(alpha, beta, k, gram == 1, theta, tau) != 0) status = 2;
        if (affine && q > 1)
            for (int j = 0; j < q; ++j) converged[j] = 0;
        for (int j = 0; j < q; ++j)
        {
            if (converged[j]) continue;
            double acc = 0.0;
            for (int i = 0; i < k; ++i)
            {
                double th = (affine && j > 0) ? theta[i] - params[0] + params[j]
                                              : theta[i];
                acc += tau[i] * tau[i] *
                       apply_function(func_id, pow(th, exponent), func_coeff);
            }
            samples[(int64_t)s * q + j] = (double)n * acc;
        }
        order[nproc++] = s;
        all = check_convergence(samples, q, min_s, order, nproc, conf, atol,
                                rtol, error, used, converged);
    }
    average_estimates(conf, outlier_sig, q, max_s, used, order, samples,
                      num_outliers, trace, error);
    free(A.tmp);
    free(v);
    free(alpha);
    free(beta);
    free(theta);
    free(tau);
    return status ? -status : all;
}
