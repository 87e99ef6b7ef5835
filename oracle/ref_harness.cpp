// Test infrastructure only: a thin C entry layer around the reference's own
// CPU SLQ sources (ameli/imate v0.25.2), compiled from where they lie by
// oracle/Makefile into oracle/_ref/libimate_ref.so.  Nothing in the product
// links or loads this file; tests/, __graft_entry__.smoke() and bench.py's
// reference arm use it to check the engine and as the timed CPU baseline.
//
// The reference binds LAPACK through Cython (`lapack_api.pxi`, which exports
// lapack_dstev / lapack_dbdsdc from scipy.linalg.cython_lapack).  Here the
// same four symbols are defined as trampolines to function pointers that the
// Python loader fills from scipy.linalg.cython_lapack's capsules, so the
// eigen-solves run on exactly the LAPACK build the reference uses.

#include <cstdint>
#include <cstring>
#include <cmath>
#include <omp.h>

#include "_definitions/types.h"
#include "_c_linear_operator/c_linear_operator.h"
#include "_c_linear_operator/c_csr_matrix.h"
#include "_c_linear_operator/c_csc_matrix.h"
#include "_c_linear_operator/c_csr_affine_matrix_function.h"
#include "_c_linear_operator/c_csc_affine_matrix_function.h"
#include "_c_linear_operator/c_dense_matrix.h"
#include "_c_linear_operator/c_dense_affine_matrix_function.h"
#include "_c_trace_estimator/c_trace_estimator.h"
#include "_c_trace_estimator/c_lanczos_tridiagonalization.h"
#include "_c_trace_estimator/c_golub_kahn_bidiagonalization.h"
#include "_c_trace_estimator/diagonalization.h"
#include "_c_trace_estimator/convergence_tools.h"
#include "_random_generator/random_number_generator.h"
#include "_random_generator/random_array_generator.h"
#include "functions/functions.h"
#include "functions/logarithm.h"
#include "functions/inverse.h"
#include "functions/identity.h"
#include "functions/exponential.h"
#include "functions/homographic.h"
#include "functions/indicator.h"
#include "functions/gaussian.h"
#include "functions/smoothstep.h"

// ---------------------------------------------------------------------------
// LAPACK trampolines (signatures of lapack_api.h)
// ---------------------------------------------------------------------------

typedef void (*stev_d_t)(char*, int*, double*, double*, double*, int*,
                         double*, int*);
typedef void (*stev_s_t)(char*, int*, float*, float*, float*, int*, float*,
                         int*);
typedef void (*bdsdc_d_t)(char*, char*, int*, double*, double*, double*, int*,
                          double*, int*, double*, int*, double*, int*, int*);
typedef void (*bdsdc_s_t)(char*, char*, int*, float*, float*, float*, int*,
                          float*, int*, float*, int*, float*, int*, int*);

static stev_d_t g_dstev = nullptr;
static stev_s_t g_sstev = nullptr;
static bdsdc_d_t g_dbdsdc = nullptr;
static bdsdc_s_t g_sbdsdc = nullptr;

extern "C" {

void lapack_sstev(char* jobz, int* n, float* d, float* e, float* z, int* ldz,
                  float* work, int* info)
{
    g_sstev(jobz, n, d, e, z, ldz, work, info);
}

void lapack_dstev(char* jobz, int* n, double* d, double* e, double* z,
                  int* ldz, double* work, int* info)
{
    g_dstev(jobz, n, d, e, z, ldz, work, info);
}

void lapack_sbdsdc(char* uplo, char* compq, int* n, float* d, float* e,
                   float* u, int* ldu, float* vt, int* ldvt, float* q,
                   int* iq, float* work, int* iwork, int* info)
{
    g_sbdsdc(uplo, compq, n, d, e, u, ldu, vt, ldvt, q, iq, work, iwork, info);
}

void lapack_dbdsdc(char* uplo, char* compq, int* n, double* d, double* e,
                   double* u, int* ldu, double* vt, int* ldvt, double* q,
                   int* iq, double* work, int* iwork, int* info)
{
    g_dbdsdc(uplo, compq, n, d, e, u, ldu, vt, ldvt, q, iq, work, iwork, info);
}

int ref_set_lapack(void* dstev, void* sstev, void* dbdsdc, void* sbdsdc)
{
    g_dstev = reinterpret_cast<stev_d_t>(dstev);
    g_sstev = reinterpret_cast<stev_s_t>(sstev);
    g_dbdsdc = reinterpret_cast<bdsdc_d_t>(dbdsdc);
    g_sbdsdc = reinterpret_cast<bdsdc_s_t>(sbdsdc);
    return (g_dstev && g_sstev && g_dbdsdc && g_sbdsdc) ? 0 : 1;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

// fmt: 0 = CSR, 1 = CSC, 2 = dense row-major (data only; c_dense_matrix.cpp
// and c_dense_affine_matrix_function.cpp).  affine: the A + t I operator.
template <typename T>
static cLinearOperator<T>* make_operator(
        const T* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int fmt, int affine)
{
    if (fmt == 2)
    {
        if (affine)
            return new cDenseAffineMatrixFunction<T>(data, 1, num_rows,
                                                     num_cols);
        return new cDenseMatrix<T>(data, num_rows, num_cols, 1);
    }
    const LongIndexType* ind = reinterpret_cast<const LongIndexType*>(indices);
    const LongIndexType* ptr = reinterpret_cast<const LongIndexType*>(indptr);
    if (fmt == 0)
    {
        if (affine)
            return new cCSRAffineMatrixFunction<T>(data, ind, ptr, num_rows,
                                                   num_cols);
        return new cCSRMatrix<T>(data, ind, ptr, num_rows, num_cols);
    }
    if (affine)
        return new cCSCAffineMatrixFunction<T>(data, ind, ptr, num_rows,
                                               num_cols);
    return new cCSCMatrix<T>(data, ind, ptr, num_rows, num_cols);
}

// The reference's function objects (functions/*.cpp) with coefficients c.
static Function* make_function(int func_id, const double* c)
{
    switch (func_id)
    {
        case 0: return new Logarithm();
        case 1: return new Inverse();
        case 3: return new Exponential(c[0]);
        case 4: return new Homographic(c[0], c[1], c[2], c[3]);
        case 5: return new Indicator(c[0], c[1]);
        case 6: return new Gaussian(c[0], c[1]);
        case 7: return new SmoothStep(c[0]);
        default: return new Identity();
    }
}

template <typename T>
static int run_trace_estimator(
        const T* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int fmt, int affine,
        T* parameters, int num_inquiries, int func_id, const double* coeff,
        int gram, T exponent,
        int orthogonalize, int64_t seed, int lanczos_degree, T lanczos_tol,
        int min_num_samples, int max_num_samples, T error_atol, T error_rtol,
        T confidence_level, T outlier_significance_level, int num_threads,
        T* trace, T* error, T* samples /* [max][q] row-major */,
        int* processed_samples_indices, int* num_samples_used,
        int* num_outliers, int* converged, float* alg_wall_time)
{
    cLinearOperator<T>* A = make_operator<T>(data, indices, indptr, num_rows,
                                             num_cols, fmt, affine);
    Function* f = make_function(func_id, coeff);
    T** rows = new T*[max_num_samples];
    for (int i = 0; i < max_num_samples * num_inquiries; ++i)
        samples[i] = NAN;
    for (int i = 0; i < max_num_samples; ++i)
        rows[i] = &samples[static_cast<int64_t>(i) * num_inquiries];
    for (int j = 0; j < num_inquiries; ++j)
    {
        converged[j] = 0;
        num_samples_used[j] = 0;
        num_outliers[j] = 0;
    }
    float wall = 0.0f;
    int all_converged = cTraceEstimator<T>::c_trace_estimator(
            A, parameters, num_inquiries, f, gram, exponent, orthogonalize,
            seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_threads, trace, error, rows,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, wall);
    *alg_wall_time = wall;
    delete[] rows;
    delete f;
    delete A;
    return all_converged;
}

// A + t B with a general CSR B (c_csr_affine_matrix_function.cpp:55-79):
// the reference runs a Krylov sequence per inquiry on each probe.
template <typename T>
static int run_trace_estimator_b(
        const T* data, const int* indices, const int* indptr,
        const T* b_data, const int* b_indices, const int* b_indptr,
        int64_t num_rows, int64_t num_cols, T* parameters, int num_inquiries,
        int func_id, const double* coeff, int gram, T exponent,
        int orthogonalize, int64_t seed, int lanczos_degree, T lanczos_tol,
        int min_num_samples, int max_num_samples, T error_atol, T error_rtol,
        T confidence_level, T outlier_significance_level, int num_threads,
        T* trace, T* error, T* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    cLinearOperator<T>* A = new cCSRAffineMatrixFunction<T>(
            data, reinterpret_cast<const LongIndexType*>(indices),
            reinterpret_cast<const LongIndexType*>(indptr), num_rows, num_cols,
            b_data, reinterpret_cast<const LongIndexType*>(b_indices),
            reinterpret_cast<const LongIndexType*>(b_indptr));
    Function* f = make_function(func_id, coeff);
    T** rows = new T*[max_num_samples];
    for (int i = 0; i < max_num_samples * num_inquiries; ++i)
        samples[i] = NAN;
    for (int i = 0; i < max_num_samples; ++i)
        rows[i] = &samples[static_cast<int64_t>(i) * num_inquiries];
    for (int j = 0; j < num_inquiries; ++j)
    {
        converged[j] = 0;
        num_samples_used[j] = 0;
        num_outliers[j] = 0;
    }
    float wall = 0.0f;
    int all_converged = cTraceEstimator<T>::c_trace_estimator(
            A, parameters, num_inquiries, f, gram, exponent, orthogonalize,
            seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_threads, trace, error, rows,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, wall);
    *alg_wall_time = wall;
    delete[] rows;
    delete f;
    delete A;
    return all_converged;
}

extern "C" {

int ref_trace_estimator_b_f64(
        const double* data, const int* indices, const int* indptr,
        const double* b_data, const int* b_indices, const int* b_indptr,
        int64_t num_rows, int64_t num_cols, double* parameters,
        int num_inquiries, int func_id, const double* coeff, int gram,
        double exponent, int orthogonalize, int64_t seed, int lanczos_degree,
        double lanczos_tol, int min_num_samples, int max_num_samples,
        double error_atol, double error_rtol, double confidence_level,
        double outlier_significance_level, int num_threads, double* trace,
        double* error, double* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    return run_trace_estimator_b<double>(
            data, indices, indptr, b_data, b_indices, b_indptr, num_rows,
            num_cols, parameters, num_inquiries, func_id, coeff, gram,
            exponent, orthogonalize, seed, lanczos_degree, lanczos_tol,
            min_num_samples, max_num_samples, error_atol, error_rtol,
            confidence_level, outlier_significance_level, num_threads, trace,
            error, samples, processed_samples_indices, num_samples_used,
            num_outliers, converged, alg_wall_time);
}

// Full reference estimator (c_trace_estimator.cpp:192-307) on a CSR, CSC or
// dense row-major matrix, or on A + t I when affine != 0.
int ref_trace_estimator_f64(
        const double* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int fmt, int affine,
        double* parameters, int num_inquiries, int func_id, const double* coeff,
        int gram, double exponent, int orthogonalize, int64_t seed,
        int lanczos_degree,
        double lanczos_tol, int min_num_samples, int max_num_samples,
        double error_atol, double error_rtol, double confidence_level,
        double outlier_significance_level, int num_threads, double* trace,
        double* error, double* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    return run_trace_estimator<double>(
            data, indices, indptr, num_rows, num_cols, fmt, affine,
            parameters, num_inquiries, func_id, coeff, gram, exponent,
            orthogonalize,
            seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_threads, trace, error, samples,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, alg_wall_time);
}

int ref_trace_estimator_f32(
        const float* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int fmt, int affine,
        float* parameters, int num_inquiries, int func_id, const double* coeff,
        int gram, float exponent, int orthogonalize, int64_t seed,
        int lanczos_degree,
        float lanczos_tol, int min_num_samples, int max_num_samples,
        float error_atol, float error_rtol, float confidence_level,
        float outlier_significance_level, int num_threads, float* trace,
        float* error, float* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    return run_trace_estimator<float>(
            data, indices, indptr, num_rows, num_cols, fmt, affine,
            parameters, num_inquiries, func_id, coeff, gram, exponent,
            orthogonalize,
            seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_threads, trace, error, samples,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, alg_wall_time);
}

// Rademacher probes exactly as the single-thread estimator draws them:
// RandomNumberGenerator(1, seed) then generate_random_array per probe
// (random_array_generator.cpp:63-165, c_trace_estimator.cpp:235,449).
void ref_random_probes(int64_t seed, int64_t n, int num_probes, double* out)
{
    RandomNumberGenerator rng(1, seed);
    for (int p = 0; p < num_probes; ++p)
        RandomArrayGenerator<double>::generate_random_array(
                rng, &out[static_cast<int64_t>(p) * n],
                static_cast<LongIndexType>(n), 0);
}

// One Lanczos tridiagonalization (c_lanczos_tridiagonalization.cpp:117-236)
// or Golub-Kahn bidiagonalization (c_golub_kahn_bidiagonalization.cpp:
// 111-232) from a given start vector.  For affine operators the parameter t
// is set before the run.  Returns lanczos_size.
int ref_krylov_f64(const double* data, const int* indices, const int* indptr,
                   int64_t num_rows, int64_t num_cols, int fmt, int affine,
                   double t, int gram, const double* v, int m, double tol,
                   int orthogonalize, double* alpha, double* beta)
{
    cLinearOperator<double>* A = make_operator<double>(
            data, indices, indptr, num_rows, num_cols, fmt, affine);
    if (affine)
        A->set_parameters(&t);
    int size;
    if (gram)
        size = c_golub_kahn_bidiagonalization<double>(
                A, v, static_cast<LongIndexType>(num_rows), m, tol,
                orthogonalize, alpha, beta);
    else
        size = c_lanczos_tridiagonalization<double>(
                A, v, static_cast<LongIndexType>(num_rows), m, tol,
                orthogonalize, alpha, beta);
    delete A;
    return size;
}

// Nodes and weights as _c_stochastic_lanczos_quadrature forms them
// (c_trace_estimator.cpp:511-555): theta = eigenvalues (or squared singular
// values for gram), tau = first eigenvector (right singular vector) entry.
int ref_nodes_weights_f64(const double* alpha, const double* beta, int size,
                          int gram, double* theta, double* tau)
{
    double* a = new double[size];
    double* b = new double[size];
    std::memcpy(a, alpha, sizeof(double) * size);
    std::memcpy(b, beta, sizeof(double) * size);
    int info;
    if (gram)
    {
        double* U = new double[size * size];
        double* VT = new double[size * size];
        info = Diagonalization<double>::svd_bidiagonal(a, b, U, VT, size);
        for (int i = 0; i < size; ++i)
        {
            theta[i] = a[i] * a[i];
            tau[i] = VT[i];
        }
        delete[] U;
        delete[] VT;
    }
    else
    {
        double* Z = new double[size * size];
        info = Diagonalization<double>::eigh_tridiagonal(a, b, Z, size);
        for (int i = 0; i < size; ++i)
        {
            theta[i] = a[i];
            tau[i] = Z[i * size];
        }
        delete[] Z;
    }
    delete[] a;
    delete[] b;
    return info;
}

int ref_max_threads(void)
{
    return omp_get_max_threads();
}

}  // extern "C"
