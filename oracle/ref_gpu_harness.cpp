// Test infrastructure only: a thin C entry layer around the reference's own
// GPU SLQ (ameli/imate v0.25.2: cuTraceEstimator over a cuCSRMatrix, with
// cuSPARSE SpMV and cuBLAS vector operations), compiled from its sources by
// oracle/Makefile (target ref_gpu) into oracle/_ref/libimate_ref_gpu.so.
// Nothing in the product links or loads this file; tests/ use it as a second
// checker and bench.py times it as the reference GPU comparator.
//
// The entry points mirror ref_harness.cpp's ref_trace_estimator_* for the
// GPU path (imate/_cu_trace_estimator/cu_trace_estimator.cu:197-315): a
// CSR matrix given as host arrays is copied to the device by the
// reference's own operator constructor (cu_csr_matrix.cu:165-224).

#include <cmath>
#include <cstdint>

#include <cuda_runtime_api.h>

#include "_definitions/types.h"
#include "_cu_linear_operator/cu_csr_matrix.h"
#include "_cu_linear_operator/cu_dense_matrix.h"
#include "_cu_trace_estimator/cu_trace_estimator.h"
#include "functions/functions.h"
#include "functions/logarithm.h"
#include "functions/inverse.h"
#include "functions/identity.h"

namespace {

Function* gpu_function(int func_id)
{
    switch (func_id)
    {
        case 0: return new Logarithm();
        case 1: return new Inverse();
        default: return new Identity();
    }
}

// indices == NULL selects the dense row-major operator (cu_dense_matrix.cu:
// 40-61, cuBLAS gemv per product) over `data`; otherwise the CSR operator.
template <typename T>
int run_gpu_trace_estimator(
        const T* data, const int* indices, const int* indptr, int64_t num_rows,
        int64_t num_cols, int func_id, int gram, T exponent, int orthogonalize,
        int64_t seed, int lanczos_degree, T lanczos_tol, int min_num_samples,
        int max_num_samples, T error_atol, T error_rtol, T confidence_level,
        T outlier_significance_level, int num_gpu_devices, T* trace, T* error,
        T* samples /* [max] */, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    cuLinearOperator<T>* A;
    if (indices)
        A = new cuCSRMatrix<T>(
                data, reinterpret_cast<const LongIndexType*>(indices),
                reinterpret_cast<const LongIndexType*>(indptr), num_rows,
                num_cols, num_gpu_devices);
    else
        A = new cuDenseMatrix<T>(data, num_rows, num_cols, 1,
                                 num_gpu_devices);
    Function* f = gpu_function(func_id);
    T** rows = new T*[max_num_samples];
    for (int i = 0; i < max_num_samples; ++i)
    {
        samples[i] = NAN;
        rows[i] = &samples[i];
    }
    T parameters[1] = {0};
    *converged = 0;
    *num_samples_used = 0;
    *num_outliers = 0;
    float wall = 0.0f;
    const int all_converged = cuTraceEstimator<T>::cu_trace_estimator(
            A, parameters, 1, f, gram, exponent, orthogonalize, seed,
            lanczos_degree, lanczos_tol, min_num_samples, max_num_samples,
            error_atol, error_rtol, confidence_level,
            outlier_significance_level, 1, num_gpu_devices, trace, error, rows,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, wall);
    *alg_wall_time = wall;
    delete[] rows;
    delete f;
    delete A;
    return all_converged;
}

}  // namespace

extern "C" {

int ref_gpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

// The reference GPU estimator on a CSR matrix, or on a dense row-major one
// when indices and indptr are NULL (one inquiry, func_id 0 = log, 1 = inv,
// 2 = identity).
int ref_gpu_trace_estimator_f64(
        const double* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int func_id, int gram,
        double exponent, int orthogonalize, int64_t seed, int lanczos_degree,
        double lanczos_tol, int min_num_samples, int max_num_samples,
        double error_atol, double error_rtol, double confidence_level,
        double outlier_significance_level, int num_gpu_devices, double* trace,
        double* error, double* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    return run_gpu_trace_estimator<double>(
            data, indices, indptr, num_rows, num_cols, func_id, gram, exponent,
            orthogonalize, seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_gpu_devices, trace, error, samples,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, alg_wall_time);
}

int ref_gpu_trace_estimator_f32(
        const float* data, const int* indices, const int* indptr,
        int64_t num_rows, int64_t num_cols, int func_id, int gram,
        float exponent, int orthogonalize, int64_t seed, int lanczos_degree,
        float lanczos_tol, int min_num_samples, int max_num_samples,
        float error_atol, float error_rtol, float confidence_level,
        float outlier_significance_level, int num_gpu_devices, float* trace,
        float* error, float* samples, int* processed_samples_indices,
        int* num_samples_used, int* num_outliers, int* converged,
        float* alg_wall_time)
{
    return run_gpu_trace_estimator<float>(
            data, indices, indptr, num_rows, num_cols, func_id, gram, exponent,
            orthogonalize, seed, lanczos_degree, lanczos_tol, min_num_samples,
            max_num_samples, error_atol, error_rtol, confidence_level,
            outlier_significance_level, num_gpu_devices, trace, error, samples,
            processed_samples_indices, num_samples_used, num_outliers,
            converged, alg_wall_time);
}

}  // extern "C"
