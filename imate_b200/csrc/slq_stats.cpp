// Host statistics of the estimator: the convergence test run after every
// processed sample and the outlier-trimmed final average, with the same
// decisions as imate/_c_trace_estimator/convergence_tools.cpp:95-376.  They
// run on the host because the reference's stopping rule is sequential in the
// sample order; the engine computes a block of samples on the device and
// replays this test over the block in order, so the number of samples used,
// the estimate and its error are those of the reference run with one thread.

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/slq.h"

extern "C" {

// Inverse error function.  Initial guess from Winitzki's closed form
// (S. Winitzki, "A handy approximation for the error function and its
// inverse", 2008, a = 0.147), refined by Newton steps on std::erf.
double slq_erfinv(double x)
{
    if (x >= 1.0) return INFINITY;
    if (x <= -1.0) return -INFINITY;
    if (x == 0.0) return 0.0;
    const double a = 0.147;
    const double pi = 3.14159265358979323846;
    const double ln = std::log(1.0 - x * x);
    const double t = 2.0 / (pi * a) + ln / 2.0;
    double y = std::sqrt(std::sqrt(t * t - ln / a) - t);
    if (x < 0) y = -y;
    for (int it = 0; it < 8; ++it)
    {
        const double step = (std::erf(y) - x) /
                            (2.0 / std::sqrt(pi) * std::exp(-y * y));
        y -= step;
        if (std::fabs(step) <= 1e-17 * std::fabs(y)) break;
    }
    return y;
}

// convergence_tools.cpp:95-194.  samples is [max][q] row-major; order lists
// the processed rows.  Returns 1 when every inquiry has converged.
int slq_check_convergence(const double* samples, int q, int min_s,
                          const int32_t* order, int nproc, double conf,
                          double atol, double rtol, double* error,
                          int32_t* used, int32_t* converged)
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
    const double z = std::sqrt(2.0) * slq_erfinv(conf);
    for (int j = 0; j < q; ++j)
    {
        if (converged[j]) continue;
        double sum = 0.0;
        for (int i = 0; i < nproc; ++i)
            sum += samples[static_cast<int64_t>(order[i]) * q + j];
        const double mean = sum / nproc;
        double sd;
        if (nproc > 1)
        {
            sum = 0.0;
            for (int i = 0; i < nproc; ++i)
            {
                const double d = samples[static_cast<int64_t>(order[i]) * q + j] - mean;
                sum += d * d;
            }
            sd = std::sqrt(sum / (nproc - 1.0));
        }
        else
        {
            sd = INFINITY;
        }
        error[j] = z * sd / std::sqrt(static_cast<double>(nproc));
        const double thr = std::fmax(atol, rtol * mean);
        if (error[j] < thr) converged[j] = 1;
        used[j] = nproc;
    }
    for (int j = 0; j < q; ++j)
        if (!converged[j]) return 0;
    return 1;
}

// convergence_tools.cpp:256-376.
void slq_average_estimates(double conf, double outlier_sig, int q, int max_s,
                           const int32_t* used, const int32_t* order,
                           const double* samples, int32_t* num_outliers,
                           double* trace, double* error)
{
    std::vector<char> out(max_s > 0 ? max_s : 1);
    const double ez = std::sqrt(2.0) * slq_erfinv(conf);
    const double oz = std::sqrt(2.0) * slq_erfinv(1.0 - outlier_sig);
    for (int j = 0; j < q; ++j)
    {
        std::fill(out.begin(), out.end(), 0);
        num_outliers[j] = 0;
        const int nu = used[j];
        auto sample = [&](int i) {
            return samples[static_cast<int64_t>(order[i]) * q + j];
        };
        double sum = 0.0;
        for (int i = 0; i < nu; ++i) sum += sample(i);
        double mean = sum / nu;
        double sd;
        if (nu > 1)
        {
            sum = 0.0;
            for (int i = 0; i < nu; ++i)
            {
                const double d = sample(i) - mean;
                sum += d * d;
            }
            sd = std::sqrt(sum / (nu - 1.0));
        }
        else
        {
            sd = INFINITY;
        }
        const double half = oz * sd;
        for (int i = 0; i < nu; ++i)
            if (std::fabs(sample(i) - mean) > half)
            {
                out[i] = 1;
                num_outliers[j] += 1;
            }
        sum = 0.0;
        for (int i = 0; i < nu; ++i)
            if (!out[i]) sum += sample(i);
        mean = sum / (nu - num_outliers[j]);
        if (nu > 1 + num_outliers[j])
        {
            sum = 0.0;
            for (int i = 0; i < nu; ++i)
                if (!out[i])
                {
                    const double d = sample(i) - mean;
                    sum += d * d;
                }
            sd = std::sqrt(sum / (nu - num_outliers[j] - 1.0));
        }
        else
        {
            sd = INFINITY;
        }
        trace[j] = mean;
        error[j] = ez * sd / std::sqrt(static_cast<double>(nu - num_outliers[j]));
    }
}

}  // extern "C"
