// Allocation-free variant of the KOH log-likelihood kernel
// (LikelihoodKOH::giveLogLikelihood, statX/infer/LikelihoodKOH.ipp:75-120).
//
// Who needs it: callers that cannot allocate device memory once they are
// running -- an MCMC driver evaluating proposals on a stream it owns, where
// the device-wide synchronisation of cudaMalloc / cudaFree would stall other
// work, or a host application that hands this library a fixed memory budget
// at start-up.  The regular entry point (sfc_koh_log_likelihood) keeps its
// workspace in buffers it grows on demand; this one takes every input and
// output as caller-owned device memory and keeps its scratch (the Cholesky
// factor and the whitened residuals) in a fixed file-scope device array.
//
// That array exists once per device for as long as the library is loaded.
// Its size caps the problem at kMaxSensors sensors and kMaxReadings readings.
// Every call shares it and it keeps the last call's contents; the kernel
// writes every scratch entry it reads, so nothing has to be cleared between
// calls.  Two calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on the array and must be serialised by the
// caller.

#include <cmath>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kMaxSensors = 128;
constexpr int kMaxReadings = 64;
constexpr int kMaxDevices = 64;
constexpr size_t kScratchDoubles = (size_t)kMaxSensors * kMaxSensors + (size_t)kMaxSensors * kMaxReadings;

// [C (ns x ns) | D (ns x n_o)]: 128 * 128 + 128 * 64 doubles = 192 KiB per device
static __device__ __align__(256) double g_koh_scratch[kScratchDoubles];

__device__ __forceinline__ double se_kernel(const double *x, const double *y, int dim, double sigma, double length)
{
    double t[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
        const double d = x[a] - y[a];
        t[a] = __dmul_rn(d, d);
    }
    const double sq = dim == 1 ? t[0] : dim == 2 ? __dadd_rn(t[0], t[1]) : __dadd_rn(t[0], __dadd_rn(t[1], t[2]));
    return __dmul_rn(__dmul_rn(sigma, sigma), exp(-sq / __dmul_rn(__dmul_rn(2., length), length)));
}

__device__ double block_sum1024(double v, double *red)
{
    red[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double s = red[0];
    __syncthreads();
    return s;
}

// one CTA of 1024 threads; scratch = [C (ns x ns) | D (ns x n_o)]
__global__ void __launch_bounds__(1024) k_koh_loglik_fixed(int ns, int n_o, const double *__restrict__ mean,
                                                           const double *__restrict__ Cs, const double *__restrict__ xs,
                                                           int dim, const double *__restrict__ Y, sfc_hparams_t hp,
                                                           double *__restrict__ scratch, double *out, int *info)
{
    __shared__ double red[1024];
    __shared__ double piv;
    __shared__ int bad;
    double *C = scratch;
    double *D = scratch + (int64_t)ns * ns;
    const double rho = hp.rho, eps = hp.mismatch_sensor_eps;
    // total covariance C = K_s + rho^2 C_s (MismatchCovariance.hpp:76-99,
    // LikelihoodKOH.ipp:19-39) and residuals D = y_k - rho mean
    for (int64_t t = threadIdx.x; t < (int64_t)ns * ns; t += blockDim.x) {
        const int k = (int)(t / ns), l = (int)(t % ns);
        double v = se_kernel(xs + 3 * k, xs + 3 * l, dim, hp.mismatch_sigma, hp.mismatch_length);
        if (k == l) v += eps * eps;
        C[t] = v + rho * rho * Cs[t];
    }
    for (int64_t t = threadIdx.x; t < (int64_t)ns * n_o; t += blockDim.x) D[t] = Y[t] - rho * mean[t / n_o];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    // in-place lower Cholesky (Eigen::LLT, LikelihoodKOH.ipp:92-93)
    for (int k = 0; k < ns; ++k) {
        if (threadIdx.x == 0) {
            const double d = C[(int64_t)k * ns + k];
            if (!(d > 0.0)) {
                bad = k + 1;
                piv = 1.0;
            } else {
                piv = sqrt(d);
            }
            C[(int64_t)k * ns + k] = piv;
        }
        __syncthreads();
        if (bad) break;
        const double pv = piv;
        for (int i = k + 1 + threadIdx.x; i < ns; i += blockDim.x) C[(int64_t)i * ns + k] /= pv;
        __syncthreads();
        const int m = ns - k - 1;
        for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += blockDim.x) {
            const int i = k + 1 + (int)(t / m), j = k + 1 + (int)(t % m);
            if (j <= i) C[(int64_t)i * ns + j] -= C[(int64_t)i * ns + k] * C[(int64_t)j * ns + k];
        }
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) {
            *info = bad;
            *out = NAN;
        }
        return;
    }
    // D = L^-1 D
    for (int k = 0; k < ns; ++k) {
        const double d = C[(int64_t)k * ns + k];
        for (int c = threadIdx.x; c < n_o; c += blockDim.x) D[(int64_t)k * n_o + c] /= d;
        __syncthreads();
        for (int64_t t = threadIdx.x; t < (int64_t)(ns - k - 1) * n_o; t += blockDim.x) {
            const int i = k + 1 + (int)(t / n_o), c = (int)(t % n_o);
            D[(int64_t)i * n_o + c] -= C[(int64_t)i * ns + k] * D[(int64_t)k * n_o + c];
        }
        __syncthreads();
    }
    double ld = 0.0;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) ld += log(C[(int64_t)k * ns + k]);
    const double sumlog = block_sum1024(ld, red);
    double t3 = 0.0;
    bool ok = true;
    for (int r = 0; r < n_o; ++r) {
        double q = 0.0;
        for (int k = threadIdx.x; k < ns; k += blockDim.x) q += D[(int64_t)k * n_o + r] * D[(int64_t)k * n_o + r];
        const double comp = -0.5 * block_sum1024(q, red);
        if (!(comp < 0.0)) ok = false;  // FTL_VERIFY( tmp3Comp < 0. ), LikelihoodKOH.ipp:113
        t3 += comp;
    }
    if (threadIdx.x == 0) {
        const double t1 = -0.5 * ns * log(2. * M_PI);
        const double t2 = -0.5 * (2. * sumlog);
        *out = n_o * (t1 + t2) + t3;
        *info = ok ? 0 : -1;
    }
}

// per-device address of g_koh_scratch, looked up once with the device current.
// The address belongs to the context that was current at the lookup (the
// device's primary context for runtime-API callers); after cudaDeviceReset,
// or for a caller that makes another context current, it is stale, so both
// are documented as unsupported in the public header.
std::mutex g_sym_mutex;
void *g_sym_addr[kMaxDevices] = {};

}  // namespace

extern "C" int32_t sfc_koh_log_likelihood_noalloc(const double *mean_dev, const double *cov_dev,
                                                  const double *sensor_coords_dev, int32_t dim, const double *y_dev,
                                                  int32_t num_sensors, int32_t num_readings, const sfc_hparams_t *hp,
                                                  double *loglik_dev, int32_t *info_dev, void *stream)
{
    if (!mean_dev || !cov_dev || !sensor_coords_dev || !y_dev || !hp || !loglik_dev || !info_dev || dim < 1 ||
        dim > 3 || num_sensors < 1 || num_readings < 1)
        return SFC_ERR_BAD_ARG;
    if (num_sensors > kMaxSensors || num_readings > kMaxReadings) return SFC_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return SFC_ERR_CUDA;
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_sym_mutex);
        if (!g_sym_addr[dev]) {
            // first call on this device: the device is current here
            if (cudaGetSymbolAddress(&g_sym_addr[dev], g_koh_scratch) != cudaSuccess) {
                g_sym_addr[dev] = nullptr;
                cudaGetLastError();
                return SFC_ERR_CUDA;
            }
        }
        scratch = g_sym_addr[dev];
    }
    k_koh_loglik_fixed<<<1, 1024, 0, (cudaStream_t)stream>>>(num_sensors, num_readings, mean_dev, cov_dev,
                                                              sensor_coords_dev, dim, y_dev, *hp, (double *)scratch,
                                                              loglik_dev, info_dev);
    // check this launch without consuming an error that earlier, unrelated
    // runtime work left for its owner: only a failed launch is cleared
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return SFC_ERR_CUDA;
    }
    return SFC_OK;
}
