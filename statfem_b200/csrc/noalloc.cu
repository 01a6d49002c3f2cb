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

#include "common.cuh"
#include "koh_dev.cuh"

namespace {

constexpr int kMaxSensors = 128;
constexpr int kMaxReadings = 64;
constexpr size_t kScratchDoubles = (size_t)kMaxSensors * kMaxSensors + (size_t)kMaxSensors * kMaxReadings;

// [C (ns x ns) | D (ns x n_o)]: 128 * 128 + 128 * 64 doubles = 192 KiB per device
static __device__ __align__(256) double g_koh_scratch[kScratchDoubles];

// one CTA of 1024 threads on the fixed scratch [C (ns x ns) | D (ns x n_o)]
__global__ void __launch_bounds__(1024) k_koh_loglik_fixed(int ns, int n_o, const double *__restrict__ mean,
                                                           const double *__restrict__ Cs, const double *__restrict__ xs,
                                                           int dim, const double *__restrict__ Y, sfc_hparams_t hp,
                                                           double *__restrict__ scratch, double *out, int *info)
{
    sfc::koh_loglik_dev(ns, n_o, mean, Cs, xs, dim, Y, hp, scratch, out, info);
}

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
    // the scratch array's address in the current context, looked up on every
    // call (a host-side lookup that allocates nothing once the module is
    // loaded), so it stays right after cudaDeviceReset and for callers that
    // switch devices or contexts
    void *scratch = nullptr;
    if (cudaGetSymbolAddress(&scratch, g_koh_scratch) != cudaSuccess) {
        cudaGetLastError();
        return SFC_ERR_CUDA;
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
