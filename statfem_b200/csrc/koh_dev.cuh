// Device routines of the KOH marginal log-likelihood
// (LikelihoodKOH::giveLogLikelihood, statX/infer/LikelihoodKOH.ipp:75-120),
// shared by the batched kernel (stats.cu) and the allocation-free entry point
// (noalloc.cu): the squared-exponential mismatch covariance
// (MismatchCovariance.hpp:76-99), an in-place lower Cholesky and forward
// substitution run by one CTA, and the log-likelihood on a caller's work
// array [C (ns x ns) | D (ns x n_o)].
#pragma once

#include <cmath>

#include "common.cuh"

namespace sfc {

// squared-exponential value, the reference's expression order
inline __device__ double se_value(const double *x, const double *y, int dim, double sigma, double length)
{
    double t[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
        const double d = x[a] - y[a];
        t[a] = __dmul_rn(d, d);
    }
    double sq = dim == 1 ? t[0] : dim == 2 ? __dadd_rn(t[0], t[1]) : __dadd_rn(t[0], __dadd_rn(t[1], t[2]));
    return __dmul_rn(__dmul_rn(sigma, sigma), exp(-sq / __dmul_rn(__dmul_rn(2., length), length)));
}

// in-place lower Cholesky of the n x n row-major A (upper part left as is);
// info[b] = 0 or k+1 at the first non-positive pivot (Eigen::LLT info != Success)
inline __device__ void chol_lower(int n, double *A, int lda, int *info)
{
    __shared__ double piv;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            const double d = A[(int64_t)k * lda + k];
            if (!(d > 0.0)) {
                bad = k + 1;
                piv = 1.0;
            } else {
                piv = sqrt(d);
            }
            A[(int64_t)k * lda + k] = piv;
        }
        __syncthreads();
        if (bad) break;
        const double pv = piv;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[(int64_t)i * lda + k] /= pv;
        __syncthreads();
        const int m = n - k - 1;
        for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += blockDim.x) {
            const int i = k + 1 + (int)(t / m), j = k + 1 + (int)(t % m);
            if (j <= i) A[(int64_t)i * lda + j] -= A[(int64_t)i * lda + k] * A[(int64_t)j * lda + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *info = bad;
    __syncthreads();
}

// B = L^-1 B (forward substitution), L lower n x n, B n x m (row-major)
inline __device__ void trsm_lower(int n, const double *L, int ldl, int m, double *B, int ldb)
{
    for (int k = 0; k < n; ++k) {
        const double d = L[(int64_t)k * ldl + k];
        for (int c = threadIdx.x; c < m; c += blockDim.x) B[(int64_t)k * ldb + c] /= d;
        __syncthreads();
        for (int64_t t = threadIdx.x; t < (int64_t)(n - k - 1) * m; t += blockDim.x) {
            const int i = k + 1 + (int)(t / m), c = (int)(t % m);
            B[(int64_t)i * ldb + c] -= L[(int64_t)i * ldl + k] * B[(int64_t)k * ldb + c];
        }
        __syncthreads();
    }
}

// MismatchCovariance::giveCovariance (statX/infer/MismatchCovariance.hpp:76-99)
inline __device__ void mismatch_cov(int ns, const double *xs, int dim, double sd, double ld, double eps, double *K)
{
    for (int64_t t = threadIdx.x; t < (int64_t)ns * ns; t += blockDim.x) {
        const int k = (int)(t / ns), l = (int)(t % ns);
        double v = se_value(xs + 3 * k, xs + 3 * l, dim, sd, ld);
        if (k == l) v += eps * eps;
        K[t] = v;
    }
    __syncthreads();
}

// LikelihoodKOH::giveLogLikelihood on one CTA; work holds ns*ns + ns*n_o
// doubles ([C | D]); info = 0, k+1 when the Cholesky pivot k failed, or -1
// for a non-negative quadratic term (FTL_VERIFY, LikelihoodKOH.ipp:113)
inline __device__ void koh_loglik_dev(int ns, int n_o, const double *__restrict__ mean, const double *__restrict__ Cs,
                               const double *__restrict__ xs, int dim, const double *__restrict__ Y,
                               const sfc_hparams_t &hp, double *__restrict__ work, double *out, int *info)
{
    double *C = work;
    double *D = work + (int64_t)ns * ns;
    mismatch_cov(ns, xs, dim, hp.mismatch_sigma, hp.mismatch_length, hp.mismatch_sensor_eps, C);
    const double rho = hp.rho;
    for (int64_t t = threadIdx.x; t < (int64_t)ns * ns; t += blockDim.x) C[t] += rho * rho * Cs[t];
    for (int64_t t = threadIdx.x; t < (int64_t)ns * n_o; t += blockDim.x) D[t] = Y[t] - rho * mean[t / n_o];
    __syncthreads();
    chol_lower(ns, C, ns, info);
    if (*info) {
        if (threadIdx.x == 0) *out = NAN;
        return;
    }
    trsm_lower(ns, C, ns, n_o, D, n_o);
    __shared__ double red[1024];
    double ld = 0.0;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) ld += log(C[(int64_t)k * ns + k]);
    red[threadIdx.x] = ld;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double sumlog = red[0];
    __syncthreads();
    // quadratic terms per reading
    double t3 = 0.0;
    bool ok = true;
    for (int r = 0; r < n_o; ++r) {
        double q = 0.0;
        for (int k = threadIdx.x; k < ns; k += blockDim.x) q += D[(int64_t)k * n_o + r] * D[(int64_t)k * n_o + r];
        red[threadIdx.x] = q;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        const double comp = -0.5 * red[0];
        if (!(comp < 0.0)) ok = false;
        t3 += comp;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double t1 = -0.5 * ns * log(2. * M_PI);
        const double t2 = -0.5 * (2. * sumlog);
        *out = n_o * (t1 + t2) + t3;
        if (!ok) *info = -1;
    }
}

}  // namespace sfc
