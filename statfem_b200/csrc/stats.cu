// statX on the GPU: nodal forcing covariance, ForwardGaussRHS, mismatch
// covariance and the Kennedy-O'Hagan likelihood / posterior, all FP64.
//
// Forcing covariance (statX/infer/CovarianceForcing.ipp:38-109) is
//   C_f[i][j] = phibar_i k(x_i,x_j) phibar_j   (same component, 0 otherwise),
// k the squared-exponential kernel (statX/infer/ExpKernel.hpp:74-92).  The
// reference materialises C_f as N^2 triplets; here M C_f M^T is evaluated
// matrix-free as W^T (K W) with W = diag(phibar) M^T:
//   * general node sets: K W with the kernel evaluated on the fly, tile by
//     tile;
//   * tensor-grid node sets (structured meshes): K = s^2 Kz (x) Ky (x) Kx, so
//     K W is three small dense products along the grid axes -- the same
//     matrix in exact arithmetic at O(N (nx+ny+nz)) instead of O(N^2).
// Small dense algebra (Cholesky, triangular solves, SPD inverses) runs in
// single-CTA kernels with a batch index in blockIdx.x.

#include <cmath>
#include <vector>

#include "common.cuh"
#include "koh_dev.cuh"

namespace sfc {

namespace {

// ---------------------------------------------------------------------------
// kernels: forcing covariance
// ---------------------------------------------------------------------------

// B[idx][a] = val for each entry of P row a (B is N x ns, zeroed before)
__global__ void k_scatter_pt(const int64_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                             const double *__restrict__ val, int64_t ns, double *__restrict__ B)
{
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < ns; a += (int64_t)gridDim.x * blockDim.x)
        for (int64_t s = ptr[a]; s < ptr[a + 1]; ++s) B[(int64_t)idx[s] * ns + a] += val[s];
}

// W[i][a] = phibar[i] * X[i][a]
__global__ void k_scale_rows(const double *__restrict__ X, const double *__restrict__ phibar, int64_t N, int64_t ns,
                             double *__restrict__ W)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * ns; t += (int64_t)gridDim.x * blockDim.x)
        W[t] = phibar[t / ns] * X[t];
}

// out[a] = sum_i X[i][a] F[i]   (one block per column a, FP64 reduction)
__global__ void k_colsum_dot(const double *__restrict__ X, const double *__restrict__ F, int64_t N, int64_t ns,
                             double *__restrict__ out)
{
    __shared__ double sh[256];
    for (int64_t a = blockIdx.x; a < ns; a += gridDim.x) {
        double s = 0;
        for (int64_t i = threadIdx.x; i < N; i += blockDim.x) s += X[i * ns + a] * F[i];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[a] = sh[0];
        __syncthreads();
    }
}

// T[i*dof+c][a] = sum_j k(x_i,x_j) W[j*dof+c][a], kernel on the fly.
// Block: 16 nodes i x all columns; j tiles of 16 nodes staged in shared memory.
constexpr int kTI = 16, kTJ = 16;
__global__ void __launch_bounds__(256) k_kw_dense(const double *__restrict__ coords, int64_t nodes, int dim, int dof,
                                                   int c, int64_t ns, const double *__restrict__ W,
                                                   double *__restrict__ T, double sigma, double length)
{
    extern __shared__ double smem[];
    double *kv = smem;                 // kTI x kTJ
    double *wt = smem + kTI * kTJ;     // kTJ x ns
    const int64_t i0 = (int64_t)blockIdx.x * kTI;
    const int nout = kTI * (int)ns;
    double acc[16];
    for (int u = 0; u < 16; ++u) acc[u] = 0.0;
    for (int64_t j0 = 0; j0 < nodes; j0 += kTJ) {
        __syncthreads();
        for (int t = threadIdx.x; t < kTI * kTJ; t += blockDim.x) {
            const int ii = t / kTJ, jj = t % kTJ;
            const int64_t i = i0 + ii, j = j0 + jj;
            kv[t] = (i < nodes && j < nodes) ? se_value(coords + 3 * i, coords + 3 * j, dim, sigma, length) : 0.0;
        }
        for (int t = threadIdx.x; t < kTJ * ns; t += blockDim.x) {
            const int jj = t / (int)ns, a = t % (int)ns;
            const int64_t j = j0 + jj;
            wt[t] = j < nodes ? W[(j * dof + c) * ns + a] : 0.0;
        }
        __syncthreads();
        for (int u = 0, o = threadIdx.x; o < nout && u < 16; o += blockDim.x, ++u) {
            const int ii = o / (int)ns, a = o % (int)ns;
            double s = acc[u];
#pragma unroll
            for (int jj = 0; jj < kTJ; ++jj) s = fma(kv[ii * kTJ + jj], wt[jj * ns + a], s);
            acc[u] = s;
        }
    }
    for (int u = 0, o = threadIdx.x; o < nout && u < 16; o += blockDim.x, ++u) {
        const int ii = o / (int)ns, a = o % (int)ns;
        const int64_t i = i0 + ii;
        if (i < nodes) T[(i * dof + c) * ns + a] = acc[u];
    }
}

// one axis of the Kronecker product: for every node, column a:
// out[node(m)] = sum_k Kd[m][k] in[node(k)]  along axis d (stride sd, length nd)
// STAGE: the nd x nd factor is staged in shared memory (it fits); else it
// is read through the cache
template <bool STAGE>
__global__ void k_kron_axis(const double *__restrict__ Kd, int nd, int64_t sd, int64_t nodes, int dof, int c,
                            int64_t ns, const double *__restrict__ in, double *__restrict__ out)
{
    extern __shared__ double sKd[];
    const double *sK = Kd;
    if (STAGE) {
        for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) sKd[t] = Kd[t];
        __syncthreads();
        sK = sKd;
    }
    const int64_t total = nodes * ns;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t node = t / ns;
        const int64_t a = t - node * ns;
        const int64_t m = (node / sd) % nd;
        const int64_t base = node - m * sd;
        double s = 0.0;
        for (int k = 0; k < nd; ++k) s = fma(sK[m * nd + k], in[((base + k * sd) * dof + c) * ns + a], s);
        out[(node * dof + c) * ns + a] = s;
    }
}

// The same axis product as a batch of small dense products, for nd <= 64
// points per line: one CTA per (line, 128 columns) stages the line's input
// rows and the factor in shared memory; warp w computes the output points
// m = w, w + 8, ... and lane l the columns l, l + 32, l + 64, l + 96, so each
// staged value feeds up to 8 multiply-adds from registers.
constexpr int kLineCols = 128;

__global__ void __launch_bounds__(256) k_kron_line(const double *__restrict__ Kd, int nd, int64_t sd, int dof, int c,
                                                   int64_t ns, const double *__restrict__ in, double *__restrict__ out)
{
    extern __shared__ double sm[];
    double *sK = sm, *sIn = sm + nd * nd;
    const int64_t L = blockIdx.x;  // line: nodes base + k sd, k < nd
    const int64_t base = (L / sd) * sd * nd + L % sd;
    const int64_t col0 = (int64_t)blockIdx.y * kLineCols;
    const int ncols = (int)(ns - col0 < kLineCols ? ns - col0 : kLineCols);
    for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) sK[t] = Kd[t];
    // eight loads in flight per thread before they are stored
    const int total = nd * kLineCols;
    for (int t0 = threadIdx.x; t0 < total; t0 += 8 * blockDim.x) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int t = t0 + u * blockDim.x, k = t / kLineCols, j = t % kLineCols;
            v[u] = (t < total && j < ncols) ? in[((base + k * sd) * dof + c) * ns + col0 + j] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < total) sIn[t] = v[u];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double acc[8][4];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[u][q] = 0.0;
    for (int k = 0; k < nd; ++k) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = sIn[k * kLineCols + lane + 32 * q];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int m = w + 8 * u;
            const double kv = m < nd ? sK[m * nd + k] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[u][q] = fma(kv, v[q], acc[u][q]);
        }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int m = w + 8 * u;
        if (m >= nd) continue;
        double *o = out + ((base + m * sd) * dof + c) * ns + col0;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (lane + 32 * q < ncols) o[lane + 32 * q] = acc[u][q];
    }
}

// C[a][b] += sum_i A[i][a] B[i][b] over a slice of rows (split-K, atomics);
// 64 x 64 output tile per block, 4 x 4 per thread
__global__ void __launch_bounds__(256) k_atb(const double *__restrict__ A, const double *__restrict__ B, int64_t K,
                                              int64_t M, int64_t Nn, int64_t rows_per_block, double alpha,
                                              double *__restrict__ C)
{
    __shared__ double sa[16][64];
    __shared__ double sb[16][64];
    const int64_t a0 = blockIdx.y * 64, b0 = blockIdx.z * 64;
    const int64_t k0 = blockIdx.x * rows_per_block;
    const int64_t k1 = min(K, k0 + rows_per_block);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[4][4] = {};
    for (int64_t kk = k0; kk < k1; kk += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int r = t / 64, cc = t % 64;
            const int64_t k = kk + r;
            sa[r][cc] = (k < k1 && a0 + cc < M) ? A[k * M + a0 + cc] : 0.0;
            sb[r][cc] = (k < k1 && b0 + cc < Nn) ? B[k * Nn + b0 + cc] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av[u] = sa[r][ty * 4 + u];
                bv[u] = sb[r][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int64_t a = a0 + ty * 4 + u, b = b0 + tx * 4 + v;
            if (a < M && b < Nn) atomicAdd(&C[a * Nn + b], alpha * acc[u][v]);
        }
}

// general row-major C = alpha op(A) op(B) + beta C  (small dense algebra)
__global__ void __launch_bounds__(256) k_gemm(int ta, int tb, int64_t M, int64_t N, int64_t K, double alpha,
                                               const double *__restrict__ A, int64_t lda, const double *__restrict__ B,
                                               int64_t ldb, double beta, double *__restrict__ C, int64_t ldc)
{
    __shared__ double sa[16][64];
    __shared__ double sb[16][64];
    const int64_t m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[4][4] = {};
    for (int64_t k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int r = t / 64, cc = t % 64;
            const int64_t k = k0 + r, m = m0 + cc, n = n0 + cc;
            sa[r][cc] = (k < K && m < M) ? (ta ? A[k * lda + m] : A[m * lda + k]) : 0.0;
            sb[r][cc] = (k < K && n < N) ? (tb ? B[n * ldb + k] : B[k * ldb + n]) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av[u] = sa[r][ty * 4 + u];
                bv[u] = sb[r][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int64_t m = m0 + ty * 4 + u, n = n0 + tx * 4 + v;
            if (m < M && n < N) C[m * ldc + n] = alpha * acc[u][v] + (beta == 0.0 ? 0.0 : beta * C[m * ldc + n]);
        }
}

// ---------------------------------------------------------------------------
// single-CTA dense FP64 kernels (blockIdx.x = batch item)
// ---------------------------------------------------------------------------

// many hyperparameter sets against the same forward model, one CTA each
__global__ void __launch_bounds__(1024) k_koh_loglik_batch(int ns, int n_o, const double *__restrict__ mean,
                                                           const double *__restrict__ Cs,
                                                           const double *__restrict__ xs, int dim,
                                                           const double *__restrict__ Y,
                                                           const sfc_hparams_t *__restrict__ hps, int64_t wsz,
                                                           double *__restrict__ work, double *out, int *info)
{
    const int b = blockIdx.x;
    const sfc_hparams_t hp = hps[b];
    koh_loglik_dev(ns, n_o, mean, Cs, xs, dim, Y, hp, work + (int64_t)b * wsz, out + b, info + b);
}

__global__ void k_mismatch(int ns, const double *xs, int dim, sfc_hparams_t hp, double *K)
{
    mismatch_cov(ns, xs, dim, hp.mismatch_sigma, hp.mismatch_length, hp.mismatch_sensor_eps, K);
}

__global__ void k_add_scaled(double *__restrict__ y, const double *__restrict__ x, double a, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        y[t] += a * x[t];
}

// C = K_s + rho^2 C_s (ns x ns) and D = Y - rho mean (ns x n_o)
__global__ void k_koh_system(int ns, int n_o, const double *__restrict__ mean, const double *__restrict__ Cs,
                             const double *__restrict__ xs, int dim, const double *__restrict__ Y, sfc_hparams_t hp,
                             double *__restrict__ C, double *__restrict__ D)
{
    const int64_t nn = (int64_t)ns * ns;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t / ns), l = (int)(t % ns);
        double v = se_value(xs + 3 * k, xs + 3 * l, dim, hp.mismatch_sigma, hp.mismatch_length);
        if (k == l) v += hp.mismatch_sensor_eps * hp.mismatch_sensor_eps;
        C[t] = v + hp.rho * hp.rho * Cs[t];
        if (t < (int64_t)ns * n_o) D[t] = Y[t] - hp.rho * mean[t / n_o];
    }
}

// log-likelihood from C^-1, the Schur pivots of C (log det C = sum log piv)
// and D: n_o (-ns/2 log 2 pi - 1/2 log det C) - 1/2 sum_r d_r^T C^-1 d_r;
// info = -1 when a quadratic term is not negative (LikelihoodKOH.ipp:100-120)
__global__ void __launch_bounds__(1024) k_koh_loglik_terms(int ns, int n_o, const double *__restrict__ Ci,
                                                           const double *__restrict__ D, const double *__restrict__ piv,
                                                           double *out, int *info)
{
    __shared__ double red[1024];
    auto block_total = [&](double v) {
        red[threadIdx.x] = v;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        const double r = red[0];
        __syncthreads();
        return r;
    };
    double ld = 0.0;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) ld += log(piv[k]);
    const double logdet = block_total(ld);
    double t3 = 0.0;
    bool ok = true;
    for (int r = 0; r < n_o; ++r) {
        double q = 0.0;
        for (int64_t t = threadIdx.x; t < (int64_t)ns * ns; t += blockDim.x) {
            const int i = (int)(t / ns), j = (int)(t % ns);
            q += D[(int64_t)i * n_o + r] * Ci[t] * D[(int64_t)j * n_o + r];
        }
        const double comp = -0.5 * block_total(q);
        if (!(comp < 0.0)) ok = false;
        t3 += comp;
    }
    if (threadIdx.x == 0) {
        *out = n_o * (-0.5 * ns * log(2. * M_PI) - 0.5 * logdet) + t3;
        if (!ok) *info = -1;
    }
}

__global__ void k_identity_minus(double *__restrict__ D, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n; t += (int64_t)gridDim.x * blockDim.x)
        D[t] = ((t / n) == (t % n) ? 1.0 : 0.0) - D[t];
}

__global__ void k_rowsum(const double *__restrict__ Y, int64_t ns, int n_o, double *__restrict__ out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ns; k += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int r = 0; r < n_o; ++r) s += Y[k * n_o + r];
        out[k] = s;
    }
}

void gemm(sfc_ctx *ctx, int ta, int tb, int64_t M, int64_t N, int64_t K, double alpha, const double *A, int64_t lda,
          const double *B, int64_t ldb, double beta, double *C, int64_t ldc)
{
    dim3 g((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64));
    k_gemm<<<g, 256, 0, ctx->stream>>>(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    count_launch(ctx);
}

// 1-D SE correlation factor along one grid axis: exp(-d^2/(2 l^2))
std::vector<double> se_axis(const std::vector<double> &x, double length)
{
    const int n = (int)x.size();
    std::vector<double> K((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double d = x[i] - x[j];
            K[(size_t)i * n + j] = std::exp(-(d * d) / (2. * length * length));
        }
    return K;
}

}  // namespace

// T = K W (per component); W, T, tmp: num_dofs x ns device arrays
void kernel_times(sfc_ctx *ctx, sfc_covar_forcing *cf, double sigma, double length, const double *W,
                         double *T, int64_t ns, double *tmp)
{
    const sfc_mesh *m = cf->mesh;
    const int64_t nodes = m->num_nodes;
    const int dof = m->dof;
    if (m->is_grid) {
        // K = sigma^2 Kz (x) Ky (x) Kx ; applied axis by axis, ping-ponging
        // between T and tmp
        const int nax = m->dim;
        DBuf<double> *dK = cf->kron;
        for (int a = 0; a < nax; ++a) {
            std::vector<double> Kd = se_axis(m->gaxis[a], length);
            if (a == 0)
                for (double &v : Kd) v *= sigma * sigma;
            upload(ctx, dK[a], Kd.data(), Kd.size());
        }
        for (int c = 0; c < dof; ++c) {
            const double *src = W;
            double *bufs[2] = {T, tmp};
            int64_t sd = 1;
            int cur = 0;
            for (int a = 0; a < nax; ++a) {
                const int nd = m->gn[a];
                double *dst = bufs[cur];
                ProfScope ps(ctx, "kron_axis", 2.0 * nodes * ns * 8);
                const size_t kb = (size_t)nd * nd * 8;
                if (nd <= 64) {
                    const size_t smem = (size_t)(nd * nd + nd * kLineCols) * 8;
                    SFC_CK(cudaFuncSetAttribute(k_kron_line, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                    const dim3 g((unsigned)(nodes / nd), (unsigned)((ns + kLineCols - 1) / kLineCols));
                    k_kron_line<<<g, 256, smem, ctx->stream>>>(dK[a].p, nd, sd, dof, c, ns, src, dst);
                } else if (kb <= 48 * 1024) {
                    k_kron_axis<true><<<grid_for(nodes * ns, 256), 256, kb, ctx->stream>>>(dK[a].p, nd, sd, nodes, dof,
                                                                                         c, ns, src, dst);
                } else if (kb <= 200 * 1024) {
                    SFC_CK(cudaFuncSetAttribute(k_kron_axis<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kb));
                    k_kron_axis<true><<<grid_for(nodes * ns, 256), 256, kb, ctx->stream>>>(dK[a].p, nd, sd, nodes, dof,
                                                                                         c, ns, src, dst);
                } else {
                    k_kron_axis<false><<<grid_for(nodes * ns, 256), 256, 0, ctx->stream>>>(dK[a].p, nd, sd, nodes,
                                                                                         dof, c, ns, src, dst);
                }
                count_launch(ctx);
                src = dst;
                cur ^= 1;
                sd *= nd;
            }
            if (src != T)  // strided copy of this component's rows back into T
                SFC_CK(cudaMemcpy2DAsync(T + (int64_t)c * ns, (size_t)dof * ns * 8, src + (int64_t)c * ns,
                                         (size_t)dof * ns * 8, (size_t)ns * 8, (size_t)nodes, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        }
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    } else {
        const size_t smem = (size_t)(kTI * kTJ + kTJ * ns) * 8;
        SFC_REQUIRE(ns <= 256, "dense forcing covariance supports at most 256 projection rows");
        SFC_CK(cudaFuncSetAttribute(k_kw_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (int c = 0; c < dof; ++c) {
            k_kw_dense<<<(unsigned)((nodes + kTI - 1) / kTI), 256, smem, ctx->stream>>>(m->coords.p, nodes, m->dim, dof,
                                                                                     c, ns, W, T, sigma, length);
            count_launch(ctx);
        }
    }
}

// C = A^T B for a symmetric product (A^T B = B^T A, as W^T K W): only the
// 128 x 128 tiles on and above the diagonal are formed, over a slice of the
// K rows per CTA (8 x 8 outputs per thread, 8-row chunks double-buffered in
// shared memory); partial tiles go to part[split][tile] and k_atb_sym_reduce
// adds them in split order and mirrors the upper tiles (deterministic, exactly
// symmetric).
constexpr int kSymT = 128;
constexpr int kSymK = 8;

__global__ void __launch_bounds__(256) k_atb_sym(const double *__restrict__ A, const double *__restrict__ B, int64_t K,
                                                 int64_t M, int64_t rows_per_split, const int2 *__restrict__ tiles,
                                                 int ntiles, double *__restrict__ part)
{
    __shared__ __align__(16) double sa[2][kSymK][kSymT];
    __shared__ __align__(16) double sb[2][kSymK][kSymT];
    const int2 tile = tiles[blockIdx.y];
    const int64_t a0 = (int64_t)tile.x * kSymT, b0 = (int64_t)tile.y * kSymT;
    const int64_t k0 = (int64_t)blockIdx.x * rows_per_split;
    const int64_t k1 = k0 + rows_per_split < K ? k0 + rows_per_split : K;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    // each thread stages 4 values of each operand per chunk: row t / 128, column t % 128
    double ra[4], rb[4];
    auto fetch = [&](int64_t kk) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int t = threadIdx.x + 256 * q, r = t / kSymT, c = t % kSymT;
            const int64_t k = kk + r;
            ra[q] = (k < k1 && a0 + c < M) ? A[k * M + a0 + c] : 0.0;
            rb[q] = (k < k1 && b0 + c < M) ? B[k * M + b0 + c] : 0.0;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int t = threadIdx.x + 256 * q, r = t / kSymT, c = t % kSymT;
            sa[buf][r][c] = ra[q];
            sb[buf][r][c] = rb[q];
        }
    };
    int buf = 0;
    if (k0 < k1) {
        fetch(k0);
        stash(0);
    }
    __syncthreads();
    for (int64_t kk = k0; kk < k1; kk += kSymK) {
        const bool more = kk + kSymK < k1;
        if (more) fetch(kk + kSymK);  // in flight during the products
#pragma unroll
        for (int r = 0; r < kSymK; ++r) {
            double av[8], bv[8];
#pragma unroll
            for (int i = 0; i < 8; i += 2) {
                const double2 x = *reinterpret_cast<const double2 *>(&sa[buf][r][ty * 8 + i]);
                const double2 y = *reinterpret_cast<const double2 *>(&sb[buf][r][tx * 8 + i]);
                av[i] = x.x; av[i + 1] = x.y;
                bv[i] = y.x; bv[i + 1] = y.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        if (more) stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
    double *o = part + ((int64_t)blockIdx.x * ntiles + blockIdx.y) * kSymT * kSymT;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) o[(ty * 8 + i) * kSymT + tx * 8 + j] = acc[i][j];
}

__global__ void k_atb_sym_reduce(const double *__restrict__ part, int splits, const int2 *__restrict__ tiles,
                                 int ntiles, int64_t M, double alpha, double *__restrict__ C)
{
    const int64_t total = (int64_t)ntiles * kSymT * kSymT;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int ti = (int)(t / (kSymT * kSymT));
        const int e = (int)(t % (kSymT * kSymT)), i = e / kSymT, j = e % kSymT;
        const int64_t a = (int64_t)tiles[ti].x * kSymT + i, b = (int64_t)tiles[ti].y * kSymT + j;
        if (a >= M || b >= M) continue;
        double sum = 0.0;
        for (int sp = 0; sp < splits; ++sp) sum += part[((int64_t)sp * ntiles + ti) * kSymT * kSymT + e];
        sum *= alpha;
        C[a * M + b] = sum;
        if (tiles[ti].x != tiles[ti].y) C[b * M + a] = sum;
    }
}

// C (ns x ns) = W^T (K W) with W = diag(phibar) X, X: num_dofs x ns (device)
void projected_covar(sfc_ctx *ctx, sfc_covar_forcing *cf, double sigma, double length, const double *X,
                            int64_t ns, double *C, DBuf<double> &work)
{
    const int64_t N = cf->num_dofs;
    work.reserve((size_t)3 * N * ns);
    double *W = work.p, *T = W + N * ns, *tmpp = T + N * ns;
    k_scale_rows<<<grid_for(N * ns, 256), 256, 0, ctx->stream>>>(X, cf->phibar.p, N, ns, W);
    count_launch(ctx);
    kernel_times(ctx, cf, sigma, length, W, T, ns, tmpp);
    ProfScope ps(ctx, "covar_atb", 2.0 * N * ns * 8);
    atb_symmetric(ctx, W, T, N, ns, C, cf->atb_part);
}

// C (M x M) = A^T B for A, B: K x M (row-major) with A^T B symmetric
void atb_symmetric(sfc_ctx *ctx, const double *A, const double *B, int64_t K, int64_t M, double *C,
                   DBuf<double> &part)
{
    const int nt = (int)((M + kSymT - 1) / kSymT);
    std::vector<int2> ht;
    for (int i = 0; i < nt; ++i)
        for (int j = i; j < nt; ++j) ht.push_back(make_int2(i, j));
    const int ntiles = (int)ht.size();
    int64_t splits = std::max<int64_t>(1, (ctx->sm_count * 2) / ntiles);
    int64_t rows = (K + splits - 1) / splits;
    rows = ((rows + kSymK - 1) / kSymK) * kSymK;
    splits = (K + rows - 1) / rows;
    static_assert(sizeof(int2) == 8, "tile list packing");
    part.reserve((size_t)splits * ntiles * kSymT * kSymT + (size_t)ntiles);
    int2 *dtiles = reinterpret_cast<int2 *>(part.p + (size_t)splits * ntiles * kSymT * kSymT);
    SFC_CK(cudaMemcpyAsync(dtiles, ht.data(), ntiles * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    k_atb_sym<<<dim3((unsigned)splits, (unsigned)ntiles), 256, 0, ctx->stream>>>(A, B, K, M, rows, dtiles, ntiles,
                                                                                  part.p);
    k_atb_sym_reduce<<<grid_for((int64_t)ntiles * kSymT * kSymT, 256), 256, 0, ctx->stream>>>(part.p, (int)splits,
                                                                                               dtiles, ntiles, M, 1.0, C);
    count_launch(ctx, 2);
}

// C (M x Nn) += A^T B for A: K x M, B: K x Nn (row-major), split-K
void atb_accumulate(sfc_ctx *ctx, const double *A, const double *B, int64_t K, int64_t M, int64_t Nn, double *C)
{
    const int64_t tiles = ((M + 63) / 64) * ((Nn + 63) / 64);
    int64_t splits = std::max<int64_t>(1, (ctx->sm_count * 4) / tiles);
    int64_t rows = (K + splits - 1) / splits;
    rows = ((rows + 15) / 16) * 16;
    splits = (K + rows - 1) / rows;
    dim3 g((unsigned)splits, (unsigned)((M + 63) / 64), (unsigned)((Nn + 63) / 64));
    k_atb<<<g, 256, 0, ctx->stream>>>(A, B, K, M, Nn, rows, 1.0, C);
    count_launch(ctx);
}

void forward_gauss_update(sfc_forward_gauss *fg, const sfc_hparams_t *hp)
{
    sfc_system *s = fg->sys;
    sfc_ctx *ctx = fg->ctx;
    const int64_t N = s->N, ns = fg->ns;
    SFC_REQUIRE(ns > 0, "projection matrix not set");
    SFC_REQUIRE(fg->cf->num_dofs == N, "covariance and system sizes differ");
    // right-hand sides P^T (N x ns)
    fg->B.reserve(N * ns);
    DBuf<double> &B = fg->B;
    SFC_CK(cudaMemsetAsync(B.p, 0, N * ns * 8, ctx->stream));
    k_scatter_pt<<<grid_for(ns, 128), 128, 0, ctx->stream>>>(fg->d_p_ptr.p, fg->d_p_idx.p, fg->d_p_val.p, ns, B.p);
    count_launch(ctx);
    // R^T = A^-T P^T : one block adjoint solve (solveSystemTranspose per row
    // in the reference, ForwardGaussRHS.hpp:104-112)
    fg->R.alloc(N * ns);
    flush_staged(s);
    {
        ProfScope ps(ctx, "phase:adjoint_solve", 0.0);
        solve_block(s, B.p, fg->R.p, (int)ns, (int)ns);
        transpose_fixup(s, B.p, fg->R.p, (int)ns, (int)ns);
    }
    ProfScope ps_cov(ctx, "phase:mean_and_covariance", 0.0);
    // mean = R F (ForwardGaussRHS.hpp:115-124)
    fg->mean.alloc(ns);
    k_colsum_dot<<<(unsigned)std::min<int64_t>(ns, 1024), 256, 0, ctx->stream>>>(fg->R.p, s->F.p, N, ns, fg->mean.p);
    count_launch(ctx);
    // C_s = R C_f R^T + (sigma_f reg)^2 P P^T  (ForwardGaussRHS.hpp:128-136)
    fg->cov.alloc(ns * ns);
    projected_covar(ctx, fg->cf, hp->forcing_sigma, hp->forcing_length, fg->R.p, ns, fg->cov.p, fg->work);
    const double add = hp->forcing_sigma * fg->reg;
    k_add_scaled<<<grid_for(ns * ns, 256), 256, 0, ctx->stream>>>(fg->cov.p, fg->d_ppt.p, add * add, ns * ns);
    count_launch(ctx);
    SFC_CK(cudaStreamSynchronize(ctx->stream));
    fg->valid = true;
}

void covar_projected_host(sfc_covar_forcing *cf, const sfc_hparams_t *hp, const double *M, int64_t rows, double *out)
{
    sfc_ctx *ctx = cf->ctx;
    const int64_t N = cf->num_dofs;
    // X = M^T (N x rows)
    std::vector<double> Xt((size_t)N * rows);
    for (int64_t a = 0; a < rows; ++a)
        for (int64_t i = 0; i < N; ++i) Xt[(size_t)i * rows + a] = M[(size_t)a * N + i];
    DBuf<double> X, C, work;
    upload(ctx, X, Xt.data(), Xt.size());
    C.alloc(rows * rows);
    projected_covar(ctx, cf, hp->forcing_sigma, hp->forcing_length, X.p, rows, C.p, work);
    download(ctx, out, C.p, rows * rows);
}

void koh_loglik(sfc_koh *k, const sfc_hparams_t *hp, double *out)
{
    sfc_ctx *ctx = k->ctx;
    sfc_forward_gauss *fg = k->fg;
    SFC_REQUIRE(fg->valid, "forward model not updated");
    SFC_REQUIRE(k->n_o > 0, "sensor values not set");
    const int ns = (int)k->ns, n_o = k->n_o;
    const int64_t nn = (int64_t)ns * ns;
    k->work.reserve((size_t)nn + (size_t)ns * n_o + ns + 16);
    k->outv.reserve(1);
    k->info.reserve(1);
    double *C = k->work.p, *D = C + nn, *piv = D + (int64_t)ns * n_o;
    int dropped = 0;
    {
        ProfScope ps(ctx, "phase:koh_loglik", 0.0);
        // C = K_s + rho^2 C_s, D = Y - rho mean (LikelihoodKOH.ipp:75-100)
        k_koh_system<<<grid_for(nn, 256), 256, 0, ctx->stream>>>(ns, n_o, fg->mean.p, fg->cov.p, k->sensor_coords.p,
                                                                  k->dim, k->Y.p, *hp, C, D);
        count_launch(ctx);
        spd_inverse_gj(ctx, C, ns, 0.0, k->gj, piv, &dropped);
        if (dropped) fail(SFC_ERR_NOT_SPD, "total covariance is not positive definite (LLT failed)");
        SFC_CK(cudaMemsetAsync(k->info.p, 0, sizeof(int), ctx->stream));
        k_koh_loglik_terms<<<1, 1024, 0, ctx->stream>>>(ns, n_o, C, D, piv, k->outv.p, k->info.p);
        count_launch(ctx);
    }
    int hi = 0;
    download(ctx, &hi, k->info.p, 1);
    if (hi < 0) fail(SFC_ERR_BAD_ARG, "non-negative quadratic term in the log-likelihood");
    download(ctx, out, k->outv.p, 1);
}

// LikelihoodKOH::giveLogLikelihood for n hyperparameter sets (rho and the
// mismatch parameters; the forcing parameters of the last forward update
// apply) in one launch; an item whose total covariance is not positive
// definite, or whose quadratic term is not negative, gives NaN
void koh_loglik_batch(sfc_koh *k, const sfc_hparams_t *hps, int n, double *out)
{
    sfc_ctx *ctx = k->ctx;
    sfc_forward_gauss *fg = k->fg;
    SFC_REQUIRE(fg->valid, "forward model not updated");
    SFC_REQUIRE(k->n_o > 0, "sensor values not set");
    const int ns = (int)k->ns;
    const int64_t wsz = 2 * (int64_t)ns * ns + (int64_t)ns * k->n_o;
    const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)(256e6 / 8) / std::max<int64_t>(wsz, 1)));
    // persistent on the likelihood object (grown, never shrunk): an MCMC loop
    // calls this every step
    DBuf<double> &work = k->bwork, &res = k->bres;
    DBuf<int> &info = k->binfo;
    DBuf<sfc_hparams_t> &h = k->bhp;
    work.reserve((size_t)chunk * wsz);
    res.reserve(chunk);
    info.reserve(chunk);
    std::vector<int> hinfo(chunk);
    for (int c0 = 0; c0 < n; c0 += chunk) {
        const int m = std::min(chunk, n - c0);
        upload(ctx, h, hps + c0, m);
        SFC_CK(cudaMemsetAsync(info.p, 0, m * sizeof(int), ctx->stream));
        k_koh_loglik_batch<<<m, 1024, 0, ctx->stream>>>(ns, k->n_o, fg->mean.p, fg->cov.p, k->sensor_coords.p, k->dim,
                                                        k->Y.p, h.p, wsz, work.p, res.p, info.p);
        count_launch(ctx);
        download(ctx, out + c0, res.p, m);
        download(ctx, hinfo.data(), info.p, m);
        for (int t = 0; t < m; ++t)
            if (hinfo[t]) out[c0 + t] = NAN;
    }
}

// LikelihoodKOH::giveProjFEconditionedData (LikelihoodKOH.ipp:311-361)
// computes Sigma = (rho^2 n_o K_s^-1 + C_s^-1)^-1 and
// m = Sigma (rho K_s^-1 sum_k y_k + C_s^-1 mean) with three explicit inverses.
// The same Sigma and m follow from the Woodbury identity the reference uses in
// giveFEconditionedDataWoodbury (:442-508) with P = I:
//   S = C_s + K_s / (rho^2 n_o) = L L^T,  [X | z] = L^-1 [C_s | ybar - rho mean],
//   Sigma = C_s - X^T X,  m = mean + X^T z / rho,
// which needs one Cholesky factor and triangular solves (backward stable)
// instead of the inverse of the ill-conditioned C_s: at the 48^3 elasticity
// configuration (cond C_s ~ 3e8, sensor noise 1e-4) Gauss-Jordan inverses of
// the three-inverse form left Sigma 8e-7 from the exact value, this form about
// 1e-9.  The factor and the solve are blocked by 32 (kChB): a one-CTA kernel
// per diagonal block, a row-parallel kernel per panel, the trailing updates
// on the multi-CTA gemm.
constexpr int kChB = 32;

// S = K_s / (rho^2 n_o) + C_s (ns x ns); W = [C_s | ybar - rho mean] (ns x (ns+1))
__global__ void k_koh_proj_setup(int ns, int n_o, const double *__restrict__ mean, const double *__restrict__ Cs,
                                 const double *__restrict__ xs, int dim, const double *__restrict__ Y,
                                 sfc_hparams_t hp, double *__restrict__ S, double *__restrict__ W)
{
    const double sc = 1.0 / (hp.rho * hp.rho * n_o);
    const int64_t nn = (int64_t)ns * ns;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn + ns; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < nn) {
            const int k = (int)(t / ns), l = (int)(t % ns);
            double kv = se_value(xs + 3 * k, xs + 3 * l, dim, hp.mismatch_sigma, hp.mismatch_length);
            if (k == l) kv += hp.mismatch_sensor_eps * hp.mismatch_sensor_eps;
            S[t] = kv * sc + Cs[t];
            W[(int64_t)k * (ns + 1) + l] = Cs[t];
        } else {
            const int i = (int)(t - nn);
            double ys = 0.0;
            for (int c = 0; c < n_o; ++c) ys += Y[(int64_t)i * n_o + c];
            W[(int64_t)i * (ns + 1) + ns] = ys / n_o - hp.rho * mean[i];
        }
    }
}

// in-place lower Cholesky of the kb x kb diagonal block at (k0, k0) of the
// n x n row-major A; a non-positive pivot sets *info (one CTA of 256)
__global__ void __launch_bounds__(256) k_chol_diag(double *A, int64_t n, int64_t k0, int kb, int *info)
{
    __shared__ double D[kChB][kChB + 1];
    __shared__ int bad;
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) D[t / kb][t % kb] = A[(k0 + t / kb) * n + k0 + t % kb];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < kb; ++k) {
        if (threadIdx.x == 0) {
            const double d = D[k][k];
            if (!(d > 0.0)) bad = 1;
            D[k][k] = d > 0.0 ? sqrt(d) : 1.0;
        }
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < kb; i += blockDim.x) D[i][k] /= D[k][k];
        __syncthreads();
        for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
            const int i = t / kb, j = t % kb;
            if (i > k && j > k && j <= i) D[i][j] -= D[i][k] * D[j][k];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
        const int i = t / kb, j = t % kb;
        if (j <= i) A[(k0 + i) * n + k0 + j] = D[i][j];
    }
    if (threadIdx.x == 0 && bad) atomicExch(info, 1);
}

// rows i >= k0 + kb of the panel: A[i, k0:k0+kb] <- A[i, k0:k0+kb] L_kk^-T
// (thread per row, L_kk staged in shared memory)
__global__ void __launch_bounds__(256) k_chol_panel(double *A, int64_t n, int64_t k0, int kb)
{
    __shared__ double L[kChB][kChB + 1];
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) L[t / kb][t % kb] = A[(k0 + t / kb) * n + k0 + t % kb];
    __syncthreads();
    const int64_t i = k0 + kb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x[kChB];
#pragma unroll
    for (int m = 0; m < kChB; ++m) x[m] = m < kb ? A[i * n + k0 + m] : 0.0;
#pragma unroll
    for (int m = 0; m < kChB; ++m) {
        if (m >= kb) break;
        double v = x[m];
        for (int q = 0; q < m; ++q) v -= x[q] * L[m][q];
        x[m] = v / L[m][m];
    }
#pragma unroll
    for (int m = 0; m < kChB; ++m)
        if (m < kb) A[i * n + k0 + m] = x[m];
}

// rows k0..k0+kb of W (ncols columns, leading dimension ldw):
// W_k <- L_kk^-1 W_k (thread per column)
__global__ void __launch_bounds__(256) k_trsm_block_rows(const double *A, int64_t n, int64_t k0, int kb, double *W,
                                                         int64_t ldw, int64_t ncols)
{
    __shared__ double L[kChB][kChB + 1];
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) L[t / kb][t % kb] = A[(k0 + t / kb) * n + k0 + t % kb];
    __syncthreads();
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    double x[kChB];
#pragma unroll
    for (int m = 0; m < kChB; ++m) x[m] = m < kb ? W[(k0 + m) * ldw + c] : 0.0;
#pragma unroll
    for (int m = 0; m < kChB; ++m) {
        if (m >= kb) break;
        double v = x[m];
        for (int q = 0; q < m; ++q) v -= L[m][q] * x[q];
        x[m] = v / L[m][m];
    }
#pragma unroll
    for (int m = 0; m < kChB; ++m)
        if (m < kb) W[(k0 + m) * ldw + c] = x[m];
}

void koh_proj(sfc_koh *k, const sfc_hparams_t *hp, double *mean, double *cov)
{
    sfc_ctx *ctx = k->ctx;
    sfc_forward_gauss *fg = k->fg;
    SFC_REQUIRE(fg->valid, "forward model not updated");
    SFC_REQUIRE(k->n_o > 0, "sensor values not set");
    const int ns = (int)k->ns, n_o = k->n_o;
    const int64_t nn = (int64_t)ns * ns;
    k->work.reserve((size_t)nn + (size_t)ns * (ns + 1) + 16);
    k->outv.reserve((size_t)ns + (size_t)nn);
    double *pm = k->outv.p, *pc = k->outv.p + ns;
    const double rho = hp->rho;
    {
        ProfScope ps(ctx, "phase:koh_posterior", 0.0);
        // S = C_s + K_s/(rho^2 n_o) = L L^T, [X | z] = L^-1 [C_s | ybar - rho mean];
        // Sigma = C_s - X^T X, m = mean + X^T z / rho
        SFC_REQUIRE(rho != 0.0, "rho must be nonzero");
        const int64_t ld = ns + 1;
        double *S = k->work.p, *W = S + nn;
        k->info.reserve(1);
        SFC_CK(cudaMemsetAsync(k->info.p, 0, sizeof(int), ctx->stream));
        k_koh_proj_setup<<<grid_for(nn + ns, 256), 256, 0, ctx->stream>>>(ns, n_o, fg->mean.p, fg->cov.p,
                                                                         k->sensor_coords.p, k->dim, k->Y.p, *hp, S, W);
        count_launch(ctx);
        for (int64_t k0 = 0; k0 < ns; k0 += kChB) {
            const int kb = (int)std::min<int64_t>(kChB, ns - k0);
            const int64_t k1 = k0 + kb;
            k_chol_diag<<<1, 256, 0, ctx->stream>>>(S, ns, k0, kb, k->info.p);
            count_launch(ctx);
            if (k1 < ns) {
                k_chol_panel<<<grid_for(ns - k1, 256), 256, 0, ctx->stream>>>(S, ns, k0, kb);
                count_launch(ctx);
                gemm(ctx, 0, 1, ns - k1, ns - k1, kb, -1.0, S + k1 * ns + k0, ns, S + k1 * ns + k0, ns, 1.0,
                     S + k1 * ns + k1, ns);
            }
        }
        for (int64_t k0 = 0; k0 < ns; k0 += kChB) {
            const int kb = (int)std::min<int64_t>(kChB, ns - k0);
            const int64_t k1 = k0 + kb;
            k_trsm_block_rows<<<grid_for(ld, 256), 256, 0, ctx->stream>>>(S, ns, k0, kb, W, ld, ld);
            count_launch(ctx);
            if (k1 < ns) gemm(ctx, 0, 0, ns - k1, ld, kb, -1.0, S + k1 * ns + k0, ns, W + k0 * ld, ld, 1.0, W + k1 * ld, ld);
        }
        int bad = 0;
        download(ctx, &bad, k->info.p, 1);
        if (bad) fail(SFC_ERR_NOT_SPD, "sensor-space matrix not positive definite (C_s + K_s / (rho^2 n_o))");
        SFC_CK(cudaMemcpyAsync(pc, fg->cov.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        SFC_CK(cudaMemcpyAsync(pm, fg->mean.p, ns * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        gemm(ctx, 1, 0, ns, ns, ns, -1.0, W, ld, W, ld, 1.0, pc, ns);
        gemm(ctx, 1, 0, ns, 1, ns, 1.0 / rho, W, ld, W + ns, ld, 1.0, pm, 1);
    }
    if (mean) download(ctx, mean, pm, ns);
    if (cov) download(ctx, cov, pc, (size_t)nn);
    SFC_CK(cudaStreamSynchronize(ctx->stream));
}

// lower Cholesky in place (n x n, row-major); false when not positive definite
static bool host_chol(std::vector<double> &A, int n)
{
    for (int j = 0; j < n; ++j) {
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double v = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = v / d;
        }
    }
    return true;
}

// x := (L L^T)^-1 x
static void host_chol_solve(const std::vector<double> &L, int n, std::vector<double> &x)
{
    for (int i = 0; i < n; ++i) {
        double v = x[i];
        for (int k = 0; k < i; ++k) v -= L[(size_t)i * n + k] * x[k];
        x[i] = v / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double v = x[i];
        for (int k = i + 1; k < n; ++k) v -= L[(size_t)k * n + i] * x[k];
        x[i] = v / L[(size_t)i * n + i];
    }
}

// The posterior mean field of giveFEconditionedDataWoodbury
// (LikelihoodKOH.ipp:442-508) at sensor-space cost.  With G = C_u P^T,
// S = K_s/(rho^2 n_o) + C_s and P G = C_s, P ubar = mean_s:
//   D (rho G K_s^-1 ysum + ubar) = ubar + G w,
//   w = rho K_s^-1 ysum - S^-1 (rho C_s K_s^-1 ysum + mean_s),
// and G = A^-1 (C_f R^T) + (sigma_f reg)^2 P^T from the adjoint solution
// R^T = A^-T P^T already at hand: ns forward solves and one forward solve for
// ubar = A^-1 F instead of the N solves of the unprojected prior.
void koh_woodbury_mean(sfc_koh *k, const sfc_hparams_t *hp, double *mean)
{
    sfc_ctx *ctx = k->ctx;
    sfc_forward_gauss *fg = k->fg;
    sfc_system *s = fg->sys;
    SFC_REQUIRE(fg->valid, "forward model not updated");
    SFC_REQUIRE(k->n_o > 0, "sensor values not set");
    const int64_t N = s->N, ns = fg->ns;
    const int n = (int)ns, n_o = k->n_o;
    const double rho = hp->rho;
    // sensor space on the host (FP64 Cholesky, ns x ns)
    std::vector<double> Cs((size_t)ns * ns), ms(ns), Y((size_t)ns * n_o), xy((size_t)ns * 3);
    download(ctx, Cs.data(), fg->cov.p, Cs.size());
    download(ctx, ms.data(), fg->mean.p, ms.size());
    download(ctx, Y.data(), k->Y.p, Y.size());
    download(ctx, xy.data(), k->sensor_coords.p, xy.size());
    std::vector<double> Ks((size_t)ns * ns);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            double d2 = 0.0;
            for (int c = 0; c < k->dim; ++c) {
                const double t = xy[(size_t)a * 3 + c] - xy[(size_t)b * 3 + c];
                d2 += t * t;
            }
            Ks[(size_t)a * n + b] = hp->mismatch_sigma * hp->mismatch_sigma *
                                        std::exp(-d2 / (2.0 * hp->mismatch_length * hp->mismatch_length)) +
                                    (a == b ? hp->mismatch_sensor_eps * hp->mismatch_sensor_eps : 0.0);
        }
    std::vector<double> S(Ks);
    for (size_t t = 0; t < S.size(); ++t) S[t] = Ks[t] / (rho * rho * n_o) + Cs[t];
    std::vector<double> Lk(Ks), Ls(S);
    if (!host_chol(Lk, n) || !host_chol(Ls, n)) fail(SFC_ERR_NOT_SPD, "sensor-space matrix not positive definite");
    std::vector<double> kys(ns, 0.0);  // K_s^-1 ysum
    for (int a = 0; a < n; ++a)
        for (int j = 0; j < n_o; ++j) kys[a] += Y[(size_t)a * n_o + j];
    host_chol_solve(Lk, n, kys);
    std::vector<double> t(ns), w(ns);
    for (int a = 0; a < n; ++a) {
        double v = ms[a];
        for (int b = 0; b < n; ++b) v += rho * Cs[(size_t)a * n + b] * kys[b];
        t[a] = v;
    }
    host_chol_solve(Ls, n, t);
    for (int a = 0; a < n; ++a) w[a] = rho * kys[a] - t[a];
    // ubar = A^-1 F (forward solve, the system's own method)
    solve_forward(s);
    // G = A^-1 (C_f R^T) + (sigma_f reg)^2 P^T
    DBuf<double> W, T, G, wd, out;
    W.alloc(N * ns);
    T.alloc(3 * N * ns);
    G.alloc(N * ns);
    k_scale_rows<<<grid_for(N * ns, 256), 256, 0, ctx->stream>>>(fg->R.p, fg->cf->phibar.p, N, ns, W.p);
    count_launch(ctx);
    kernel_times(ctx, fg->cf, hp->forcing_sigma, hp->forcing_length, W.p, T.p, ns, T.p + N * ns);
    k_scale_rows<<<grid_for(N * ns, 256), 256, 0, ctx->stream>>>(T.p, fg->cf->phibar.p, N, ns, W.p);
    count_launch(ctx);
    solve_multi(s, W.p, G.p, (int)ns, (int)ns);
    const double add = hp->forcing_sigma * fg->reg;
    k_add_scaled<<<grid_for(N * ns, 256), 256, 0, ctx->stream>>>(G.p, fg->B.p, add * add, N * ns);
    count_launch(ctx);
    // mean = ubar + G w
    upload(ctx, wd, w.data(), ns);
    out.alloc(N);
    SFC_CK(cudaMemcpyAsync(out.p, s->X.p, N * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    gemm(ctx, 0, 0, N, 1, ns, 1.0, G.p, ns, wd.p, 1, 1.0, out.p, 1);
    download(ctx, mean, out.p, N);
}

// giveFEconditionedDataWoodbury (LikelihoodKOH.ipp:442-508)
void koh_woodbury(sfc_koh *k, const sfc_hparams_t *hp, double *mean, double *cov)
{
    sfc_ctx *ctx = k->ctx;
    sfc_forward_gauss *fg = k->fg;
    sfc_system *s = fg->sys;
    SFC_REQUIRE(fg->valid, "forward model not updated");
    SFC_REQUIRE(k->n_o > 0, "sensor values not set");
    const int64_t N = s->N, ns = fg->ns;
    SFC_REQUIRE(N <= 8192, "full-field Woodbury posterior limited to 8192 dofs");
    const double rho = hp->rho;
    const int n_o = k->n_o;
    // K_s, K_s^-1, S = K_s/(rho^2 n_o) + C_s, S^-1
    DBuf<double> Ks, Ksi, Si, ysum, P;
    Ks.alloc(ns * ns);
    Ksi.alloc(ns * ns);
    Si.alloc(ns * ns);
    ysum.alloc(ns);
    k_mismatch<<<1, 1024, 0, ctx->stream>>>((int)ns, k->sensor_coords.p, k->dim, *hp, Ks.p);
    SFC_CK(cudaMemcpyAsync(Ksi.p, Ks.p, ns * ns * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    SFC_CK(cudaMemcpyAsync(Si.p, fg->cov.p, ns * ns * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    k_add_scaled<<<grid_for(ns * ns, 256), 256, 0, ctx->stream>>>(Si.p, Ks.p, 1.0 / (rho * rho * n_o), ns * ns);
    k_rowsum<<<1, 256, 0, ctx->stream>>>(k->Y.p, ns, n_o, ysum.p);
    count_launch(ctx, 3);
    int d1 = 0, d2 = 0;
    spd_inverse_gj(ctx, Ksi.p, ns, 0.0, k->gj, nullptr, &d1);
    spd_inverse_gj(ctx, Si.p, ns, 0.0, k->gj, nullptr, &d2);
    if (d1 || d2) fail(SFC_ERR_NOT_SPD, "sensor-space matrix not invertible");
    // dense P (ns x N)
    std::vector<double> hP((size_t)ns * N, 0.0);
    for (int64_t a = 0; a < ns; ++a)
        for (int64_t t = fg->p_ptr[a]; t < fg->p_ptr[a + 1]; ++t) hP[(size_t)a * N + fg->p_idx[t]] += fg->p_val[t];
    upload(ctx, P, hP.data(), hP.size());
    // unprojected prior: R_I^T = A^-T I (N adjoint solves), C_u, u-bar
    DBuf<double> I, RI, Cu, ubar;
    std::vector<double> hI((size_t)N * N, 0.0);
    for (int64_t i = 0; i < N; ++i) hI[(size_t)i * N + i] = 1.0;
    upload(ctx, I, hI.data(), hI.size());
    RI.alloc(N * N);
    solve_block(s, I.p, RI.p, (int)N, (int)N);
    transpose_fixup(s, I.p, RI.p, (int)N, (int)N);
    ubar.alloc(N);
    k_colsum_dot<<<(unsigned)std::min<int64_t>(N, 1024), 256, 0, ctx->stream>>>(RI.p, s->F.p, N, N, ubar.p);
    count_launch(ctx);
    Cu.alloc(N * N);
    DBuf<double> work;
    projected_covar(ctx, fg->cf, hp->forcing_sigma, hp->forcing_length, RI.p, N, Cu.p, work);
    const double add = hp->forcing_sigma * fg->reg;
    // + (sigma_f reg)^2 I  (P = I in the unprojected update)
    k_add_scaled<<<grid_for(N * N, 256), 256, 0, ctx->stream>>>(Cu.p, I.p, add * add, N * N);
    count_launch(ctx);
    // G = C_u P^T (N x ns); H = G S^-1 (N x ns); D = I - H P (N x N)
    DBuf<double> G, H, D, t1, t2;
    G.alloc(N * ns);
    H.alloc(N * ns);
    D.alloc(N * N);
    gemm(ctx, 0, 1, N, ns, N, 1.0, Cu.p, N, P.p, N, 0.0, G.p, ns);
    gemm(ctx, 0, 0, N, ns, ns, 1.0, G.p, ns, Si.p, ns, 0.0, H.p, ns);
    gemm(ctx, 0, 0, N, N, ns, 1.0, H.p, ns, P.p, N, 0.0, D.p, N);
    k_identity_minus<<<grid_for(N * N, 256), 256, 0, ctx->stream>>>(D.p, N);
    count_launch(ctx);
    // vecA = rho G K_s^-1 ysum ; mean = D (vecA + ubar)
    t1.alloc(ns);
    t2.alloc(N);
    gemm(ctx, 0, 0, ns, 1, ns, 1.0, Ksi.p, ns, ysum.p, 1, 0.0, t1.p, 1);
    SFC_CK(cudaMemcpyAsync(t2.p, ubar.p, N * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    gemm(ctx, 0, 0, N, 1, ns, rho, G.p, ns, t1.p, 1, 1.0, t2.p, 1);
    DBuf<double> pm;
    pm.alloc(N);
    gemm(ctx, 0, 0, N, 1, N, 1.0, D.p, N, t2.p, 1, 0.0, pm.p, 1);
    if (mean) download(ctx, mean, pm.p, N);
    if (cov) {
        DBuf<double> pc;
        pc.alloc(N * N);
        gemm(ctx, 0, 0, N, N, N, 1.0, D.p, N, Cu.p, N, 0.0, pc.p, N);
        download(ctx, cov, pc.p, N * N);
    }
    SFC_CK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace sfc
