// Dense FP64 inverse of a symmetric positive (semi)definite matrix by block
// Gauss-Jordan elimination without pivoting, on the GPU: the in-place form
//     A[k,k] <- D^-1,  A[k,j] <- D^-1 A[k,j],  A[i,k] <- -A[i,k] D^-1,
//     A[i,j] <- A[i,j] - A[i,k] D^-1 A[k,j]
// for 32-wide panels k (D the panel's diagonal block), two launches per
// panel.  Used for the coarse matrix of the two-level preconditioner (with
// dependent pivots dropped: a generalised inverse on the independent modes)
// and for the sensor-space matrices of the KOH likelihood and posterior
// (LikelihoodKOH.ipp:75-120, 311-361), where a non-positive pivot is the
// reference's failed LLT.  The Schur-complement pivots are the squared
// diagonal of the Cholesky factor, so their logarithms sum to log det A.

#include <algorithm>

#include "common.cuh"

namespace sfc {

namespace {

constexpr int kGJ = 32;  // panel width

__global__ void k_diag_of(const double *__restrict__ A, int64_t n, double *__restrict__ d)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = A[i * n + i];
}

// Gauss-Jordan step, part 1: invert the kb x kb diagonal block D of panel k0
// (in shared memory, every CTA redundantly; a pivot that is not above
// rel x the dof's original diagonal is dropped: its row and column are
// zeroed), save the old column panel colp[i][m] = A[i][k0+m] and form the new
// row panel rowp[m][j] = (D^-1 A[k0.., j])[m] (= D^-1 itself inside the block).
__global__ void __launch_bounds__(256) k_gj_panel(const double *__restrict__ A, int64_t n, int64_t k0, int kb,
                                                  const double *__restrict__ adiag, double rel, double *__restrict__ rowp,
                                                  double *__restrict__ colp, int *dropped, double *pivots)
{
    __shared__ double D[kGJ][kGJ + 1];
    __shared__ double rowv[kGJ], colv[kGJ];
    __shared__ int drop;
    for (int t = threadIdx.x; t < kGJ * kGJ; t += blockDim.x) {
        const int r = t / kGJ, c = t % kGJ;
        D[r][c] = (r < kb && c < kb) ? A[(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    for (int p = 0; p < kb; ++p) {
        if (threadIdx.x == 0) {
            const double piv = D[p][p];
            drop = !(piv > rel * adiag[k0 + p]);
            if (pivots && blockIdx.x == 0) pivots[k0 + p] = piv;
        }
        if (threadIdx.x < kGJ) {
            rowv[threadIdx.x] = D[p][threadIdx.x];
            colv[threadIdx.x] = D[threadIdx.x][p];
        }
        __syncthreads();
        const double piv = rowv[p];
        for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
            const int r = t / kb, c = t % kb;
            double v;
            if (drop)
                v = (r == p || c == p) ? 0.0 : D[r][c];
            else if (r == p && c == p)
                v = 1.0 / piv;
            else if (r == p)
                v = rowv[c] / piv;
            else if (c == p)
                v = -colv[r] / piv;
            else
                v = D[r][c] - colv[r] * rowv[c] / piv;
            D[r][c] = v;
        }
        if (drop && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(dropped, 1);
        __syncthreads();
    }
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        for (int m = 0; m < kb; ++m) colp[j * kGJ + m] = A[j * n + k0 + m];
        if (j >= k0 && j < k0 + kb) {
            for (int m = 0; m < kb; ++m) rowp[m * n + j] = D[m][j - k0];
        } else {
            double aj[kGJ];
#pragma unroll
            for (int l = 0; l < kGJ; ++l) aj[l] = l < kb ? A[(k0 + l) * n + j] : 0.0;
            for (int m = 0; m < kb; ++m) {
                double s = 0.0;
#pragma unroll
                for (int l = 0; l < kGJ; ++l) s += D[m][l] * aj[l];
                rowp[m * n + j] = s;
            }
        }
    }
}

// Gauss-Jordan step, part 2 (64 x 64 tile per CTA):
//   rows of the panel:     A[i][j] = rowp[i-k0][j]
//   columns of the panel:  A[i][j] = -colp[i] . rowp[:, j]   (= -A[i,k] D^-1)
//   elsewhere:             A[i][j] -= colp[i] . rowp[:, j]
__global__ void __launch_bounds__(256) k_gj_update(double *__restrict__ A, int64_t n, int64_t k0, int kb,
                                                   const double *__restrict__ rowp, const double *__restrict__ colp)
{
    __shared__ double cp[64][kGJ + 1];
    __shared__ double rp[kGJ][64 + 1];
    const int64_t i0 = (int64_t)blockIdx.y * 64, j0 = (int64_t)blockIdx.x * 64;
    for (int t = threadIdx.x; t < 64 * kGJ; t += blockDim.x) {
        const int r = t / kGJ, m = t % kGJ;
        cp[r][m] = (i0 + r < n && m < kb) ? colp[(i0 + r) * kGJ + m] : 0.0;
        const int mm = t / 64, c = t % 64;
        rp[mm][c] = (j0 + c < n && mm < kb) ? rowp[mm * n + j0 + c] : 0.0;
    }
    __syncthreads();
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    for (int u = 0; u < 4; ++u) {
        const int64_t i = i0 + ty + 16 * u;
        if (i >= n) continue;
        for (int v = 0; v < 4; ++v) {
            const int64_t j = j0 + tx + 16 * v;
            if (j >= n) continue;
            if (i >= k0 && i < k0 + kb) {
                A[i * n + j] = rp[i - k0][tx + 16 * v];
                continue;
            }
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < kGJ; ++m) s += cp[ty + 16 * u][m] * rp[m][tx + 16 * v];
            A[i * n + j] = (j >= k0 && j < k0 + kb) ? -s : A[i * n + j] - s;
        }
    }
}


}  // namespace

void GjScratch::reserve(int64_t n)
{
    diag.reserve(n);
    rowp.reserve(kGJ * n);
    colp.reserve(kGJ * n);
    word.reserve(1);
}

void spd_inverse_gj(sfc_ctx *ctx, double *A, int64_t n, double rel, GjScratch &w, double *pivots, int *dropped)
{
    w.reserve(n);
    k_diag_of<<<grid_for(n, 256), 256, 0, ctx->stream>>>(A, n, w.diag.p);
    SFC_CK(cudaMemsetAsync(w.word.p, 0, sizeof(int), ctx->stream));
    count_launch(ctx);
    const unsigned gp = grid_for(n, 256), gt = (unsigned)((n + 63) / 64);
    for (int64_t k0 = 0; k0 < n; k0 += kGJ) {
        const int kb = (int)std::min<int64_t>(kGJ, n - k0);
        k_gj_panel<<<gp, 256, 0, ctx->stream>>>(A, n, k0, kb, w.diag.p, rel, w.rowp.p, w.colp.p, w.word.p, pivots);
        k_gj_update<<<dim3(gt, gt), 256, 0, ctx->stream>>>(A, n, k0, kb, w.rowp.p, w.colp.p);
        count_launch(ctx, 2);
    }
    int h = 0;
    download(ctx, &h, w.word.p, 1);
    if (dropped) *dropped = h;
}

}  // namespace sfc
