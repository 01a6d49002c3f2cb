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

constexpr int kGJ = 32;         // panel width
constexpr int kPanelCols = 64;  // columns per CTA of the panel kernel

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
    // warp 0 inverts the diagonal block in registers: lane c holds column c
    if (threadIdx.x < 32) {
        const int c = threadIdx.x;
        double col[kGJ];
#pragma unroll
        for (int r = 0; r < kGJ; ++r) col[r] = (r < kb && c < kb) ? A[(k0 + r) * n + k0 + c] : 0.0;
        int ndrop = 0;
        const double ad = c < kb ? adiag[k0 + c] : 0.0;  // lane p's is broadcast at pivot p
        for (int p = 0; p < kb; ++p) {
            // pivot = D[p][p] (lane p), column p of D (lane p's registers)
            double piv = 0.0, colv[kGJ];
#pragma unroll
            for (int r = 0; r < kGJ; ++r) {
                colv[r] = __shfl_sync(0xffffffffu, col[r], p);
                if (r == p) piv = colv[r];
            }
            const bool drop = !(piv > rel * __shfl_sync(0xffffffffu, ad, p));
            if (pivots && blockIdx.x == 0 && c == 0) pivots[k0 + p] = piv;
            double rowp_c = 0.0;  // D[p][c]
#pragma unroll
            for (int r = 0; r < kGJ; ++r)
                if (r == p) rowp_c = col[r];
            if (drop) {
                ++ndrop;
#pragma unroll
                for (int r = 0; r < kGJ; ++r)
                    if (r == p || c == p) col[r] = 0.0;
            } else {
                const double ip = 1.0 / piv;
#pragma unroll
                for (int r = 0; r < kGJ; ++r) {
                    double v;
                    if (r == p && c == p)
                        v = ip;
                    else if (r == p)
                        v = rowp_c * ip;
                    else if (c == p)
                        v = -colv[r] * ip;
                    else
                        v = col[r] - colv[r] * (rowp_c * ip);
                    col[r] = v;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kGJ; ++r) D[r][c] = col[r];
        if (blockIdx.x == 0 && c == 0 && ndrop) atomicAdd(dropped, ndrop);
    }
    __syncthreads();
    // this CTA's 64 columns j0.. (and rows, for the column panel)
    __shared__ double T[kGJ][kPanelCols + 1];
    const int64_t j0 = (int64_t)blockIdx.x * kPanelCols;
    for (int t = threadIdx.x; t < kPanelCols * kGJ; t += blockDim.x) {
        const int jj = t / kGJ, m = t % kGJ;  // m fastest: row j0 + jj of A read contiguously
        const int64_t j = j0 + jj;
        if (j < n && m < kb) colp[j * kGJ + m] = A[j * n + k0 + m];
        const int l = t / kPanelCols, c = t % kPanelCols;
        T[l][c] = (l < kb && j0 + c < n) ? A[(k0 + l) * n + j0 + c] : 0.0;
    }
    __syncthreads();
    const int c = threadIdx.x % kPanelCols, mg = threadIdx.x / kPanelCols;  // 4 groups of 8 rows of D^-1
    const int64_t j = j0 + c;
    if (j < n) {
        const bool inside = j >= k0 && j < k0 + kb;
#pragma unroll
        for (int u = 0; u < kGJ / 4; ++u) {
            const int m = mg * (kGJ / 4) + u;
            if (m >= kb) continue;
            double v;
            if (inside) {
                v = D[m][j - k0];
            } else {
                v = 0.0;
#pragma unroll 8
                for (int l = 0; l < kGJ; ++l) v += D[m][l] * T[l][c];
            }
            rowp[m * n + j] = v;
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
    {  // all 16 loads of a thread in flight before the stores (launched with 256 threads)
        double vc[64 * kGJ / 256], vr[64 * kGJ / 256];
#pragma unroll
        for (int u = 0; u < 64 * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u;
            const int r = t / kGJ, m = t % kGJ;
            vc[u] = (i0 + r < n && m < kb) ? colp[(i0 + r) * kGJ + m] : 0.0;
            const int mm = t / 64, c = t % 64;
            vr[u] = (j0 + c < n && mm < kb) ? rowp[mm * n + j0 + c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 64 * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u;
            cp[t / kGJ][t % kGJ] = vc[u];
            rp[t / 64][t % 64] = vr[u];
        }
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

void GjScratch::drop_graphs()
{
    for (auto &g : graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs.clear();
}

GjScratch::~GjScratch() { drop_graphs(); }

void GjScratch::reserve(int64_t n)
{
    if ((size_t)n > diag.n || (size_t)(kGJ * n) > rowp.n || !word.p) drop_graphs();  // buffers move
    diag.reserve(n);
    rowp.reserve(kGJ * n);
    colp.reserve(kGJ * n);
    word.reserve(1);
}

namespace {
void gj_enqueue(cudaStream_t st, double *A, int64_t n, double rel, GjScratch &w, double *pivots)
{
    k_diag_of<<<grid_for(n, 256), 256, 0, st>>>(A, n, w.diag.p);
    cudaMemsetAsync(w.word.p, 0, sizeof(int), st);
    const unsigned gp = (unsigned)((n + kPanelCols - 1) / kPanelCols), gt = (unsigned)((n + 63) / 64);
    for (int64_t k0 = 0; k0 < n; k0 += kGJ) {
        const int kb = (int)std::min<int64_t>(kGJ, n - k0);
        k_gj_panel<<<gp, 256, 0, st>>>(A, n, k0, kb, w.diag.p, rel, w.rowp.p, w.colp.p, w.word.p, pivots);
        k_gj_update<<<dim3(gt, gt), 256, 0, st>>>(A, n, k0, kb, w.rowp.p, w.colp.p);
    }
}
}  // namespace

// The launch sequence of one inverse depends only on (A, n, rel, pivots) and
// the scratch buffers, so it is captured once into a CUDA graph and replayed
// (2 n / 32 + 1 short launches would otherwise be host-bound).
void spd_inverse_gj(sfc_ctx *ctx, double *A, int64_t n, double rel, GjScratch &w, double *pivots, int *dropped)
{
    w.reserve(n);
    const int nlaunch = 1 + 2 * (int)((n + kGJ - 1) / kGJ);
    GjScratch::Graph *g = nullptr;
    for (auto &e : w.graphs)
        if (e.A == A && e.n == n && e.rel == rel && e.pivots == pivots) g = &e;
    if (!g) {
        if (w.graphs.size() >= 8) w.drop_graphs();
        cudaStream_t st;
        SFC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            gj_enqueue(st, A, n, rel, w, pivots);
            e = cudaStreamEndCapture(st, &graph);
        }
        cudaStreamDestroy(st);
        SFC_CK(e);
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        SFC_CK(e);
        w.graphs.push_back({A, n, rel, pivots, exec});
        g = &w.graphs.back();
    }
    SFC_CK(cudaGraphLaunch(g->exec, ctx->stream));
    count_launch(ctx, nlaunch);
    int h = 0;
    download(ctx, &h, w.word.p, 1);
    if (dropped) *dropped = h;
}

}  // namespace sfc
