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
    // launched with 256 threads
    __shared__ double D[2][kGJ][kGJ + 1];
    __shared__ double T[kGJ][kPanelCols + 1];
    __shared__ double sad[kGJ];
    const int64_t j0 = (int64_t)blockIdx.x * kPanelCols;
    if (threadIdx.x < kGJ) sad[threadIdx.x] = threadIdx.x < kb ? adiag[k0 + threadIdx.x] : 0.0;
    // stage the diagonal block, this CTA's 64 columns of the row panel and its
    // 64 rows of the column panel, every load of a thread in flight together
    {
        double vd[kGJ * kGJ / 256], vt[kPanelCols * kGJ / 256], vc[kPanelCols * kGJ / 256];
#pragma unroll
        for (int u = 0; u < kGJ * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u, r = t / kGJ, c = t % kGJ;
            vd[u] = (r < kb && c < kb) ? A[(k0 + r) * n + k0 + c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kPanelCols * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u;
            const int l = t / kPanelCols, c = t % kPanelCols;
            vt[u] = (l < kb && j0 + c < n) ? A[(k0 + l) * n + j0 + c] : 0.0;
            const int jj = t / kGJ, m = t % kGJ;  // m fastest: row j0 + jj of A read contiguously
            vc[u] = (j0 + jj < n && m < kb) ? A[(j0 + jj) * n + k0 + m] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kGJ * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u;
            D[0][t / kGJ][t % kGJ] = vd[u];
        }
#pragma unroll
        for (int u = 0; u < kPanelCols * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u;
            T[t / kPanelCols][t % kPanelCols] = vt[u];
            const int jj = t / kGJ, m = t % kGJ;
            if (j0 + jj < n && m < kb) colp[(j0 + jj) * kGJ + m] = vc[u];
        }
    }
    __syncthreads();
    // Gauss-Jordan on the diagonal block: every thread owns 4 entries, reads
    // buffer cur and writes the other, one barrier per pivot; the drop test
    // is evaluated identically by every thread
    int cur = 0, ndrop = 0;
    for (int p = 0; p < kb; ++p) {
        const double piv = D[cur][p][p];
        const bool drop = !(piv > rel * sad[p]);
        if (pivots && blockIdx.x == 0 && threadIdx.x == 0) pivots[k0 + p] = piv;
        ndrop += drop;
        const double ip = drop ? 0.0 : 1.0 / piv;
#pragma unroll
        for (int u = 0; u < kGJ * kGJ / 256; ++u) {
            const int t = threadIdx.x + 256 * u, r = t / kGJ, c = t % kGJ;
            double v;
            if (drop)
                v = (r == p || c == p) ? 0.0 : D[cur][r][c];
            else if (r == p && c == p)
                v = ip;
            else if (r == p)
                v = D[cur][p][c] * ip;
            else if (c == p)
                v = -D[cur][r][p] * ip;
            else
                v = D[cur][r][c] - D[cur][r][p] * (D[cur][p][c] * ip);
            D[cur ^ 1][r][c] = v;
        }
        cur ^= 1;
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && ndrop) atomicAdd(dropped, ndrop);
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
                v = D[cur][m][j - k0];
            } else {
                v = 0.0;
#pragma unroll 8
                for (int l = 0; l < kGJ; ++l) v += D[cur][m][l] * T[l][c];
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
    ++ctx->graph_replays;
    int h = 0;
    download(ctx, &h, w.word.p, 1);
    if (dropped) *dropped = h;
}

}  // namespace sfc
