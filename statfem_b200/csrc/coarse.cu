// Two-level preconditioner: the nodal 3x3 block-Jacobi smoother (elasticity)
// or point Jacobi (scalar Poisson meshes) plus an additive coarse correction
// on the rigid-body modes (elasticity) or the constant (Poisson) of
// geometric aggregates,
//
//     M^-1 r = D^-1 r + P A_c^+ P^T r,     A_c = P^T S P,
//
// where P holds, for every aggregate (a box of nodes), its six rigid-body
// modes (three translations and three rotations about the aggregate's
// centroid), zero on constrained dofs, and A_c^+ is the inverse of the
// Galerkin matrix on the span of the modes that are not numerically dependent.
// Both terms are symmetric positive (semi)definite and the first is definite,
// so M is SPD and plain PCG applies.  The reference solves with a direct
// factorisation (corlib/SystemSolveEigenSparse.hpp:273-404); this is the
// iterative replacement's stronger preconditioner: block Jacobi alone needs a
// number of iterations that grows with the mesh size, the coarse space removes
// the smooth, nearly rigid error components that it cannot reach.
//
// Layout and cost per iteration (K right-hand sides, nc = 6 x aggregates):
//  * k_coarse_restrict32: c = P^T r, a cluster of CTAs per aggregate (a
//    version fused into the x/r update ran slower: its register count halved
//    the resident warps);
//  * k_coarse_gemm32: e = A_c^+ c (FP32, dense, L2-resident, a tiled product
//    split over k across a cluster) and the coarse share c.e of each
//    column's r.z;
//  * the p update (solvers.cu) adds z += P e on the fly from each node's
//    aggregate id and centroid offset (k_ncpupdate32; k_cbpupdate32 on scalar
//    meshes).
// Setup per operator: the Galerkin product on the GPU (a cluster of CTAs per
// aggregate, FP64, deterministic), then the inverse by block Gauss-Jordan
// elimination (dense.cu: FP64, 32-wide panels, one CUDA graph) with dependent
// pivots dropped.  Scalar meshes take one constant mode per aggregate, point
// Jacobi as the smoother and the CSR operator in the Galerkin product.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <new>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"

namespace sfc {

namespace {

namespace cg = cooperative_groups;

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int kSlots = 27;   // 3 x 3 x 3 colour classes of the box grid
constexpr int kMaxAggs = 512;    // 3-dof meshes: 6 coarse dofs per aggregate
constexpr int kMaxAggs1 = 2048;  // scalar meshes: 1 coarse dof per aggregate

// R(d): column k is e_k x d (the displacement of rotation mode k at offset d)
__device__ __forceinline__ void rot_matrix(const float4 m, double (&R)[9])
{
    const double dx = m.x, dy = m.y, dz = m.z;
    // rows: components; columns: rotation axes
    R[0] = 0.0;  R[1] = dz;   R[2] = -dy;
    R[3] = -dz;  R[4] = 0.0;  R[5] = dx;
    R[6] = dy;   R[7] = -dx;  R[8] = 0.0;
}

__device__ __forceinline__ int mask_bits(const float4 m) { return (int)m.w; }

// per node: offset from its aggregate's centroid in units of the box edge
// (x, y, z) and the constrained components as bits in w
__global__ void k_coarse_modes(const float4 *__restrict__ offset, const unsigned char *__restrict__ mask,
                               int64_t nodes, int dof, float4 *__restrict__ mode)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        float4 m = offset[i];
        const int bits = dof == 1 ? (mask[i] ? 1 : 0)
                                  : (mask[3 * i] ? 1 : 0) | (mask[3 * i + 1] ? 2 : 0) | (mask[3 * i + 2] ? 4 : 0);
        m.w = (float)bits;
        mode[i] = m;
    }
}

// A_c = P^T S P.  A cluster of kGalSplit CTAs of kGalWarps warps per
// aggregate a: a warp takes a node i of a, its lanes the blocks (i, j) of S, and each lane forms the 6 x 6
// product M_i^T S_ij M_j (M = diag(free) [I | R(d)]) for the colour class of
// j's aggregate (unique among a's neighbours).  Lanes with the same class
// are summed by warp shuffles (the 27 blocks of a node reach at most 8
// classes) into the warp's own accumulators; the cluster's warp accumulators
// are added in a fixed order at the end (through distributed shared memory),
// so the result is deterministic.
constexpr int kGalWarps = 4;
constexpr int kGalSplit = 4;

__device__ __forceinline__ double warp_sum_masked(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __cluster_dims__(kGalSplit, 1, 1) __launch_bounds__(32 * kGalWarps) k_coarse_galerkin(const int32_t *__restrict__ agg_ptr,
                                                                    const int32_t *__restrict__ agg_nodes,
                                                                    const int32_t *__restrict__ node_agg,
                                                                    const int32_t *__restrict__ agg_slot,
                                                                    const int32_t *__restrict__ nbr,
                                                                    const float4 *__restrict__ mode,
                                                                    const int32_t *__restrict__ bptr,
                                                                    const int32_t *__restrict__ bcol,
                                                                    const double *__restrict__ bval, int64_t nc,
                                                                    double *__restrict__ A)
{
    __shared__ double acc[kGalWarps][kSlots * 36];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int a = blockIdx.x / kGalSplit;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kGalWarps * kSlots * 36; t += blockDim.x) (&acc[0][0])[t] = 0.0;
    __syncthreads();
    for (int32_t t = agg_ptr[a] + (int32_t)rank * kGalWarps + w; t < agg_ptr[a + 1]; t += kGalWarps * kGalSplit) {
        const int32_t i = agg_nodes[t];
        const float4 mi = mode[i];
        double Ri[9];
        rot_matrix(mi, Ri);
        const int bi = mask_bits(mi);
        for (int32_t b0 = bptr[i]; b0 < bptr[i + 1]; b0 += 32) {
            const int32_t b = b0 + lane;
            const bool has = b < bptr[i + 1];
            double G[36];
            int slot = -1;
            if (has) {
                const int32_t j = bcol[b];
                const float4 mj = mode[j];
                double Rj[9];
                rot_matrix(mj, Rj);
                const int bj = mask_bits(mj);
                slot = agg_slot[node_agg[j]];
                double Sp[9];
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        Sp[3 * r + c] = ((bi >> r) & 1) || ((bj >> c) & 1) ? 0.0 : bval[9 * (int64_t)b + 3 * r + c];
                // G = [[S', S' R_j], [R_i^T S', R_i^T S' R_j]]
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double u = Sp[3 * r] * Rj[k] + Sp[3 * r + 1] * Rj[3 + k] + Sp[3 * r + 2] * Rj[6 + k];
                        G[r * 6 + k] = Sp[3 * r + k];
                        G[r * 6 + 3 + k] = u;
                        G[(3 + r) * 6 + k] = Ri[r] * Sp[k] + Ri[3 + r] * Sp[3 + k] + Ri[6 + r] * Sp[6 + k];
                    }
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        G[(3 + r) * 6 + 3 + k] = Ri[r] * G[3 + k] + Ri[3 + r] * G[6 + 3 + k] + Ri[6 + r] * G[12 + 3 + k];
            } else {
#pragma unroll
                for (int m = 0; m < 36; ++m) G[m] = 0.0;
            }
            // segmented sum over the lanes of each colour class present
            unsigned left = __ballot_sync(0xffffffffu, has);
            while (left) {
                const int leader = __ffs(left) - 1;
                const int cls = __shfl_sync(0xffffffffu, slot, leader);
                const bool mine = has && slot == cls;
                left &= ~__ballot_sync(0xffffffffu, mine);
                double keep = 0.0;
#pragma unroll
                for (int m = 0; m < 36; ++m) {
                    const double v = warp_sum_masked(mine ? G[m] : 0.0);
                    if (lane == (m & 31)) keep = (m < 32) ? v : keep;
                    if (m >= 32 && lane == m - 32) acc[w][cls * 36 + m] += v;
                }
                acc[w][cls * 36 + lane] += keep;
            }
        }
    }
    cl.sync();
    for (int t = (int)rank * blockDim.x + threadIdx.x; t < kSlots * 36; t += kGalSplit * blockDim.x) {
        const int slot = t / 36, mk = t - slot * 36;
        const int32_t b = nbr[kSlots * a + slot];
        if (b < 0) continue;
        double sum = 0.0;
        for (unsigned r = 0; r < kGalSplit; ++r) {
            const double *ra = cl.map_shared_rank(&acc[0][0], r);
#pragma unroll
            for (int q = 0; q < kGalWarps; ++q) sum += ra[q * kSlots * 36 + t];
        }
        A[(int64_t)(6 * a + mk / 6) * nc + 6 * b + mk % 6] = sum;
    }
    cl.sync();  // the other CTAs' accumulators stay alive until every read is done
}

// Scalar (1-dof) meshes: one constant mode per aggregate, A_c[a][b] = sum of
// S_ij over free i in a and free j in b.  Same cluster / warp layout as
// k_coarse_galerkin, lanes over a CSR row's entries.
__global__ void __cluster_dims__(kGalSplit, 1, 1) __launch_bounds__(32 * kGalWarps)
    k_coarse_galerkin1(const int32_t *__restrict__ agg_ptr, const int32_t *__restrict__ agg_nodes,
                       const int32_t *__restrict__ node_agg, const int32_t *__restrict__ agg_slot,
                       const int32_t *__restrict__ nbr, const float4 *__restrict__ mode,
                       const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
                       const double *__restrict__ aval, int64_t nc, double *__restrict__ A)
{
    __shared__ double acc[kGalWarps][kSlots];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int a = blockIdx.x / kGalSplit;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kGalWarps * kSlots; t += blockDim.x) (&acc[0][0])[t] = 0.0;
    __syncthreads();
    for (int32_t t = agg_ptr[a] + (int32_t)rank * kGalWarps + w; t < agg_ptr[a + 1]; t += kGalWarps * kGalSplit) {
        const int32_t i = agg_nodes[t];
        const bool fi = !(mask_bits(mode[i]) & 1);
        for (int32_t s0 = row_ptr[i]; s0 < row_ptr[i + 1]; s0 += 32) {
            const int32_t sl = s0 + lane;
            const bool has = sl < row_ptr[i + 1];
            double g = 0.0;
            int slot = -1;
            if (has) {
                const int32_t j = col[sl];
                slot = agg_slot[node_agg[j]];
                if (fi && !(mask_bits(mode[j]) & 1)) g = aval[sl];
            }
            unsigned left = __ballot_sync(0xffffffffu, has);
            while (left) {
                const int leader = __ffs(left) - 1;
                const int cls = __shfl_sync(0xffffffffu, slot, leader);
                const bool mine = has && slot == cls;
                left &= ~__ballot_sync(0xffffffffu, mine);
                const double v = warp_sum_masked(mine ? g : 0.0);
                if (lane == 0) acc[w][cls] += v;
            }
        }
    }
    cl.sync();
    for (int t = (int)rank * blockDim.x + threadIdx.x; t < kSlots; t += kGalSplit * blockDim.x) {
        const int32_t b = nbr[kSlots * a + t];
        if (b < 0) continue;
        double sum = 0.0;
        for (unsigned r = 0; r < kGalSplit; ++r) {
            const double *ra = cl.map_shared_rank(&acc[0][0], r);
#pragma unroll
            for (int q = 0; q < kGalWarps; ++q) sum += ra[q * kSlots + t];
        }
        A[(int64_t)a * nc + b] = sum;
    }
    cl.sync();  // the other CTAs' accumulators stay alive until every read is done
}

// b = (a + a^T) / 2 in FP32 with row stride ldb >= n (the padding stays as it is)
__global__ void k_to_f32_sym(const double *__restrict__ a, float *__restrict__ b, int64_t n, int64_t ldb)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / n, j = t % n;
        b[i * ldb + j] = (float)(0.5 * (a[t] + a[j * n + i]));
    }
}

// c[6a + m][col] = (P^T r)[6a + m][col] for K = 32 V interleaved columns: a
// cluster of kRestrictSplit CTAs per aggregate (warp per node), partial sums
// added in rank order through distributed shared memory.  Two CTAs per
// aggregate keep the 48^3 elasticity grid (216 aggregates) within one wave
// of resident CTAs; four left a half-empty second wave (52 against 50 us per
// launch).
constexpr int kRestrictSplit = 2;

template <int V>
__global__ void __cluster_dims__(kRestrictSplit, 1, 1) __launch_bounds__(256, 4)
    k_coarse_restrict32(const float *__restrict__ r, const int32_t *__restrict__ agg_ptr,
                        const int32_t *__restrict__ agg_nodes, const float4 *__restrict__ mode, float *__restrict__ c,
                        const int *stop)
{
    constexpr int K = 32 * V;
    __shared__ float red[8][6][K];
    if (stop && *stop) return;  // uniform: stop changes only between launches
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int a = blockIdx.x / kRestrictSplit;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float acc[6][V];
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
        for (int v = 0; v < V; ++v) acc[m][v] = 0.f;
    // two nodes per trip: six row loads in flight per warp; the nodes' ids
    // and modes are fetched one per lane ahead of the trips and broadcast
    auto load_node = [&](int32_t i, const float4 &m, float (&rv)[3][V]) {
        const int bits = (int)m.w;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float *src = r + (3 * (int64_t)i + q) * K + lane * V;
            if constexpr (V == 4) {
                const float4 t4 = *reinterpret_cast<const float4 *>(src);
                rv[q][0] = t4.x; rv[q][1] = t4.y; rv[q][2] = t4.z; rv[q][3] = t4.w;
            } else if constexpr (V == 2) {
                const float2 t2 = *reinterpret_cast<const float2 *>(src);
                rv[q][0] = t2.x; rv[q][1] = t2.y;
            } else {
                rv[q][0] = *src;
            }
            if ((bits >> q) & 1)
#pragma unroll
                for (int v = 0; v < V; ++v) rv[q][v] = 0.f;
        }
    };
    auto add_node = [&](const float4 &m, const float (&rv)[3][V]) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            acc[0][v] += rv[0][v];
            acc[1][v] += rv[1][v];
            acc[2][v] += rv[2][v];
            acc[3][v] += m.y * rv[2][v] - m.z * rv[1][v];
            acc[4][v] += m.z * rv[0][v] - m.x * rv[2][v];
            acc[5][v] += m.x * rv[1][v] - m.y * rv[0][v];
        }
    };
    const int32_t step = 8 * kRestrictSplit, end = agg_ptr[a + 1];
    const int32_t first = agg_ptr[a] + (int32_t)rank * 8 + w;  // this warp's nodes: first + k step
    const int mine = first < end ? (end - 1 - first) / step + 1 : 0;
    auto bcast = [&](const float4 &m, int k) {
        return make_float4(__shfl_sync(0xffffffffu, m.x, k), __shfl_sync(0xffffffffu, m.y, k),
                           __shfl_sync(0xffffffffu, m.z, k), __shfl_sync(0xffffffffu, m.w, k));
    };
    for (int base = 0; base < mine; base += 32) {
        int32_t li = 0;
        float4 lm = make_float4(0.f, 0.f, 0.f, 0.f);
        if (base + lane < mine) {
            li = agg_nodes[first + (base + lane) * step];
            lm = mode[li];
        }
        const int cnt = min(32, mine - base);
        int k = 0;
        for (; k + 1 < cnt; k += 2) {
            const int32_t i0 = __shfl_sync(0xffffffffu, li, k), i1 = __shfl_sync(0xffffffffu, li, k + 1);
            const float4 m0 = bcast(lm, k), m1 = bcast(lm, k + 1);
            float r0[3][V], r1[3][V];
            load_node(i0, m0, r0);
            load_node(i1, m1, r1);
            add_node(m0, r0);
            add_node(m1, r1);
        }
        if (k < cnt) {
            const int32_t i0 = __shfl_sync(0xffffffffu, li, k);
            const float4 m0 = bcast(lm, k);
            float r0[3][V];
            load_node(i0, m0, r0);
            add_node(m0, r0);
        }
    }
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
        for (int v = 0; v < V; ++v) red[w][m][lane * V + v] = acc[m][v];
    __syncthreads();
    for (int t = threadIdx.x; t < 6 * K; t += blockDim.x) {
        const int m = t / K, col = t % K;
        float sum = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) sum += red[q][m][col];
        red[0][m][col] = sum;  // entry (m, col) is read and written by this thread only
    }
    cl.sync();
    for (int t = (int)rank * blockDim.x + threadIdx.x; t < 6 * K; t += kRestrictSplit * blockDim.x) {
        float sum = 0.f;
        for (unsigned j = 0; j < kRestrictSplit; ++j) sum += cl.map_shared_rank(&red[0][0][0], j)[t];
        c[(6 * (int64_t)a + t / K) * K + t % K] = sum;
    }
    cl.sync();  // the other CTAs' shared memory stays alive until every read is done
}

// scalar meshes: c[a][col] = sum of r[i][col] over the free nodes i of a
template <int V>
__global__ void __cluster_dims__(kRestrictSplit, 1, 1) __launch_bounds__(256)
    k_coarse_restrict32_1(const float *__restrict__ r, const int32_t *__restrict__ agg_ptr,
                          const int32_t *__restrict__ agg_nodes, const float4 *__restrict__ mode,
                          float *__restrict__ c, const int *stop)
{
    constexpr int K = 32 * V;
    __shared__ float red[8][K];
    if (stop && *stop) return;  // uniform: stop changes only between launches
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int a = blockIdx.x / kRestrictSplit;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = 0.f;
    const int32_t step = 8 * kRestrictSplit, end = agg_ptr[a + 1];
    for (int32_t t = agg_ptr[a] + (int32_t)rank * 8 + w; t < end; t += step) {
        const int32_t i = agg_nodes[t];
        if ((int)mode[i].w & 1) continue;  // warp-uniform: one node per warp
        float rv[V];
        const float *src = r + (int64_t)i * K + lane * V;
#pragma unroll
        for (int v = 0; v < V; ++v) rv[v] = src[v];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] += rv[v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) red[w][lane * V + v] = acc[v];
    __syncthreads();
    for (int t = threadIdx.x; t < K; t += blockDim.x) {
        float sum = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) sum += red[q][t];
        red[0][t] = sum;
    }
    cl.sync();
    for (int t = (int)rank * blockDim.x + threadIdx.x; t < K; t += kRestrictSplit * blockDim.x) {
        float sum = 0.f;
        for (unsigned j = 0; j < kRestrictSplit; ++j) sum += cl.map_shared_rank(&red[0][0], j)[t];
        c[(int64_t)a * K + t] = sum;
    }
    cl.sync();
}

// e = A c with A the coarse inverse (FP32, symmetric, lda x lda, zero past
// nc) and c, e [lda][K]; rz[col] += sum_rows c e in FP64.  A tiled FP32
// product on CUDA cores: a CTA owns 64 rows x 32 columns of e and a quarter
// of the k range, with 4 x 4 outputs per thread from shared-memory tiles
// (the A tile is read as rows k of A, i.e. already transposed, because A is
// symmetric) filled by cp.async one 32-wide k chunk ahead; the four k
// quarters form a cluster and are added in rank order through distributed
// shared memory, so the result does not depend on scheduling.
constexpr int kGemmRows = 64, kGemmCols = 32, kGemmK = 32, kGemmSplit = 4;

template <int V>
__global__ void __cluster_dims__(1, 1, kGemmSplit) __launch_bounds__(128)
    k_coarse_gemm32(const float *__restrict__ A, const float *__restrict__ c, float *__restrict__ e, int64_t lda,
                    int64_t nc, double *rz, const int *stop)
{
    constexpr int K = 32 * V;
    __shared__ __align__(16) float sa[2][kGemmK][kGemmRows];
    __shared__ __align__(16) float sc[2][kGemmK][kGemmCols];
    __shared__ __align__(16) float part[kGemmRows][kGemmCols];
    __shared__ double sred[4][kGemmCols];
    if (stop && *stop) return;  // uniform: stop changes only between launches
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int tid = threadIdx.x, rg = tid % 16, cgp = tid / 16;  // rows 4 rg.., columns 4 cgp..
    const int64_t row0 = (int64_t)blockIdx.x * kGemmRows;
    const int col0 = blockIdx.y * kGemmCols;
    const int64_t nchunks = lda / kGemmK, per = (nchunks + kGemmSplit - 1) / kGemmSplit;
    const int64_t kc0 = min((int64_t)rank * per, nchunks), kc1 = min(kc0 + per, nchunks);
    auto fetch = [&](int64_t kc, int buf) {
        const int64_t k0 = kc * kGemmK;
        // A rows k0.., columns row0..row0+63: 512 16-byte pieces, 4 per thread
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int q = tid + 128 * j, kr = q / 16, cc = q % 16;
            cp_async16(&sa[buf][kr][cc * 4], A + (k0 + kr) * lda + row0 + cc * 4);
        }
        // c rows k0.., columns col0..col0+31: 256 pieces, 2 per thread
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int q = tid + 128 * j, kr = q / 8, cc = q % 8;
            cp_async16(&sc[buf][kr][cc * 4], c + (k0 + kr) * K + col0 + cc * 4);
        }
        cp_async_commit();
    };
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    if (kc0 < kc1) fetch(kc0, 0);
    for (int64_t kc = kc0; kc < kc1; ++kc) {
        const int buf = (int)((kc - kc0) & 1);
        if (kc + 1 < kc1) {
            fetch(kc + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < kGemmK; ++kk) {
            const float4 a4 = *reinterpret_cast<const float4 *>(&sa[buf][kk][rg * 4]);
            const float4 c4 = *reinterpret_cast<const float4 *>(&sc[buf][kk][cgp * 4]);
            const float av[4] = {a4.x, a4.y, a4.z, a4.w}, cv[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], cv[j], acc[i][j]);
        }
        __syncthreads();  // the buffer is refilled by the next iteration's fetch
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        *reinterpret_cast<float4 *>(&part[rg * 4 + i][cgp * 4]) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
    cl.sync();
    // this CTA finishes rows [16 rank, 16 rank + 16) of the tile: column tid % 32, rows 4 apart
    constexpr int MY = kGemmRows / kGemmSplit;
    const int col = tid % kGemmCols;
    double d = 0.0;
#pragma unroll
    for (int j = 0; j < MY / 4; ++j) {
        const int lr = (int)rank * MY + tid / kGemmCols + 4 * j;
        float sum = 0.f;
        for (unsigned q = 0; q < kGemmSplit; ++q) sum += cl.map_shared_rank(&part[0][0], q)[lr * kGemmCols + col];
        const int64_t row = row0 + lr;
        e[row * K + col0 + col] = sum;
        if (row < nc) d += (double)c[row * K + col0 + col] * sum;
    }
    cl.sync();  // partial tiles stay alive until every CTA has read them
    if (!rz) return;
    sred[tid / kGemmCols][col] = d;
    __syncthreads();
    if (tid < kGemmCols) atomicAdd(rz + col0 + tid, sred[0][tid] + sred[1][tid] + sred[2][tid] + sred[3][tid]);
}

// single FP64 vector: c[6a + m] = (P^T r)[6a + m]
__global__ void __launch_bounds__(256) k_coarse_restrict64(const double *__restrict__ r,
                                                           const int32_t *__restrict__ agg_ptr,
                                                           const int32_t *__restrict__ agg_nodes,
                                                           const float4 *__restrict__ mode, double *__restrict__ c,
                                                           const int *done)
{
    __shared__ double red[6][8];
    if (done && *done) return;
    const int a = blockIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int32_t t = agg_ptr[a] + threadIdx.x; t < agg_ptr[a + 1]; t += blockDim.x) {
        const int32_t i = agg_nodes[t];
        const float4 m = mode[i];
        const int bits = (int)m.w;
        const double r0 = (bits & 1) ? 0.0 : r[3 * (int64_t)i], r1 = (bits & 2) ? 0.0 : r[3 * (int64_t)i + 1],
                     r2 = (bits & 4) ? 0.0 : r[3 * (int64_t)i + 2];
        acc[0] += r0;
        acc[1] += r1;
        acc[2] += r2;
        acc[3] += (double)m.y * r2 - (double)m.z * r1;
        acc[4] += (double)m.z * r0 - (double)m.x * r2;
        acc[5] += (double)m.x * r1 - (double)m.y * r0;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        double v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[m][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[threadIdx.x][q];
        c[6 * a + threadIdx.x] = s;
    }
}

// scalar meshes, one FP64 vector: c[a] = sum of r over the free nodes of a
__global__ void __launch_bounds__(256) k_coarse_restrict64_1(const double *__restrict__ r,
                                                             const int32_t *__restrict__ agg_ptr,
                                                             const int32_t *__restrict__ agg_nodes,
                                                             const float4 *__restrict__ mode, double *__restrict__ c,
                                                             const int *done)
{
    __shared__ double red[8];
    if (done && *done) return;
    const int a = blockIdx.x;
    double acc = 0.0;
    for (int32_t t = agg_ptr[a] + threadIdx.x; t < agg_ptr[a + 1]; t += blockDim.x) {
        const int32_t i = agg_nodes[t];
        if (!((int)mode[i].w & 1)) acc += r[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sum += red[q];
        c[a] = sum;
    }
}

// e = A c (FP64, warp per row); rz += c.e
__global__ void __launch_bounds__(256) k_coarse_apply64(const double *__restrict__ A, const double *__restrict__ c,
                                                        double *__restrict__ e, int64_t nc, double *rz, const int *done)
{
    __shared__ double sh[8];
    if (done && *done) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t row = (int64_t)blockIdx.x * 8 + w;
    double part = 0.0;
    if (row < nc) {
        // four independent partial sums keep four loads of the row in flight
        const double *Ar = A + row * nc;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int64_t k = lane;
        for (; k + 96 < nc; k += 128) {
            s0 += Ar[k] * c[k];
            s1 += Ar[k + 32] * c[k + 32];
            s2 += Ar[k + 64] * c[k + 64];
            s3 += Ar[k + 96] * c[k + 96];
        }
        for (; k < nc; k += 32) s0 += Ar[k] * c[k];
        double s = (s0 + s1) + (s2 + s3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            e[row] = s;
            part = s * c[row];
        }
    }
    if (lane == 0) sh[w] = part;
    __syncthreads();
    if (threadIdx.x == 0 && rz) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += sh[q];
        atomicAdd(rz, t);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct BoxGrid {
    int nb[3] = {1, 1, 1};            // boxes per axis
    double ext[3] = {0, 0, 0}, emax = 0.0;
    int32_t nagg = 0;
    std::vector<int32_t> node_agg;    // aggregate of each node
    std::vector<int32_t> box_agg;     // aggregate of each box, -1 when empty
};

// Box grid over a node set: boxes per axis for about `size` nodes along each
// axis (about max_aggs boxes at most), coarsened (halved per axis) until
// every element's nodes lie in boxes at most one apart along each axis;
// aggregates are the non-empty boxes numbered in box order.  Host only.
bool box_aggregation(const double *X, int64_t nodes, const uint32_t *conn, int64_t num_elems, int nn, int size,
                     int max_aggs, BoxGrid &g)
{
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = INFINITY;
        hi[d] = -INFINITY;
    }
    for (int64_t i = 0; i < nodes; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], X[3 * i + d]);
            hi[d] = std::max(hi[d], X[3 * i + d]);
        }
    double emax = 0.0;
    for (int d = 0; d < 3; ++d) {
        g.ext[d] = hi[d] - lo[d];
        emax = std::max(emax, g.ext[d]);
    }
    g.emax = emax;
    if (!(emax > 0.0)) return false;
    const double *ext = g.ext;
    int dim = 0;
    double vol = 1.0;
    for (int d = 0; d < 3; ++d)
        if (ext[d] > 1e-12 * emax) {
            ++dim;
            vol *= ext[d];
        }
    const double per = std::pow((double)std::max(size, 2), dim);
    const double target = std::min<double>(max_aggs, std::max(1.0, (double)nodes / per));
    const double hb = std::pow(vol / target, 1.0 / dim);
    int *nb = g.nb;
    for (int d = 0; d < 3; ++d) nb[d] = ext[d] > 1e-12 * emax ? std::max(1, (int)std::lround(ext[d] / hb)) : 1;
    std::vector<int32_t> box(nodes * 3);
    bool ok = false;
    for (int attempt = 0; attempt < 32 && !ok; ++attempt) {
        for (int64_t i = 0; i < nodes; ++i)
            for (int d = 0; d < 3; ++d) {
                int b = ext[d] > 1e-12 * emax ? (int)std::floor((X[3 * i + d] - lo[d]) / ext[d] * nb[d]) : 0;
                box[3 * i + d] = std::min(std::max(b, 0), nb[d] - 1);
            }
        ok = true;
        for (int64_t e = 0; e < num_elems && ok; ++e)
            for (int d = 0; d < 3 && ok; ++d) {
                int bmin = INT32_MAX, bmax = INT32_MIN;
                for (int k = 0; k < nn; ++k) {
                    const uint32_t v = conn[(size_t)e * nn + k];
                    if ((int64_t)v >= nodes) return false;
                    const int b = box[3 * (int64_t)v + d];
                    bmin = std::min(bmin, b);
                    bmax = std::max(bmax, b);
                }
                if (bmax - bmin > 1) ok = false;
            }
        if (!ok) {
            if (nb[0] == 1 && nb[1] == 1 && nb[2] == 1) break;
            for (int d = 0; d < 3; ++d) nb[d] = std::max(1, nb[d] / 2);
        }
    }
    if (!ok) return false;
    const int64_t nboxes = (int64_t)nb[0] * nb[1] * nb[2];
    g.box_agg.assign(nboxes, -1);
    g.node_agg.resize(nodes);
    int32_t nagg = 0;
    for (int64_t i = 0; i < nodes; ++i) {
        const int64_t id = box[3 * i] + (int64_t)nb[0] * (box[3 * i + 1] + (int64_t)nb[1] * box[3 * i + 2]);
        g.box_agg[id] = 1;
    }
    for (int64_t id = 0; id < nboxes; ++id)  // aggregates in box order
        if (g.box_agg[id] > 0) g.box_agg[id] = nagg++;
        else g.box_agg[id] = -1;
    for (int64_t i = 0; i < nodes; ++i)
        g.node_agg[i] = g.box_agg[box[3 * i] + (int64_t)nb[0] * (box[3 * i + 1] + (int64_t)nb[1] * box[3 * i + 2])];
    g.nagg = nagg;
    return true;
}

// Aggregates = the non-empty boxes of a grid laid over the mesh's bounding
// box, about `size` nodes along each axis (about kMaxAggs boxes at most on
// 3-dof meshes, kMaxAggs1 on scalar ones).  The
// colour classes (box index mod 3 per axis) make the Galerkin product a
// single pass; they need every element's nodes to lie in boxes at most one
// apart per axis, which is checked over the connectivity (the grid is
// coarsened until it holds).
static bool coarse_aggregate(sfc_system *s, int size)
{
    sfc_ctx *ctx = s->ctx;
    const sfc_mesh *m = s->pattern_mesh;
    CoarseSpace &cs = s->coarse;
    cs.built = false;
    if (!m) return false;
    const int dof = m->dof;
    if (dof == 3) {
        if (!s->has_bsr || m->num_nodes != s->nodes) return false;
    } else if (dof != 1 || m->num_dofs != s->N) {
        return false;
    }
    const int64_t nodes = m->num_nodes;
    const int max_aggs = dof == 3 ? kMaxAggs : kMaxAggs1;
    const double *X = m->h_coords.data();
    std::vector<uint32_t> conn((size_t)m->num_elems * m->nn);
    download(ctx, conn.data(), m->conn.p, conn.size());
    BoxGrid g;
    if (!box_aggregation(X, nodes, conn.data(), m->num_elems, m->nn, size, max_aggs, g)) return false;
    const int32_t nagg = g.nagg;
    const int *nb = g.nb;
    const double *ext = g.ext;
    const double emax = g.emax;
    const std::vector<int32_t> &node_agg = g.node_agg;
    const std::vector<int32_t> &box_agg = g.box_agg;
    const int64_t nboxes = (int64_t)nb[0] * nb[1] * nb[2];
    std::vector<int32_t> agg_ptr(nagg + 1, 0), agg_nodes(nodes);
    for (int64_t i = 0; i < nodes; ++i) ++agg_ptr[node_agg[i] + 1];
    for (int32_t a = 0; a < nagg; ++a) agg_ptr[a + 1] += agg_ptr[a];
    {
        std::vector<int32_t> fill(agg_ptr.begin(), agg_ptr.end() - 1);
        for (int64_t i = 0; i < nodes; ++i) agg_nodes[fill[node_agg[i]]++] = (int32_t)i;
    }
    std::vector<double> cen(3 * (size_t)nagg, 0.0);
    for (int64_t i = 0; i < nodes; ++i)
        for (int d = 0; d < 3; ++d) cen[3 * node_agg[i] + d] += X[3 * i + d];
    for (int32_t a = 0; a < nagg; ++a)
        for (int d = 0; d < 3; ++d) cen[3 * a + d] /= (double)(agg_ptr[a + 1] - agg_ptr[a]);
    double hsum = 0.0;
    int hn = 0;
    for (int d = 0; d < 3; ++d)
        if (ext[d] > 1e-12 * emax) {
            hsum += ext[d] / nb[d];
            ++hn;
        }
    const double h = hsum / hn;
    std::vector<float4> off(nodes);
    for (int64_t i = 0; i < nodes; ++i) {
        const int32_t a = node_agg[i];
        off[i] = make_float4((float)((X[3 * i] - cen[3 * a]) / h), (float)((X[3 * i + 1] - cen[3 * a + 1]) / h),
                             (float)((X[3 * i + 2] - cen[3 * a + 2]) / h), 0.f);
    }
    std::vector<int32_t> slot(nagg), nbr((size_t)nagg * kSlots, -1);
    for (int64_t id = 0; id < nboxes; ++id) {
        const int32_t a = box_agg[id];
        if (a < 0) continue;
        const int bx = (int)(id % nb[0]), by = (int)((id / nb[0]) % nb[1]), bz = (int)(id / ((int64_t)nb[0] * nb[1]));
        slot[a] = bx % 3 + 3 * (by % 3) + 9 * (bz % 3);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = bx + dx, y = by + dy, z = bz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= nb[0] || y >= nb[1] || z >= nb[2]) continue;
                    const int32_t b = box_agg[x + (int64_t)nb[0] * (y + (int64_t)nb[1] * z)];
                    if (b < 0) continue;
                    nbr[(size_t)a * kSlots + (x % 3) + 3 * (y % 3) + 9 * (z % 3)] = b;
                }
    }
    cs.nagg = nagg;
    cs.dof = dof;
    cs.nodes = nodes;
    cs.nc = (dof == 3 ? 6 : 1) * (int64_t)nagg;
    for (int d = 0; d < 3; ++d) cs.nb[d] = nb[d];
    upload(ctx, cs.node_agg, node_agg.data(), nodes);
    upload(ctx, cs.agg_ptr, agg_ptr.data(), agg_ptr.size());
    upload(ctx, cs.agg_nodes, agg_nodes.data(), nodes);
    upload(ctx, cs.agg_slot, slot.data(), nagg);
    upload(ctx, cs.nbr, nbr.data(), nbr.size());
    upload(ctx, cs.offset, off.data(), nodes);
    cs.mode.alloc(nodes);
    cs.mesh = m;
    cs.size = size;
    cs.built = true;
    cs.op_serial = 0;
    return true;
}

// (Re)builds the coarse space for the current operator; false when the
// system has none (no mesh attached, or no valid box grid).
bool coarse_prepare(sfc_system *s)
{
    CoarseSpace &cs = s->coarse;
    const int size = s->opt.coarse_size > 0 ? s->opt.coarse_size : 8;
    if (!cs.built || cs.mesh != s->pattern_mesh || cs.size != size) {
        if (!coarse_aggregate(s, size)) return false;
    }
    if (cs.op_serial == s->op_serial) return true;
    sfc_ctx *ctx = s->ctx;
    ProfScope ps(ctx, "phase:coarse_setup", 0.0);
    const int64_t nodes = cs.nodes, nc = cs.nc;
    k_coarse_modes<<<grid_for(nodes, 256), 256, 0, ctx->stream>>>(cs.offset.p, s->mask.p, nodes, cs.dof, cs.mode.p);
    cs.a64.alloc(nc * nc);
    cs.lda = (nc + 63) / 64 * 64;
    cs.a32.alloc(cs.lda * cs.lda);
    SFC_CK(cudaMemsetAsync(cs.a32.p, 0, cs.lda * cs.lda * sizeof(float), ctx->stream));
    SFC_CK(cudaMemsetAsync(cs.a64.p, 0, nc * nc * sizeof(double), ctx->stream));
    {
        ProfScope pg(ctx, "coarse_galerkin", 0.0);
        if (cs.dof == 3)
            k_coarse_galerkin<<<(unsigned)(cs.nagg * kGalSplit), 32 * kGalWarps, 0, ctx->stream>>>(
                cs.agg_ptr.p, cs.agg_nodes.p, cs.node_agg.p, cs.agg_slot.p, cs.nbr.p, cs.mode.p, s->bptr.p, s->bcol.p,
                s->bval64.p, nc, cs.a64.p);
        else
            k_coarse_galerkin1<<<(unsigned)(cs.nagg * kGalSplit), 32 * kGalWarps, 0, ctx->stream>>>(
                cs.agg_ptr.p, cs.agg_nodes.p, cs.node_agg.p, cs.agg_slot.p, cs.nbr.p, cs.mode.p, s->row_ptr.p,
                s->col.p, s->a_op.p, nc, cs.a64.p);
    }
    count_launch(ctx, 2);
    cs.gj.reserve(nc);
    int dropped = 0;
    {
        ProfScope pg(ctx, "coarse_inverse", 0.0);
        spd_inverse_gj(ctx, cs.a64.p, nc, 1e-10, cs.gj, nullptr, &dropped);
    }
    k_to_f32_sym<<<grid_for(nc * nc, 256), 256, 0, ctx->stream>>>(cs.a64.p, cs.a32.p, nc, cs.lda);
    count_launch(ctx);
    cs.dropped = dropped;
    cs.op_serial = s->op_serial;
    return true;
}

// c32 / e32 for K columns: lda rows, c32's rows past nc zero (the product
// multiplies them by A's zero padding); called outside stream capture before
// a block solve, so inside a captured interval nothing is allocated or set
void coarse_block_reserve(sfc_system *s, int K)
{
    CoarseSpace &cs = s->coarse;
    cs.c32.reserve(cs.lda * K);
    cs.e32.reserve(cs.lda * K);
    // the padding rows of the [lda][K] layout (a block of another K may have
    // written there): zeroed again whenever the allocation or K changes
    if (cs.c32_zeroed != cs.c32.p || cs.c32_zeroed_K != K || cs.c32_zeroed_lda != cs.lda) {
        SFC_CK(cudaMemsetAsync(cs.c32.p + cs.nc * K, 0, (size_t)(cs.lda - cs.nc) * K * sizeof(float),
                               s->ctx->stream));
        cs.c32_zeroed = cs.c32.p;
        cs.c32_zeroed_K = K;
        cs.c32_zeroed_lda = cs.lda;
    }
}

template <int V>
void coarse_block_apply(sfc_system *s, const float *r, double *rz, const int *stop)
{
    constexpr int K = 32 * V;
    CoarseSpace &cs = s->coarse;
    sfc_ctx *ctx = s->ctx;
    coarse_block_reserve(s, K);
    {
        ProfScope ps(ctx, "coarse_restrict32", (double)cs.dof * cs.nodes * K * 4 + 20.0 * cs.nodes + 4.0 * cs.nc * K);
        if (cs.dof == 3)
            k_coarse_restrict32<V><<<(unsigned)(cs.nagg * kRestrictSplit), 256, 0, ctx->stream>>>(
                r, cs.agg_ptr.p, cs.agg_nodes.p, cs.mode.p, cs.c32.p, stop);
        else
            k_coarse_restrict32_1<V><<<(unsigned)(cs.nagg * kRestrictSplit), 256, 0, ctx->stream>>>(
                r, cs.agg_ptr.p, cs.agg_nodes.p, cs.mode.p, cs.c32.p, stop);
        count_launch(ctx);
    }
    coarse_block_gemm<V>(s, rz, stop);
}
template void coarse_block_apply<1>(sfc_system *, const float *, double *, const int *);
template void coarse_block_apply<2>(sfc_system *, const float *, double *, const int *);
template void coarse_block_apply<4>(sfc_system *, const float *, double *, const int *);

// e = A_c^+ c for a restriction c already in cs.c32 (the fused r update and
// restriction of the block solver writes it)
template <int V>
void coarse_block_gemm(sfc_system *s, double *rz, const int *stop)
{
    constexpr int K = 32 * V;
    CoarseSpace &cs = s->coarse;
    sfc_ctx *ctx = s->ctx;
    ProfScope ps(ctx, "coarse_apply32", 4.0 * cs.nc * cs.nc + 8.0 * cs.nc * K);
    const dim3 grid((unsigned)(cs.lda / kGemmRows), K / kGemmCols, kGemmSplit);
    k_coarse_gemm32<V><<<grid, 128, 0, ctx->stream>>>(cs.a32.p, cs.c32.p, cs.e32.p, cs.lda, cs.nc, rz, stop);
    count_launch(ctx);
}
template void coarse_block_gemm<1>(sfc_system *, double *, const int *);
template void coarse_block_gemm<2>(sfc_system *, double *, const int *);
template void coarse_block_gemm<4>(sfc_system *, double *, const int *);

void coarse_vec_apply(sfc_system *s, const double *r, double *rz, const int *done)
{
    CoarseSpace &cs = s->coarse;
    sfc_ctx *ctx = s->ctx;
    cs.c64.reserve(cs.nc);
    cs.e64.reserve(cs.nc);
    {
        ProfScope ps(ctx, "coarse_restrict64", (double)cs.dof * cs.nodes * 8 + 20.0 * cs.nodes + 8.0 * cs.nc);
        if (cs.dof == 3)
            k_coarse_restrict64<<<(unsigned)cs.nagg, 256, 0, ctx->stream>>>(r, cs.agg_ptr.p, cs.agg_nodes.p,
                                                                            cs.mode.p, cs.c64.p, done);
        else
            k_coarse_restrict64_1<<<(unsigned)cs.nagg, 256, 0, ctx->stream>>>(r, cs.agg_ptr.p, cs.agg_nodes.p,
                                                                              cs.mode.p, cs.c64.p, done);
    }
    {
        ProfScope ps(ctx, "coarse_apply64", 8.0 * cs.nc * cs.nc + 16.0 * cs.nc);
        k_coarse_apply64<<<(unsigned)((cs.nc + 7) / 8), 256, 0, ctx->stream>>>(cs.a64.p, cs.c64.p, cs.e64.p, cs.nc,
                                                                                rz, done);
    }
    count_launch(ctx, 2);
}

}  // namespace sfc

// Host-only: the box aggregation of the two-level preconditioner for a node
// set, without a device (for inspection and CPU tests of the grid rule).
extern "C" int32_t sfc_coarse_boxes(const double *coords, int64_t num_nodes, const uint32_t *conn, int64_t num_elems,
                                    int32_t nodes_per_elem, int32_t size, int32_t max_aggs, int32_t *node_agg,
                                    int32_t *num_aggs, int32_t *boxes_per_axis)
{
    if (!coords || num_nodes <= 0 || !node_agg || !num_aggs || max_aggs < 1 ||
        (num_elems > 0 && (!conn || nodes_per_elem < 1)) || num_elems < 0)
        return SFC_ERR_BAD_ARG;
    try {
        sfc::BoxGrid g;
        if (!sfc::box_aggregation(coords, num_nodes, conn, num_elems, nodes_per_elem, size > 0 ? size : 8, max_aggs,
                                  g))
            return SFC_ERR_BAD_ARG;
        std::copy(g.node_agg.begin(), g.node_agg.end(), node_agg);
        *num_aggs = g.nagg;
        if (boxes_per_axis)
            for (int d = 0; d < 3; ++d) boxes_per_axis[d] = g.nb[d];
        return SFC_OK;
    } catch (const std::bad_alloc &) {
        return SFC_ERR_NO_MEMORY;
    }
}
