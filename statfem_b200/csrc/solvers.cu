// SPD sparse solves on the GPU: the replacement of the reference's
// Eigen::SparseLU behind SystemSolveEigenSparse::solveSystem /
// solveSystemTranspose (corlib/SystemSolveEigenSparse.hpp:273-404).
//
// The row-zeroed reference system A (corlib/Triplet.hpp:219-260) is solved
// through its symmetric elimination S (free rows keep free columns,
// constrained rows keep their diagonal): A u = F  <=>  S u = F - K_fc u_c, and
// A^T r = p  <=>  S r = p on the free dofs with r_c = (p_c - K_cf r_f)/scalar.
//
// Two methods:
//  * plain FP64 PCG, one right-hand side at a time (point Jacobi, the
//    baseline method; or the two-level preconditioner of coarse.cu): CSR SpMV
//    with sub-warp row groups, fused p.q reduction, fused x/r/z update with
//    the r.r and r.z reductions;
//  * mixed block PCG: up to 128 right-hand sides share each pass over the
//    FP32 copy of the matrix (one warp per row, each lane owns 1-4 columns of
//    an RHS-interleaved [N][K] block), iterations in FP32, and an outer FP64
//    loop recomputes the true residual b - S x with the FP64 matrix and
//    restarts FP32 PCG on it (iterative refinement) until every column meets
//    the FP64 relative-residual target.
// All reductions accumulate in FP64.  Scalars are kept per iteration (and per
// column) in device arrays, so no scalar kernel or host round trip sits
// between the three launches of an iteration; the host checks convergence
// every `check_every` iterations.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"

namespace sfc {

namespace {

namespace cg = cooperative_groups;

constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of one value per thread, result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0;
    if (w == 0) {
        r = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// ---------------------------------------------------------------------------
// single right-hand side, FP64
// ---------------------------------------------------------------------------

// y = S x over rows, G lanes per row; dot += x.y
template <int G>
__global__ void __launch_bounds__(kRedThreads) k_spmv64(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                         const double *__restrict__ a, const double *__restrict__ x,
                                                         double *__restrict__ y, int64_t N, double *dot,
                                                         const int *done)
{
    __shared__ double sh[32];
    if (done && *done) return;
    // The row loop runs over a warp-uniform base so that every lane of a warp
    // takes the same number of trips and reaches each full-mask shuffle.
    const int lane = threadIdx.x & 31, g = lane % G;
    constexpr int kRowsPerWarp = 32 / G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d = 0.0;
    for (int64_t base = warp * kRowsPerWarp; base < N; base += stride) {
        const int64_t i = base + lane / G;
        const bool valid = i < N;
        double s = 0.0;
        if (valid) {
            const int32_t e = rp[i + 1];
            for (int32_t k = rp[i] + g; k < e; k += G) s += a[k] * x[col[k]];
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
        if (valid && g == 0) {
            y[i] = s;
            d += x[i] * s;
        }
    }
    if (dot) {
        d = block_sum(d, sh);
        if (threadIdx.x == 0) atomicAdd(dot, d);
    }
}

// y = S x through the node-block (3 x 3) view on 3-dof meshes: one warp per
// node, lanes over its blocks (one index and nine values per block instead of
// nine indices); dot += x.y
__global__ void __launch_bounds__(kRedThreads) k_bspmv64(const int32_t *__restrict__ bptr,
                                                          const int32_t *__restrict__ bcol,
                                                          const double *__restrict__ bval,
                                                          const double *__restrict__ x, double *__restrict__ y,
                                                          int64_t nodes, double *dot, const int *done)
{
    __shared__ double sh[32];
    if (done && *done) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double d = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nodes; i += warps) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int32_t b = bptr[i] + lane; b < bptr[i + 1]; b += 32) {
            const int64_t j = bcol[b];
            const double *v = bval + 9 * (int64_t)b;
            const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
            a0 += v[0] * x0 + v[1] * x1 + v[2] * x2;
            a1 += v[3] * x0 + v[4] * x1 + v[5] * x2;
            a2 += v[6] * x0 + v[7] * x1 + v[8] * x2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) {
            y[3 * i] = a0;
            y[3 * i + 1] = a1;
            y[3 * i + 2] = a2;
            d += x[3 * i] * a0 + x[3 * i + 1] * a1 + x[3 * i + 2] * a2;
        }
    }
    if (dot) {
        d = block_sum(d, sh);
        if (threadIdx.x == 0) atomicAdd(dot, d);
    }
}

// r = b' (lifted rhs), x = 0, p = z = D^-1 r; rz0 = r.z, bb = r.r
__global__ void __launch_bounds__(kRedThreads) k_pcg_init(const double *__restrict__ b, const double *__restrict__ dinv,
                                                           double *__restrict__ x, double *__restrict__ r,
                                                           double *__restrict__ p, int64_t N, double *rz0, double *bb)
{
    __shared__ double sh[32];
    double a = 0, c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = b[i], zi = dinv[i] * ri;
        x[i] = 0.0;
        r[i] = ri;
        p[i] = zi;
        a += ri * zi;
        c += ri * ri;
    }
    a = block_sum(a, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) {
        atomicAdd(rz0, a);
        atomicAdd(bb, c);
    }
}

// alpha = rz/pq; x += alpha p; r -= alpha q; z = D^-1 r; rz' = r.z; rr' = r.r
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(double *__restrict__ x, double *__restrict__ r,
                                                             const double *__restrict__ p, const double *__restrict__ q,
                                                             const double *__restrict__ dinv, int64_t N,
                                                             const double *pq, const double *rz, double *rz_next,
                                                             double *rr_next, const int *done, int *err)
{
    __shared__ double sh[32];
    if (*done) return;
    const double den = *pq;
    if (!(den > 0.0)) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    const double alpha = *rz / den;
    double a = 0, c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double zi = dinv[i] * ri;
        a += ri * zi;
        c += ri * ri;
    }
    a = block_sum(a, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) {
        atomicAdd(rz_next, a);
        atomicAdd(rr_next, c);
    }
}

// convergence test on rr'; else beta = rz'/rz, p = D^-1 r + beta p
__global__ void k_pcg_pupdate(double *__restrict__ p, const double *__restrict__ r, const double *__restrict__ dinv,
                              int64_t N, const double *rz, const double *rz_next, const double *rr_next, double thr,
                              int it_next, int *done, const int *err)
{
    if (*done || *err) return;
    if (*rr_next <= thr) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *done = it_next;
        return;
    }
    const double beta = *rz_next / *rz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = dinv[i] * r[i] + beta * p[i];
}

// scalar two-level variant: p = D^-1 r + e[agg(i)] + beta p (INIT: p = z)
template <bool INIT>
__global__ void k_pcg1_pupdate(double *__restrict__ p, const double *__restrict__ r, const double *__restrict__ dinv,
                               const int32_t *__restrict__ node_agg, const float4 *__restrict__ mode,
                               const double *__restrict__ e, int64_t N, const double *rz, const double *rz_next,
                               const double *rr_next, double thr, int it_next, int *done, const int *err)
{
    double beta = 0.0;
    if constexpr (!INIT) {
        if (*done || *err) return;
        if (*rr_next <= thr) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *done = it_next;
            return;
        }
        beta = *rz_next / *rz;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double z = dinv[i] * r[i] + (((int)mode[i].w & 1) ? 0.0 : e[node_agg[i]]);
        p[i] = INIT ? z : z + beta * p[i];
    }
}

// lifting of prescribed values: b_f = F_f - sum_{j constrained} a_ref[f,j] g_j,
// g_j = F_j / a_ref[j,j]; constrained rows keep F.
__global__ void k_lift(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, const int32_t *__restrict__ diag,
                       const double *__restrict__ a_ref, const unsigned char *__restrict__ mask,
                       const double *__restrict__ F, int64_t N, double *__restrict__ b)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double v = F[i];
        if (!mask[i])
            for (int32_t s = rp[i]; s < rp[i + 1]; ++s) {
                const int32_t j = col[s];
                if (mask[j]) v -= a_ref[s] * (F[j] / a_ref[diag[j]]);
            }
        b[i] = v;
    }
}

// the same lifting for nrhs interleaved columns ([N][ld] in and out)
__global__ void k_lift_block(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                             const int32_t *__restrict__ diag, const double *__restrict__ a_ref,
                             const unsigned char *__restrict__ mask, const double *__restrict__ B, int ld, int nrhs,
                             int64_t N, double *__restrict__ out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * nrhs; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / nrhs;
        const int c = (int)(t - i * nrhs);
        double v = B[i * ld + c];
        if (!mask[i])
            for (int32_t s = rp[i]; s < rp[i + 1]; ++s) {
                const int32_t j = col[s];
                if (mask[j]) v -= a_ref[s] * (B[(int64_t)j * ld + c] / a_ref[diag[j]]);
            }
        out[i * ld + c] = v;
    }
}

__global__ void k_axpby(double *__restrict__ y, const double *__restrict__ x, double a, double b, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}

__global__ void __launch_bounds__(kRedThreads) k_dot(const double *__restrict__ a, const double *__restrict__ b,
                                                      int64_t n, double *out)
{
    __shared__ double sh[32];
    double s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// ---------------------------------------------------------------------------
// block of K = 32*V right-hand sides, RHS-interleaved [N][K]
// ---------------------------------------------------------------------------
// Q = S P (FP32 values, FP32 vectors, FP32 accumulate), warp per row;
// pq[c] += sum_i P[i][c] Q[i][c] in FP64
template <int V>
__global__ void __launch_bounds__(256) k_spmm32(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                const float *__restrict__ a, const float *__restrict__ P,
                                                float *__restrict__ Q, int64_t N, double *pq, const int *stop)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    if (*stop) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        float acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = 0.f;
        const int32_t b = rp[i], e = rp[i + 1];
        for (int32_t s0 = b; s0 < e; s0 += 32) {
            const int32_t s = s0 + lane;
            const float av = s < e ? a[s] : 0.f;
            const int32_t cv = s < e ? col[s] : 0;
            const int n = min(32, e - s0);
            for (int j = 0; j < n; ++j) {
                const float aj = __shfl_sync(0xffffffffu, av, j);
                const int32_t cj = __shfl_sync(0xffffffffu, cv, j);
                float pv[V];
                ldv<V>(P + (int64_t)cj * K + lane * V, pv);
#pragma unroll
                for (int v = 0; v < V; ++v) acc[v] = fmaf(aj, pv[v], acc[v]);
            }
        }
        stv<V>(Q + i * K + lane * V, acc);
        float pi[V];
        ldv<V>(P + i * K + lane * V, pi);
#pragma unroll
        for (int v = 0; v < V; ++v) dacc[v] += (double)pi[v] * (double)acc[v];
    }
    block_cols_add<V>(dacc, sh, pq);
}

// Q = S P for 3-dof meshes through the node-block view: one warp per node
// (three rows).  A chunk of up to 32 blocks (column node + 3x3 values) is
// staged in shared memory; for each block the warp loads the column node's
// three P rows (3*K contiguous floats) once and updates all three output rows,
// so every gathered row of P feeds three rows of Q.
template <int V>
__global__ void __launch_bounds__(256) k_bspmm32(const int32_t *__restrict__ bptr, const int32_t *__restrict__ bcol,
                                                 const float *__restrict__ bval, const float *__restrict__ P,
                                                 float *__restrict__ Q, int64_t nodes, double *pq, const int *stop)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    __shared__ float sv[8][32 * 9];
    __shared__ int sc[8][32];
    if (*stop) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nodes; i += warps) {
        float acc[3][V];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) acc[r][v] = 0.f;
        const int32_t b0 = bptr[i], b1 = bptr[i + 1];
        for (int32_t bb = b0; bb < b1; bb += 32) {
            const int nbk = min(32, b1 - bb);
            __syncwarp();
            if (lane < nbk) sc[w][lane] = bcol[bb + lane];
            for (int t = lane; t < 9 * nbk; t += 32) sv[w][t] = bval[(int64_t)bb * 9 + t];
            __syncwarp();
            // groups of U blocks: all 3U row loads are issued before the FMAs
            // so that several gathers are in flight per warp
            constexpr int U = V >= 4 ? 2 : 4;
            int t = 0;
            for (; t + U <= nbk; t += U) {
                float pv[U][3][V];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const float *pj = P + (int64_t)(3 * sc[w][t + u]) * K + lane * V;
                    ldv<V>(pj, pv[u][0]);
                    ldv<V>(pj + K, pv[u][1]);
                    ldv<V>(pj + 2 * K, pv[u][2]);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const float *bv = &sv[w][(t + u) * 9];
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        const float a0 = bv[3 * r], a1 = bv[3 * r + 1], a2 = bv[3 * r + 2];
#pragma unroll
                        for (int v = 0; v < V; ++v)
                            acc[r][v] =
                                fmaf(a2, pv[u][2][v], fmaf(a1, pv[u][1][v], fmaf(a0, pv[u][0][v], acc[r][v])));
                    }
                }
            }
            for (; t < nbk; ++t) {
                const float *pj = P + (int64_t)(3 * sc[w][t]) * K + lane * V;
                float p0[V], p1[V], p2[V];
                ldv<V>(pj, p0);
                ldv<V>(pj + K, p1);
                ldv<V>(pj + 2 * K, p2);
                const float *bv = &sv[w][t * 9];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const float a0 = bv[3 * r], a1 = bv[3 * r + 1], a2 = bv[3 * r + 2];
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        acc[r][v] = fmaf(a2, p2[v], fmaf(a1, p1[v], fmaf(a0, p0[v], acc[r][v])));
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const int64_t o = (3 * i + r) * K + lane * V;
            stv<V>(Q + o, acc[r]);
            float pi[V];
            ldv<V>(P + o, pi);
#pragma unroll
            for (int v = 0; v < V; ++v) dacc[v] += (double)pi[v] * (double)acc[r][v];
        }
    }
    block_cols_add<V>(dacc, sh, pq);
}

// R = B - S X in FP64 through the node-block view (see k_bspmm32)
template <int V>
__global__ void __launch_bounds__(256) k_bresid64(const int32_t *__restrict__ bptr, const int32_t *__restrict__ bcol,
                                                  const double *__restrict__ bval, const double *__restrict__ X,
                                                  const double *__restrict__ B, double *__restrict__ R, int64_t nodes,
                                                  double *rr)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    __shared__ double sv[8][32 * 9];
    __shared__ int sc[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nodes; i += warps) {
        double acc[3][V];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) acc[r][v] = 0.0;
        const int32_t b0 = bptr[i], b1 = bptr[i + 1];
        for (int32_t bb = b0; bb < b1; bb += 32) {
            const int nbk = min(32, b1 - bb);
            __syncwarp();
            if (lane < nbk) sc[w][lane] = bcol[bb + lane];
            for (int t = lane; t < 9 * nbk; t += 32) sv[w][t] = bval[(int64_t)bb * 9 + t];
            __syncwarp();
            for (int t = 0; t < nbk; ++t) {
                const double *xj = X + (int64_t)(3 * sc[w][t]) * K + lane * V;
                const double *bv = &sv[w][t * 9];
                double xv[3][V];
#pragma unroll
                for (int q = 0; q < 3; ++q) ldv64<V>(xj + q * K, xv[q]);
#pragma unroll
                for (int v = 0; v < V; ++v)
#pragma unroll
                    for (int r = 0; r < 3; ++r)
                        acc[r][v] = fma(bv[3 * r + 2], xv[2][v], fma(bv[3 * r + 1], xv[1][v], fma(bv[3 * r], xv[0][v], acc[r][v])));
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int64_t o = (3 * i + r) * K + lane * V + v;
                const double rv = B[o] - acc[r][v];
                R[o] = rv;
                dacc[v] += rv * rv;
            }
    }
    block_cols_add<V>(dacc, sh, rr);
}

// R = B - S X in FP64 (warp per row); rr[c] += R[i][c]^2
// R = B and rr[c] += sum_i B[i][c]^2: the residual of x = 0 (no product)
template <int V>
__global__ void __launch_bounds__(256) k_bcopy_norm64(const double *__restrict__ B, double *__restrict__ R, int64_t N,
                                                      double *rr)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int64_t o = i * K + lane * V + v;
            const double b = B[o];
            R[o] = b;
            dacc[v] += b * b;
        }
    block_cols_add<V>(dacc, sh, rr);
}

template <int V>
__global__ void __launch_bounds__(256) k_resid64(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                 const double *__restrict__ a, const double *__restrict__ X,
                                                 const double *__restrict__ B, double *__restrict__ R, int64_t N,
                                                 double *rr)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        double acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = 0.0;
        const int32_t b = rp[i], e = rp[i + 1];
        for (int32_t s0 = b; s0 < e; s0 += 32) {
            const int32_t s = s0 + lane;
            const double av = s < e ? a[s] : 0.0;
            const int32_t cv = s < e ? col[s] : 0;
            const int n = min(32, e - s0);
            for (int j = 0; j < n; ++j) {
                const double aj = __shfl_sync(0xffffffffu, av, j);
                const int32_t cj = __shfl_sync(0xffffffffu, cv, j);
                const double *xp = X + (int64_t)cj * K + lane * V;
#pragma unroll
                for (int v = 0; v < V; ++v) acc[v] = fma(aj, xp[v], acc[v]);
            }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const double rv = B[i * K + lane * V + v] - acc[v];
            R[i * K + lane * V + v] = rv;
            dacc[v] += rv * rv;
        }
    }
    block_cols_add<V>(dacc, sh, rr);
}

// r32 = r64 * scale_c, x32 = 0, p = z = D^-1 r32 for restarted columns; rz0[c], rr0[c]
template <int V, bool SETP = true>
__global__ void __launch_bounds__(256) k_binit32(const double *__restrict__ R64, const double *__restrict__ scale,
                                                 const float *__restrict__ dinv, const int *__restrict__ restart,
                                                 float *__restrict__ r, float *__restrict__ x, float *__restrict__ p,
                                                 int64_t N, double *rz0, double *rr0)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double a1[V], a2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) a1[v] = a2[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const float di = dinv[i];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int64_t o = i * K + lane * V + v;
            const float rv = (float)(R64[o] * scale[lane * V + v]);
            const float zv = di * rv;
            r[o] = rv;
            x[o] = 0.f;
            if (SETP && restart[lane * V + v]) p[o] = zv;
            a1[v] += (double)rv * zv;
            a2[v] += (double)rv * rv;
        }
    }
    block_cols_add<V>(a1, sh, rz0);
    __syncthreads();
    block_cols_add<V>(a2, sh, rr0);
}

// per column: frozen when rr[it][c] <= thr[c]; alpha = rz/pq; x += alpha p;
// r -= alpha q; rz'[c], rr'[c]
template <int V>
__global__ void __launch_bounds__(256) k_bupdate32(float *__restrict__ x, float *__restrict__ r,
                                                   const float *__restrict__ p, const float *__restrict__ q,
                                                   const float *__restrict__ dinv, int64_t N, const double *pq,
                                                   const double *rz, const double *rr, const double *thr,
                                                   double *rz_next, double *rr_next, const int *stop, int *err)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    if (*stop) return;
    const int lane = threadIdx.x & 31;
    float alpha[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        const bool frozen = rr[c] <= thr[c] || err[c];
        const double den = pq[c];
        if (!frozen && !(den > 0.0)) err[c] = 1;  // per-column breakdown: the column restarts
        alpha[v] = (frozen || !(den > 0.0)) ? 0.f : (float)(rz[c] / den);
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double a1[V], a2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) a1[v] = a2[v] = 0.0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const int64_t o = i * K + lane * V;
        float xv[V], rv[V], pv[V], qv[V];
        ldv<V>(x + o, xv);
        ldv<V>(r + o, rv);
        ldv<V>(p + o, pv);
        ldv<V>(q + o, qv);
        const float di = dinv[i];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            xv[v] = fmaf(alpha[v], pv[v], xv[v]);
            rv[v] = fmaf(-alpha[v], qv[v], rv[v]);
            const float zv = di * rv[v];
            a1[v] += (double)rv[v] * zv;
            a2[v] += (double)rv[v] * rv[v];
        }
        stv<V>(x + o, xv);
        stv<V>(r + o, rv);
    }
    block_cols_add<V>(a1, sh, rz_next);
    __syncthreads();
    block_cols_add<V>(a2, sh, rr_next);
}

// p = D^-1 r + beta p for active columns (rr' > thr)
template <int V>
__global__ void __launch_bounds__(256) k_bpupdate32(float *__restrict__ p, const float *__restrict__ r,
                                                    const float *__restrict__ dinv, int64_t N, const double *rz,
                                                    const double *rz_next, const double *rr_next, const double *thr,
                                                    const int *stop, const int *brk)
{
    constexpr int K = 32 * V;
    if (*stop) return;
    const int lane = threadIdx.x & 31;
    float beta[V];
    bool act[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        act[v] = rr_next[c] > thr[c] && !brk[c];
        beta[v] = act[v] ? (float)(rz_next[c] / rz[c]) : 0.f;
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const int64_t o = i * K + lane * V;
        float pv[V], rv[V];
        ldv<V>(p + o, pv);
        ldv<V>(r + o, rv);
        const float di = dinv[i];
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (act[v]) pv[v] = fmaf(beta[v], pv[v], di * rv[v]);
        stv<V>(p + o, pv);
    }
}

// scalar two-level p update: z = D^-1 r + e[agg(i)] (0 on constrained dofs),
// p = z + beta p for the active columns (INIT: p = z for the restarted ones)
template <int V, bool INIT>
__global__ void __launch_bounds__(256) k_cbpupdate32(float *__restrict__ p, const float *__restrict__ r,
                                                     const float *__restrict__ dinv,
                                                     const int32_t *__restrict__ node_agg,
                                                     const float4 *__restrict__ mode, const float *__restrict__ e,
                                                     int64_t N, const double *rz, const double *rz_next,
                                                     const double *rr_next, const double *thr, const int *stop,
                                                     const int *brk, const int *restart)
{
    constexpr int K = 32 * V;
    if (!INIT && *stop) return;
    const int lane = threadIdx.x & 31;
    float beta[V];
    bool act[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        if constexpr (INIT) {
            act[v] = restart[c] != 0;
            beta[v] = 0.f;
        } else {
            act[v] = rr_next[c] > thr[c] && !brk[c];
            beta[v] = act[v] ? (float)(rz_next[c] / rz[c]) : 0.f;
        }
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const int64_t o = i * K + lane * V;
        float pv[V], rv[V], ev[V];
        ldv<V>(p + o, pv);
        ldv<V>(r + o, rv);
        const bool free = !((int)mode[i].w & 1);
        ldv<V>(e + (int64_t)node_agg[i] * K + lane * V, ev);
        const float di = dinv[i];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float z = di * rv[v] + (free ? ev[v] : 0.f);
            if (act[v]) pv[v] = INIT ? z : fmaf(beta[v], pv[v], z);
        }
        stv<V>(p + o, pv);
    }
}

// ---- nodal 3x3 block-Jacobi variants of the three vector kernels -------------
// One warp per node (rows 3n..3n+2); z = Dinv_n r with the inverse of the
// node's diagonal block (row-major, FP32).
template <int V>
__device__ __forceinline__ void bj_apply(const float *__restrict__ D, const float (&r)[3][V], float (&z)[3][V])
{
    float d[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) d[k] = D[k];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int v = 0; v < V; ++v) z[i][v] = fmaf(d[3 * i + 2], r[2][v], fmaf(d[3 * i + 1], r[1][v], d[3 * i] * r[0][v]));
}

template <int V, bool SETP = true>
__global__ void __launch_bounds__(256) k_ninit32(const double *__restrict__ R64, const double *__restrict__ scale,
                                                 const float *__restrict__ bdinv, const int *__restrict__ restart,
                                                 float *__restrict__ r, float *__restrict__ x, float *__restrict__ p,
                                                 int64_t nodes, double *rz0, double *rr0)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double a1[V], a2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) a1[v] = a2[v] = 0.0;
    for (int64_t n = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; n < nodes; n += warps) {
        float rv[3][V], zv[3][V];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int v = 0; v < V; ++v) rv[i][v] = (float)(R64[(3 * n + i) * K + lane * V + v] * scale[lane * V + v]);
        bj_apply<V>(bdinv + 9 * n, rv, zv);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t o = (3 * n + i) * K + lane * V;
            float zero[V], pv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) zero[v] = 0.f;
            stv<V>(r + o, rv[i]);
            stv<V>(x + o, zero);
            if constexpr (SETP) {
                ldv<V>(p + o, pv);
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (restart[lane * V + v]) pv[v] = zv[i][v];
                stv<V>(p + o, pv);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                a1[v] += (double)rv[i][v] * zv[i][v];
                a2[v] += (double)rv[i][v] * rv[i][v];
            }
        }
    }
    block_cols_add<V>(a1, sh, rz0);
    __syncthreads();
    block_cols_add<V>(a2, sh, rr0);
}

// XUPD = false: x is left to the p update (k_npupdate32 / k_ncpupdate32 with
// x given), so this pass reads r and q only
template <int V, bool XUPD = true>
__global__ void __launch_bounds__(256, 4) k_nupdate32(float *__restrict__ x, float *__restrict__ r,
                                                   const float *__restrict__ p, const float *__restrict__ q,
                                                   const float *__restrict__ bdinv, int64_t nodes, const double *pq,
                                                   const double *rz, const double *rr, const double *thr,
                                                   double *rz_next, double *rr_next, const int *stop, int *err)
{
    constexpr int K = 32 * V;
    __shared__ double sh[8 * K];
    if (*stop) return;
    const int lane = threadIdx.x & 31;
    float alpha[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        const bool frozen = rr[c] <= thr[c] || err[c];
        const double den = pq[c];
        if (!frozen && !(den > 0.0)) err[c] = 1;
        alpha[v] = (frozen || !(den > 0.0)) ? 0.f : (float)(rz[c] / den);
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double a1[V], a2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) a1[v] = a2[v] = 0.0;
    for (int64_t n = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; n < nodes; n += warps) {
        float rv[3][V], zv[3][V];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t o = (3 * n + i) * K + lane * V;
            float qv[V];
            ldv<V>(r + o, rv[i]);
            ldv<V>(q + o, qv);
            if constexpr (XUPD) {
                float xv[V], pv[V];
                ldv<V>(x + o, xv);
                ldv<V>(p + o, pv);
#pragma unroll
                for (int v = 0; v < V; ++v) xv[v] = fmaf(alpha[v], pv[v], xv[v]);
                stv<V>(x + o, xv);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) rv[i][v] = fmaf(-alpha[v], qv[v], rv[i][v]);
            stv<V>(r + o, rv[i]);
        }
        bj_apply<V>(bdinv + 9 * n, rv, zv);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int v = 0; v < V; ++v) {
                a1[v] += (double)rv[i][v] * zv[i][v];
                a2[v] += (double)rv[i][v] * rv[i][v];
            }
    }
    block_cols_add<V>(a1, sh, rz_next);
    __syncthreads();
    block_cols_add<V>(a2, sh, rr_next);
}

// Two-level r update fused with the coarse restriction: r -= alpha q, r.z and
// r.r with z the nodal block-Jacobi share (k_nupdate32<V, false>), and the
// restriction c[6a + m][col] = (P^T r)[6a + m][col] of the updated r
// (k_coarse_restrict32), so r is read once per iteration instead of twice.
// The nodes are visited by aggregate: a cluster of S CTAs of W warps per
// aggregate, a warp per node, node ids and modes fetched one per lane ahead
// of the trips; the restriction's partial sums are added in rank order
// through distributed shared memory (no atomics, the same sums on every
// run), the dots as in k_nupdate32.
template <int V, int W, int S>
__global__ void __cluster_dims__(S, 1, 1) __launch_bounds__(32 * W, 24 / W)
    k_nrupdate32(float *__restrict__ r, const float *__restrict__ q, const float *__restrict__ bdinv,
                 const int32_t *__restrict__ agg_ptr, const int32_t *__restrict__ agg_nodes,
                 const float4 *__restrict__ mode, float *__restrict__ c, const double *pq, const double *rz,
                 const double *rr, const double *thr, double *rz_next, double *rr_next, const int *stop, int *err)
{
    constexpr int K = 32 * V;
    __shared__ float red[W][6][K];
    __shared__ double sh[W * K];
    if (*stop) return;  // uniform: stop changes only between launches
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int a = blockIdx.x / S;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float alpha[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int col = lane * V + v;
        const bool frozen = rr[col] <= thr[col] || err[col];
        const double den = pq[col];
        if (!frozen && !(den > 0.0) && rank == 0 && a == 0) err[col] = 1;
        alpha[v] = (frozen || !(den > 0.0)) ? 0.f : (float)(rz[col] / den);
    }
    // r.z and r.r over this warp's nodes (a few dozen) in FP32, then FP64
    // across warps and CTAs
    float a1f[V], a2f[V];
#pragma unroll
    for (int v = 0; v < V; ++v) a1f[v] = a2f[v] = 0.f;
    // the warp's restriction partial sums live in its own rows of red (each
    // lane its own columns), which keeps the trip within 80 registers
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
        for (int v = 0; v < V; ++v) red[w][m][lane * V + v] = 0.f;
    const int32_t step = W * S, end = agg_ptr[a + 1];
    const int32_t first = agg_ptr[a] + (int32_t)rank * W + w;  // this warp's nodes: first + k step
    const int mine = first < end ? (end - 1 - first) / step + 1 : 0;
    for (int base = 0; base < mine; base += 32) {
        int32_t li = 0;
        float4 lm = make_float4(0.f, 0.f, 0.f, 0.f);
        if (base + lane < mine) {
            li = agg_nodes[first + (base + lane) * step];
            lm = mode[li];
        }
        const int cnt = min(32, mine - base);
#pragma unroll 1
        for (int k = 0; k < cnt; ++k) {
            const int64_t n = __shfl_sync(0xffffffffu, li, k);
            const float mx = __shfl_sync(0xffffffffu, lm.x, k), my = __shfl_sync(0xffffffffu, lm.y, k),
                        mz = __shfl_sync(0xffffffffu, lm.z, k);
            const int bits = (int)__shfl_sync(0xffffffffu, lm.w, k);
            float rv[3][V], zv[3][V];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t o = (3 * n + i) * K + lane * V;
                float qv[V];
                ldv<V>(r + o, rv[i]);
                ldv<V>(q + o, qv);
#pragma unroll
                for (int v = 0; v < V; ++v) rv[i][v] = fmaf(-alpha[v], qv[v], rv[i][v]);
                stv<V>(r + o, rv[i]);
            }
            bj_apply<V>(bdinv + 9 * n, rv, zv);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    a1f[v] = fmaf(rv[i][v], zv[i][v], a1f[v]);
                    a2f[v] = fmaf(rv[i][v], rv[i][v], a2f[v]);
                }
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if ((bits >> i) & 1)
#pragma unroll
                    for (int v = 0; v < V; ++v) rv[i][v] = 0.f;
            float acc[V];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                float *row = &red[w][m][lane * V];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float t = m < 3    ? rv[m][v]
                                    : m == 3 ? my * rv[2][v] - mz * rv[1][v]
                                    : m == 4 ? mz * rv[0][v] - mx * rv[2][v]
                                             : mx * rv[1][v] - my * rv[0][v];
                    acc[v] = row[v] + t;
                }
#pragma unroll
                for (int v = 0; v < V; ++v) row[v] = acc[v];
            }
        }
    }
    double a1[V], a2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        a1[v] = a1f[v];
        a2[v] = a2f[v];
    }
    block_cols_add<V>(a1, sh, rz_next);
    __syncthreads();
    block_cols_add<V>(a2, sh, rr_next);
    __syncthreads();
    for (int t = threadIdx.x; t < 6 * K; t += blockDim.x) {
        const int m = t / K, col = t % K;
        float sum = 0.f;
#pragma unroll
        for (int j = 0; j < W; ++j) sum += red[j][m][col];
        red[0][m][col] = sum;  // entry (m, col) is read and written by this thread only
    }
    cl.sync();
    for (int t = (int)rank * blockDim.x + threadIdx.x; t < 6 * K; t += S * blockDim.x) {
        float sum = 0.f;
        for (unsigned j = 0; j < S; ++j) sum += cl.map_shared_rank(&red[0][0][0], j)[t];
        c[(6 * (int64_t)a + t / K) * K + t % K] = sum;
    }
    cl.sync();  // the other CTAs' shared memory stays alive until every read is done
}

// x (nullable): x += alpha p with this iteration's alpha (computed as in
// k_nupdate32) before p is overwritten
__device__ __forceinline__ float iter_alpha(int c, const double *pq, const double *rz, const double *rr,
                                            const double *thr, const int *brk)
{
    const bool frozen = rr[c] <= thr[c] || brk[c];
    const double den = pq[c];
    return (frozen || !(den > 0.0)) ? 0.f : (float)(rz[c] / den);
}

template <int V>
__global__ void __launch_bounds__(256) k_npupdate32(float *__restrict__ p, const float *__restrict__ r,
                                                    const float *__restrict__ bdinv, int64_t nodes, const double *rz,
                                                    const double *rz_next, const double *rr_next, const double *thr,
                                                    const int *stop, const int *brk, float *__restrict__ x,
                                                    const double *pq, const double *rr)
{
    constexpr int K = 32 * V;
    if (*stop) return;
    const int lane = threadIdx.x & 31;
    float beta[V], alpha[V];
    bool act[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        act[v] = rr_next[c] > thr[c] && !brk[c];
        beta[v] = act[v] ? (float)(rz_next[c] / rz[c]) : 0.f;
        alpha[v] = x ? iter_alpha(c, pq, rz, rr, thr, brk) : 0.f;
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t n = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; n < nodes; n += warps) {
        float rv[3][V], zv[3][V];
#pragma unroll
        for (int i = 0; i < 3; ++i) ldv<V>(r + (3 * n + i) * K + lane * V, rv[i]);
        bj_apply<V>(bdinv + 9 * n, rv, zv);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t o = (3 * n + i) * K + lane * V;
            float pv[V];
            ldv<V>(p + o, pv);
            if (x) {
                float xv[V];
                ldv<V>(x + o, xv);
#pragma unroll
                for (int v = 0; v < V; ++v) xv[v] = fmaf(alpha[v], pv[v], xv[v]);
                stv<V>(x + o, xv);
            }
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (act[v]) pv[v] = fmaf(beta[v], pv[v], zv[i][v]);
            stv<V>(p + o, pv);
        }
    }
}

// two-level variant of the p update: z = Dinv_n r_n + M_n e_a (the coarse
// correction e of the node's aggregate a, M_n = diag(free) [I | R(d_n)]:
// translation t plus rotation w x d), then p = z + beta p for the active
// columns.  INIT: p = z for the restarted columns, others keep p.
// (four 256-thread CTAs per SM: at most 64 registers)
template <int V, bool INIT>
__global__ void __launch_bounds__(256, 4) k_ncpupdate32(float *__restrict__ p, const float *__restrict__ r,
                                                     const float *__restrict__ bdinv,
                                                     const int32_t *__restrict__ node_agg,
                                                     const float4 *__restrict__ mode, const float *__restrict__ e,
                                                     int64_t nodes, const double *rz, const double *rz_next,
                                                     const double *rr_next, const double *thr, const int *stop,
                                                     const int *brk, const int *restart, float *__restrict__ x,
                                                     const double *pq, const double *rr)
{
    constexpr int K = 32 * V;
    if (!INIT && *stop) return;
    const int lane = threadIdx.x & 31;
    float beta[V], alpha[V];
    bool act[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int c = lane * V + v;
        if constexpr (INIT) {
            act[v] = restart[c] != 0;
            beta[v] = 0.f;
            alpha[v] = 0.f;
        } else {
            act[v] = rr_next[c] > thr[c] && !brk[c];
            beta[v] = act[v] ? (float)(rz_next[c] / rz[c]) : 0.f;
            alpha[v] = x ? iter_alpha(c, pq, rz, rr, thr, brk) : 0.f;
        }
    }
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t n = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; n < nodes; n += warps) {
        float rv[3][V], zv[3][V];
#pragma unroll
        for (int i = 0; i < 3; ++i) ldv<V>(r + (3 * n + i) * K + lane * V, rv[i]);
        bj_apply<V>(bdinv + 9 * n, rv, zv);
        const int32_t a = node_agg[n];
        const float4 m = mode[n];
        const int bits = (int)m.w;
        // M_n e_a streamed one mode row at a time (translations, then the
        // rotations w x d), so that only one row of e is live
        const float *ea = e + 6 * (int64_t)a * K + lane * V;
        float cc[3][V], t[V];
#pragma unroll
        for (int k = 0; k < 3; ++k) ldv<V>(ea + k * K, cc[k]);
        ldv<V>(ea + 3 * K, t);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            cc[1][v] -= t[v] * m.z;
            cc[2][v] += t[v] * m.y;
        }
        ldv<V>(ea + 4 * K, t);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            cc[0][v] += t[v] * m.z;
            cc[2][v] -= t[v] * m.x;
        }
        ldv<V>(ea + 5 * K, t);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            cc[0][v] -= t[v] * m.y;
            cc[1][v] += t[v] * m.x;
            if (!(bits & 1)) zv[0][v] += cc[0][v];
            if (!(bits & 2)) zv[1][v] += cc[1][v];
            if (!(bits & 4)) zv[2][v] += cc[2][v];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t o = (3 * n + i) * K + lane * V;
            float pv[V];
            ldv<V>(p + o, pv);
            if (!INIT && x) {
                float xv[V];
                ldv<V>(x + o, xv);
#pragma unroll
                for (int v = 0; v < V; ++v) xv[v] = fmaf(alpha[v], pv[v], xv[v]);
                stv<V>(x + o, xv);
            }
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (act[v]) pv[v] = fmaf(beta[v], pv[v], zv[i][v]);
            stv<V>(p + o, pv);
        }
    }
}

// ---- FP64 two-level PCG (one vector, 3-dof nodes, thread per node) ---------
__device__ __forceinline__ void bj_apply64(const float *__restrict__ D, const double (&r)[3], double (&z)[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
        z[i] = (double)D[3 * i] * r[0] + (double)D[3 * i + 1] * r[1] + (double)D[3 * i + 2] * r[2];
}

// r = b, x = 0; rz0 += r . Dinv r (block-Jacobi share), bb += r . r
__global__ void __launch_bounds__(kRedThreads) k_pcg2_init(const double *__restrict__ b, const float *__restrict__ bdinv,
                                                            double *__restrict__ x, double *__restrict__ r,
                                                            int64_t nodes, double *rz0, double *bb)
{
    __shared__ double sh[32];
    double a = 0, c = 0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes; n += (int64_t)gridDim.x * blockDim.x) {
        double rv[3], zv[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rv[i] = b[3 * n + i];
            r[3 * n + i] = rv[i];
            x[3 * n + i] = 0.0;
        }
        bj_apply64(bdinv + 9 * n, rv, zv);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            a += rv[i] * zv[i];
            c += rv[i] * rv[i];
        }
    }
    a = block_sum(a, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) {
        atomicAdd(rz0, a);
        atomicAdd(bb, c);
    }
}

// alpha = rz/pq; x += alpha p; r -= alpha q; rz' += r . Dinv r; rr' += r . r
__global__ void __launch_bounds__(kRedThreads) k_pcg2_update(double *__restrict__ x, double *__restrict__ r,
                                                              const double *__restrict__ p, const double *__restrict__ q,
                                                              const float *__restrict__ bdinv, int64_t nodes,
                                                              const double *pq, const double *rz, double *rz_next,
                                                              double *rr_next, const int *done, int *err)
{
    __shared__ double sh[32];
    if (*done) return;
    const double den = *pq;
    if (!(den > 0.0)) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    const double alpha = *rz / den;
    double a = 0, c = 0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes; n += (int64_t)gridDim.x * blockDim.x) {
        double rv[3], zv[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t k = 3 * n + i;
            x[k] += alpha * p[k];
            rv[i] = r[k] - alpha * q[k];
            r[k] = rv[i];
        }
        bj_apply64(bdinv + 9 * n, rv, zv);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            a += rv[i] * zv[i];
            c += rv[i] * rv[i];
        }
    }
    a = block_sum(a, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) {
        atomicAdd(rz_next, a);
        atomicAdd(rr_next, c);
    }
}

// convergence test on rr'; else p = Dinv r + M e + beta p (INIT: p = z)
template <bool INIT>
__global__ void k_pcg2_pupdate(double *__restrict__ p, const double *__restrict__ r, const float *__restrict__ bdinv,
                               const int32_t *__restrict__ node_agg, const float4 *__restrict__ mode,
                               const double *__restrict__ e, int64_t nodes, const double *rz,
                               const double *rz_next, const double *rr_next, double thr, int it_next, int *done,
                               const int *err)
{
    double beta = 0.0;
    if constexpr (!INIT) {
        if (*done || *err) return;
        if (*rr_next <= thr) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *done = it_next;
            return;
        }
        beta = *rz_next / *rz;
    }
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes; n += (int64_t)gridDim.x * blockDim.x) {
        double rv[3], zv[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) rv[i] = r[3 * n + i];
        bj_apply64(bdinv + 9 * n, rv, zv);
        const int64_t a = node_agg[n];
        const float4 m = mode[n];
        const int bits = (int)m.w;
        const double *ea = e + 6 * a;
        const double dx = m.x, dy = m.y, dz = m.z;
        const double c[3] = {ea[0] + ea[4] * dz - ea[5] * dy, ea[1] + ea[5] * dx - ea[3] * dz,
                             ea[2] + ea[3] * dy - ea[4] * dx};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double z = zv[i] + (((bits >> i) & 1) ? 0.0 : c[i]);
            p[3 * n + i] = INIT ? z : z + beta * p[3 * n + i];
        }
    }
}

// Convergence test after every inner iteration of a check interval: the
// first iteration after which all columns are below their thresholds sets
// *stop (every later kernel of the interval returns at once) and records in
// *ran how many of the interval's iterations ran (it_local + 1).
template <int K>
__global__ void k_bcheck_it(const double *rr, const double *thr, int *stop, int *ran, int it_local)
{
    __shared__ int any;
    if (*stop) return;  // uniform: only check kernels set it, and none runs beside this one
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int c = threadIdx.x; c < K; c += blockDim.x)
        if (rr[c] > thr[c]) any = 1;
    __syncthreads();
    if (threadIdx.x == 0 && !any) {
        *stop = 1;
        *ran = it_local + 1;
    }
}

// x64 += norm_c * x32
template <int V>
__global__ void k_bacc64(double *__restrict__ X64, const float *__restrict__ x32, const double *__restrict__ norm,
                         int64_t N)
{
    constexpr int K = 32 * V;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * K; t += (int64_t)gridDim.x * blockDim.x)
        X64[t] += norm[t % K] * (double)x32[t];
}

// gather columns [c0, c0+kb) of B (row stride ld) into a zero-padded [N][K]
__global__ void k_gather_cols(const double *__restrict__ B, int ld, int c0, int kb, int K, int64_t N,
                              double *__restrict__ out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / K;
        const int c = (int)(t - i * K);
        out[t] = c < kb ? B[i * ld + c0 + c] : 0.0;
    }
}

// X[i][c] += d[i] (column c of an [N][K] block)
__global__ void k_add_col(double *__restrict__ X, int K, int c, const double *__restrict__ d, int64_t N)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        X[i * K + c] += d[i];
}

__global__ void k_scatter_cols(const double *__restrict__ in, int ld, int c0, int kb, int K, int64_t N,
                               double *__restrict__ X)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * (int64_t)kb; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / kb;
        const int c = (int)(t - i * kb);
        X[i * ld + c0 + c] = in[i * K + c];
    }
}

// A^T fixup on constrained dofs: Y[c][a] += sum over free rows f of
// a_ref[f,c] X[f][a]
__global__ void k_fix_accum(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                            const double *__restrict__ a_ref, const unsigned char *__restrict__ mask,
                            const double *__restrict__ X, int ld, int nrhs, int64_t N, double *__restrict__ Y)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * nrhs; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = t / nrhs;
        const int a = (int)(t - f * nrhs);
        if (mask[f]) continue;
        const double xf = X[f * ld + a];
        for (int32_t s = rp[f]; s < rp[f + 1]; ++s) {
            const int32_t j = col[s];
            if (mask[j]) atomicAdd(&Y[(int64_t)j * nrhs + a], a_ref[s] * xf);
        }
    }
}

// The same fix-up as a gather, for structurally symmetric patterns (every
// system assembled from a mesh): one warp per constrained dof c reads the
// couplings a_ref[f, c] of its free neighbours f (found in row f by binary
// search, the columns being sorted) and forms
//   X[c][a] = (B[c][a] - sum_f a_ref[f, c] X[f][a]) / a_ref[c, c]
// in a fixed order, with no atomics and no N x nrhs scratch.
__global__ void __launch_bounds__(256) k_fix_gather(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                    const int32_t *__restrict__ diag, const double *__restrict__ a_ref,
                                                    const unsigned char *__restrict__ mask,
                                                    const double *__restrict__ B, int ld, int nrhs, int64_t N,
                                                    double *__restrict__ X)
{
    constexpr int NA = 8;  // columns per lane and pass
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < N; c += warps) {
        if (!mask[c]) continue;  // warp-uniform
        const double dcc = a_ref[diag[c]];
        const int32_t e0 = rp[c], e1 = rp[c + 1];
        for (int a0 = 0; a0 < nrhs; a0 += 32 * NA) {
            double acc[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) acc[q] = 0.0;
            for (int32_t s0 = e0; s0 < e1; s0 += 32) {
                const int32_t sl = s0 + lane;
                int32_t f = 0;
                double w = 0.0;
                if (sl < e1) {
                    f = col[sl];
                    if (f != c && !mask[f]) {
                        int32_t lo = rp[f], hi = rp[f + 1] - 1;
                        while (lo <= hi) {  // column c in the sorted row f
                            const int32_t mid = (lo + hi) >> 1;
                            const int32_t cm = col[mid];
                            if (cm == c) {
                                w = a_ref[mid];
                                break;
                            }
                            if (cm < c)
                                lo = mid + 1;
                            else
                                hi = mid - 1;
                        }
                    }
                }
                const int n = min(32, e1 - s0);
                for (int t = 0; t < n; ++t) {
                    const double wt = __shfl_sync(0xffffffffu, w, t);
                    const int32_t ft = __shfl_sync(0xffffffffu, f, t);
                    if (wt == 0.0) continue;  // warp-uniform
#pragma unroll
                    for (int q = 0; q < NA; ++q) {
                        const int a = a0 + lane + 32 * q;
                        if (a < nrhs) acc[q] += wt * X[(int64_t)ft * ld + a];
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                const int a = a0 + lane + 32 * q;
                if (a < nrhs) X[c * ld + a] = (B[c * ld + a] - acc[q]) / dcc;
            }
        }
    }
}

__global__ void k_fix_apply(const int32_t *__restrict__ diag, const double *__restrict__ a_ref,
                            const unsigned char *__restrict__ mask, const double *__restrict__ B,
                            const double *__restrict__ Y, int ld, int nrhs, int64_t N, double *__restrict__ X)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * nrhs; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t / nrhs;
        const int a = (int)(t - c * nrhs);
        if (!mask[c]) continue;
        X[c * ld + a] = (B[c * ld + a] - Y[c * nrhs + a]) / a_ref[diag[c]];
    }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
struct PcgResult {
    int iters;
    bool converged;
};

void launch_spmv64(sfc_system *s, const double *x, double *y, double *dot, const int *done)
{
    const double avg = (double)s->nnz / (double)std::max<int64_t>(s->N, 1);
    sfc_ctx *ctx = s->ctx;
    const int lanes = s->spmv_lanes;  // tuned, else chosen by the mean row length
    ProfScope ps(ctx, "spmv64",
                 (lanes == 0 && s->has_bsr ? (double)s->nblocks * 76 + 4.0 * (s->nodes + 1)
                                           : (double)s->nnz * 12 + 4.0 * (s->N + 1)) +
                     16.0 * s->N);
    const unsigned grid = (unsigned)(ctx->sm_count * 8);
    if (lanes == 0 && s->has_bsr) {  // 3-dof mesh: node blocks
        k_bspmv64<<<grid_for(s->nodes * 32, kRedThreads, grid), kRedThreads, 0, ctx->stream>>>(
            s->bptr.p, s->bcol.p, s->bval64.p, x, y, s->nodes, dot, done);
    } else if (lanes == 32 || (lanes == 0 && avg > 24))
        k_spmv64<32><<<grid_for(s->N * 32, kRedThreads, grid), kRedThreads, 0, ctx->stream>>>(s->row_ptr.p, s->col.p,
                                                                                              s->a_op.p, x, y, s->N, dot, done);
    else if (lanes == 16 || (lanes == 0 && avg > 12))
        k_spmv64<16><<<grid_for(s->N * 16, kRedThreads, grid), kRedThreads, 0, ctx->stream>>>(s->row_ptr.p, s->col.p,
                                                                                              s->a_op.p, x, y, s->N, dot, done);
    else if (lanes == 8 || (lanes == 0 && avg > 6))
        k_spmv64<8><<<grid_for(s->N * 8, kRedThreads, grid), kRedThreads, 0, ctx->stream>>>(s->row_ptr.p, s->col.p,
                                                                                            s->a_op.p, x, y, s->N, dot, done);
    else
        k_spmv64<4><<<grid_for(s->N * 4, kRedThreads, grid), kRedThreads, 0, ctx->stream>>>(s->row_ptr.p, s->col.p,
                                                                                            s->a_op.p, x, y, s->N, dot, done);
    count_launch(ctx);
}

// the two-level preconditioner is used when it is selected and the system
// has a coarse space (a 3-dof mesh with a valid box grid); builds it for the
// current operator
bool use_two_level(sfc_system *s)
{
    if (s->opt.precond != SFC_PRECOND_TWO_LEVEL) return false;
    if (s->has_bsr && !s->bdinv32.p) return false;  // 3-dof mesh without its block-Jacobi smoother
    return coarse_prepare(s);
}

// FP64 PCG on S x = b (device vectors, length N): point Jacobi, or with
// `two` the two-level preconditioner (nodal block Jacobi + coarse correction;
// the caller has run coarse_prepare)
PcgResult pcg64(sfc_system *s, const double *b, double *x, double tol, int max_iter, int check, bool two)
{
    sfc_ctx *ctx = s->ctx;
    const int64_t N = s->N;
    s->w64.reserve(3 * N);
    double *r = s->w64.p, *p = r + N, *q = p + N;
    const int nsc = 3 * (max_iter + 2) + 1;
    s->scal.reserve(nsc);
    double *pq = s->scal.p, *rz = pq + (max_iter + 2), *rr = rz + (max_iter + 2), *bb = rr + (max_iter + 2);
    s->flags.reserve(2);
    int *done = s->flags.p, *err = s->flags.p + 1;
    SFC_CK(cudaMemsetAsync(s->scal.p, 0, nsc * sizeof(double), ctx->stream));
    SFC_CK(cudaMemsetAsync(s->flags.p, 0, 2 * sizeof(int), ctx->stream));
    const unsigned g = grid_for(N, kRedThreads, ctx->sm_count * 4);
    const int64_t nodes = s->nodes;
    const unsigned gn = grid_for(nodes, kRedThreads, ctx->sm_count * 4);
    const CoarseSpace &cs = s->coarse;
    const bool two1 = two && cs.dof == 1;  // scalar mesh: point Jacobi + constant modes
    two = two && cs.dof == 3;
    if (two1) {
        k_pcg_init<<<g, kRedThreads, 0, ctx->stream>>>(b, s->dinv.p, x, r, p, N, rz, bb);  // rz: Jacobi share
        count_launch(ctx);
        coarse_vec_apply(s, r, rz, nullptr);
        k_pcg1_pupdate<true><<<g, kRedThreads, 0, ctx->stream>>>(p, r, s->dinv.p, cs.node_agg.p, cs.mode.p, cs.e64.p,
                                                                 N, nullptr, nullptr, nullptr, 0.0, 0, done, err);
    } else if (two) {
        k_pcg2_init<<<gn, kRedThreads, 0, ctx->stream>>>(b, s->bdinv32.p, x, r, nodes, rz, bb);
        count_launch(ctx);
        coarse_vec_apply(s, r, rz, nullptr);
        k_pcg2_pupdate<true><<<gn, kRedThreads, 0, ctx->stream>>>(p, r, s->bdinv32.p, cs.node_agg.p, cs.mode.p,
                                                                  cs.e64.p, nodes, nullptr, nullptr, nullptr, 0.0, 0,
                                                                  done, err);
    } else {
        k_pcg_init<<<g, kRedThreads, 0, ctx->stream>>>(b, s->dinv.p, x, r, p, N, rz, bb);
    }
    count_launch(ctx);
    double hbb = 0;
    download(ctx, &hbb, bb, 1);
    if (hbb == 0.0) return {0, true};
    const double thr = tol * tol * hbb;
    int it = 0;
    PcgResult res{max_iter, false};
    for (it = 0; it < max_iter; ++it) {
        launch_spmv64(s, p, q, pq + it, done);
        if (two) {
            {
                ProfScope ps(ctx, "pcg_update", 56.0 * N + 36.0 * nodes);
                k_pcg2_update<<<gn, kRedThreads, 0, ctx->stream>>>(x, r, p, q, s->bdinv32.p, nodes, pq + it, rz + it,
                                                                   rz + it + 1, rr + it + 1, done, err);
            }
            count_launch(ctx);
            coarse_vec_apply(s, r, rz + it + 1, done);
            {
                ProfScope ps(ctx, "pcg_pupdate", 32.0 * N + 56.0 * nodes);
                k_pcg2_pupdate<false><<<gn, kRedThreads, 0, ctx->stream>>>(
                    p, r, s->bdinv32.p, cs.node_agg.p, cs.mode.p, cs.e64.p, nodes, rz + it, rz + it + 1, rr + it + 1,
                    thr, it + 1, done, err);
            }
            count_launch(ctx);
        } else {
            {
                ProfScope ps(ctx, "pcg_update", 56.0 * N);
                k_pcg_update<<<g, kRedThreads, 0, ctx->stream>>>(x, r, p, q, s->dinv.p, N, pq + it, rz + it,
                                                                 rz + it + 1, rr + it + 1, done, err);
            }
            if (two1) {
                count_launch(ctx);
                coarse_vec_apply(s, r, rz + it + 1, done);
                ProfScope ps(ctx, "pcg_pupdate", 32.0 * N + 12.0 * N);
                k_pcg1_pupdate<false><<<g, kRedThreads, 0, ctx->stream>>>(p, r, s->dinv.p, cs.node_agg.p, cs.mode.p,
                                                                          cs.e64.p, N, rz + it, rz + it + 1,
                                                                          rr + it + 1, thr, it + 1, done, err);
                count_launch(ctx);
            } else {
                ProfScope ps(ctx, "pcg_pupdate", 32.0 * N);
                k_pcg_pupdate<<<g, kRedThreads, 0, ctx->stream>>>(p, r, s->dinv.p, N, rz + it, rz + it + 1,
                                                                  rr + it + 1, thr, it + 1, done, err);
                count_launch(ctx, 2);
            }
        }
        if ((it + 1) % check == 0 || it + 1 == max_iter) {
            int hf[2];
            download(ctx, hf, s->flags.p, 2);
            if (hf[1]) fail(SFC_ERR_NOT_SPD, "PCG breakdown: p^T A p <= 0");
            if (hf[0]) {
                res = {hf[0], true};
                break;
            }
        }
    }
    return res;
}

double true_rel_residual(sfc_system *s, const double *b, const double *x)
{
    sfc_ctx *ctx = s->ctx;
    const int64_t N = s->N;
    s->tmpN2.reserve(N);
    DBuf<double> &t = s->tmpN2;
    struct {
        double *p;
    } d{ctx->dsmall.p};
    SFC_CK(cudaMemsetAsync(d.p, 0, 2 * sizeof(double), ctx->stream));
    launch_spmv64(s, x, t.p, nullptr, nullptr);
    k_axpby<<<grid_for(N, 256), 256, 0, ctx->stream>>>(t.p, b, 1.0, -1.0, N);  // t = b - Sx
    const unsigned g = grid_for(N, kRedThreads, ctx->sm_count * 4);
    k_dot<<<g, kRedThreads, 0, ctx->stream>>>(t.p, t.p, N, d.p);
    k_dot<<<g, kRedThreads, 0, ctx->stream>>>(b, b, N, d.p + 1);
    count_launch(ctx, 3);
    double h[2];
    download(ctx, h, d.p, 2);
    return h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
}

template <int V>
void block_mixed(sfc_system *s, const double *B, double *X, int nrhs, int ld, sfc_solve_stats_t &st)
{
    constexpr int K = 32 * V;
    sfc_ctx *ctx = s->ctx;
    const int64_t N = s->N;
    const auto &o = s->opt;
    const int max_iter = o.max_iter > 0 ? o.max_iter : 20000;
    const int check = o.check_every > 0 ? o.check_every : 16;
    const double tol = o.tol > 0 ? o.tol : 1e-8;
    const double itol = o.inner_tol > 0 ? o.inner_tol : 1e-4;
    // persistent workspaces (grown, never freed per call)
    s->blk64.reserve(3 * N * K);
    s->blk32.reserve(4 * N * K);
    s->colsc.reserve(6 * K);
    struct {
        double *p;
    } b64{s->blk64.p}, x64{s->blk64.p + N * K}, r64{s->blk64.p + 2 * N * K}, cs{s->colsc.p};
    float *xr = s->blk32.p, *rr32 = xr + N * K, *pp = rr32 + N * K, *qq = pp + N * K;
    // Per-iteration column scalars in a ring of R slots of 3K doubles
    // (p.q | r.z | r.r).  Iteration it reads r.z and r.r of slot it % R and
    // accumulates its p.q, the new r.z and the new r.r into slot (it+1) % R,
    // which it zeroes first (the slot's last reader, iteration it+1-R, is
    // done).  With R = check every check interval uses the same slots, so
    // one captured graph serves every interval.
    const int R = check >= 2 ? check : 2;
    const int64_t nsc = 3 * (int64_t)R * K;
    s->scal.reserve(nsc);
    auto sl = [&](int i) { return s->scal.p + (int64_t)(i % R) * 3 * K; };
    double *bn2 = cs.p, *rn2 = bn2 + K, *scale = rn2 + K, *norm = scale + K, *thr = norm + K;
    // flags[0]: all columns below their thresholds; flags[1 + c]: breakdown
    // (p^T A p <= 0) in column c; flags[1 + K]: iterations of the current
    // check interval that ran before flags[0] was set (0: all of them)
    s->flags.reserve(2 + K);
    int *stop = s->flags.p, *err = s->flags.p + 1, *ran = s->flags.p + 1 + K;
    std::vector<int> hflags(2 + K), nbreak(K), fallback(K), nstall(K);
    int n_fallback = 0;
    const bool debug = std::getenv("SFC_DEBUG_SOLVER") != nullptr;
    const unsigned gw = (unsigned)(ctx->sm_count * 8);  // warp-per-row kernels: 8 warps/block
    const bool bsr = s->has_bsr;
    const bool two_any = use_two_level(s);
    const CoarseSpace &crs = s->coarse;
    const bool two = two_any && crs.dof == 3;   // block Jacobi + rigid-body modes
    const bool two1 = two_any && crs.dof == 1;  // point Jacobi + constant modes (scalar mesh)
    const bool bj = bsr && (o.precond == SFC_PRECOND_BLOCK_JACOBI || two) && s->bdinv32.p;
    // two-level with block Jacobi: the r update and the coarse restriction in
    // one pass over r (SFC_RESTRICT=separate keeps the two kernels)
    const char *fenv = std::getenv("SFC_RESTRICT");
    const bool fuse_restrict = two && bj && !(fenv && std::string(fenv) == "separate");
    // R = B - S X (FP64) and Q = S P (FP32), node-block kernels for 3-dof meshes
    // the true residual on the lattice view unless SFC_RESID=bsr
    const char *renv = std::getenv("SFC_RESID");
    const bool xresid_off = renv && std::string(renv) == "bsr";
    if (bsr && s->has_lattice && s->bq64.p && !xresid_off) xresid_prepare(K);
    auto resid = [&](const double *X, const double *Bm, double *R, double *out) {
        ProfScope ps(ctx, "resid64",
                     bsr ? (double)s->nblocks * 76 + 4.0 * (s->nodes + 1) + 3.0 * N * K * 8
                         : (double)s->nnz * 12 + 4.0 * (N + 1) + 3.0 * N * K * 8);
        if (bsr && s->has_lattice && s->bq64.p && !xresid_off) {
            xline_resid64(s, X, Bm, R, K, out);
            return;
        }
        if (bsr)
            k_bresid64<V><<<gw, 256, 0, ctx->stream>>>(s->bptr.p, s->bcol.p, s->bval64.p, X, Bm, R, s->nodes, out);
        else
            k_resid64<V><<<gw, 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->a_op.p, X, Bm, R, N, out);
        count_launch(ctx);
    };
    auto spmm = [&](const float *Pm, float *Qm, double *out) {
        ProfScope ps(ctx, "spmm32",
                     bsr ? (double)s->nblocks * 40 + 4.0 * (s->nodes + 1) + 2.0 * N * K * 4
                         : (double)s->nnz * 8 + 4.0 * (N + 1) + 2.0 * N * K * 4);
        if (bsr && s->has_lattice && s->lat_mode == 2) {
            xline_spmm32(s, Pm, Qm, K, out, stop);
            return;
        }
        if (bsr && s->has_lattice && s->lat_mode == 1 && K >= 64) {
            lattice_spmm32(s, Pm, Qm, K, out, stop);
            return;
        }
        if (bsr)
            k_bspmm32<V><<<gw, 256, 0, ctx->stream>>>(s->bptr.p, s->bcol.p, s->bval32.p, Pm, Qm, s->nodes, out, stop);
        else
            k_spmm32<V><<<gw, 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->a_op32.p, Pm, Qm, N, out, stop);
        count_launch(ctx);
    };
    s->restart.reserve(K);
    DBuf<int> &restart = s->restart;
    // r32 = scaled r64, x32 = 0, p = z for restarted columns; rz, rr into the slots
    auto init32 = [&](double *rz_slot, double *rr_slot) {
        if (two) {
            // p = z needs the coarse correction of the new residual first
            k_ninit32<V, false><<<gw, 256, 0, ctx->stream>>>(r64.p, scale, s->bdinv32.p, restart.p, rr32, xr, pp,
                                                             s->nodes, rz_slot, rr_slot);
            count_launch(ctx);
            coarse_block_apply<V>(s, rr32, rz_slot, nullptr);
            k_ncpupdate32<V, true><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->bdinv32.p, crs.node_agg.p, crs.mode.p,
                                                                crs.e32.p, s->nodes, nullptr, nullptr, nullptr,
                                                                nullptr, nullptr, nullptr, restart.p, nullptr, nullptr,
                                                                nullptr);
        } else if (two1) {
            k_binit32<V, false><<<gw, 256, 0, ctx->stream>>>(r64.p, scale, s->dinv32.p, restart.p, rr32, xr, pp, N,
                                                             rz_slot, rr_slot);
            count_launch(ctx);
            coarse_block_apply<V>(s, rr32, rz_slot, nullptr);
            k_cbpupdate32<V, true><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->dinv32.p, crs.node_agg.p, crs.mode.p,
                                                                crs.e32.p, N, nullptr, nullptr, nullptr, nullptr,
                                                                nullptr, nullptr, restart.p);
        } else if (bj)
            k_ninit32<V><<<gw, 256, 0, ctx->stream>>>(r64.p, scale, s->bdinv32.p, restart.p, rr32, xr, pp, s->nodes,
                                                      rz_slot, rr_slot);
        else
            k_binit32<V><<<gw, 256, 0, ctx->stream>>>(r64.p, scale, s->dinv32.p, restart.p, rr32, xr, pp, N, rz_slot,
                                                      rr_slot);
        count_launch(ctx);
    };
    // one inner iteration: Q = S P, alpha, x/r update with r.z and r.r,
    // coarse correction, beta and the p update
    auto iterate = [&](int it) {
        double *cur = sl(it), *nxt = sl(it + 1);
        SFC_CK(cudaMemsetAsync(nxt, 0, (size_t)3 * K * 8, ctx->stream));
        double *pqi = nxt, *rz0 = cur + K, *rr0 = cur + 2 * K, *rz1 = nxt + K, *rr1 = nxt + 2 * K;
        spmm(pp, qq, pqi);
        if (fuse_restrict) {
            coarse_block_reserve(s, K);  // no-op once reserved (always, inside a capture)
            {
                ProfScope ps(ctx, "nrupdate32", 3.0 * N * K * 4 + 52.0 * s->nodes + 4.0 * crs.nc * K);
                constexpr int W = 8, S = 2;  // 16 warps per aggregate
                k_nrupdate32<V, W, S><<<(unsigned)(crs.nagg * S), 32 * W, 0, ctx->stream>>>(
                    rr32, qq, s->bdinv32.p, crs.agg_ptr.p, crs.agg_nodes.p, crs.mode.p, crs.c32.p, pqi, rz0, rr0,
                    thr, rz1, rr1, stop, err);
            }
            count_launch(ctx);
            coarse_block_gemm<V>(s, rz1, stop);
        } else {
            {
                ProfScope ps(ctx, "bupdate32", (bj ? 3.0 : 6.0) * N * K * 4 + (bj ? 12.0 : 4.0) * N);
                if (bj)
                    k_nupdate32<V, false><<<gw, 256, 0, ctx->stream>>>(xr, rr32, pp, qq, s->bdinv32.p, s->nodes,
                                                                       pqi, rz0, rr0, thr, rz1, rr1, stop, err);
                else
                    k_bupdate32<V><<<gw, 256, 0, ctx->stream>>>(xr, rr32, pp, qq, s->dinv32.p, N, pqi, rz0,
                                                                rr0, thr, rz1, rr1, stop, err);
            }
            count_launch(ctx);
            if (two_any) coarse_block_apply<V>(s, rr32, rz1, stop);
        }
        {
            ProfScope ps(ctx, "bpupdate32",
                         (bj ? 5.0 : 3.0) * N * K * 4 + (bj ? 12.0 : 4.0) * N + (two ? 8.0 * s->nodes : 0.0));
            if (two)
                k_ncpupdate32<V, false><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->bdinv32.p, crs.node_agg.p,
                                                                     crs.mode.p, crs.e32.p, s->nodes, rz0, rz1,
                                                                     rr1, thr, stop, err, nullptr, xr, pqi,
                                                                     rr0);
            else if (bj)
                k_npupdate32<V><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->bdinv32.p, s->nodes, rz0, rz1,
                                                             rr1, thr, stop, err, xr, pqi, rr0);
            else if (two1)
                k_cbpupdate32<V, false><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->dinv32.p, crs.node_agg.p,
                                                                     crs.mode.p, crs.e32.p, N, rz0, rz1,
                                                                     rr1, thr, stop, err, nullptr);
            else
                k_bpupdate32<V><<<gw, 256, 0, ctx->stream>>>(pp, rr32, s->dinv32.p, N, rz0, rz1, rr1,
                                                             thr, stop, err);
        }
        // convergence after every iteration: the rest of the interval returns
        // at once when all columns are below their thresholds
        k_bcheck_it<K><<<1, 128, 0, ctx->stream>>>(rr1, thr, stop, ran, it % check);
        count_launch(ctx, 2);
    };
    // A whole check interval as one CUDA graph: the ring's zeroing, `check`
    // iterations and the convergence flag, captured once per launch
    // configuration (the key lists every pointer and size baked into the
    // launches) and replayed for every later interval.  Not used while kernel
    // profiling records events around each launch, nor with
    // SFC_BLOCK_GRAPH=0 in the environment.
    const char *genv = std::getenv("SFC_BLOCK_GRAPH");
    const bool use_graph = !ctx->prof && check >= 2 && !(genv && genv[0] == '0');
    const bool lattice = bsr && s->has_lattice && s->lat_mode == 1 && K >= 64;
    auto launch_chunk_graph = [&]() -> bool {
        GraphExec &g = s->blk_graph[V == 1 ? 0 : V == 2 ? 1 : 2];
        // everything the captured launches allocate or set up, done outside the capture
        if (two_any) coarse_block_reserve(s, K);
        if (lattice) lattice_prepare(s, pp, K);
        if (bsr && s->has_lattice && s->lat_mode == 2) xline_prepare(K);
        const std::vector<uintptr_t> key = {
            (uintptr_t)K, (uintptr_t)check, (uintptr_t)N, (uintptr_t)s->nodes, (uintptr_t)gw,
            (uintptr_t)(bsr | (bj << 1) | (two << 2) | (two1 << 3) | (lattice << 4) | (fuse_restrict << 5)),
            (uintptr_t)s->scal.p,
            (uintptr_t)s->blk32.p, (uintptr_t)s->colsc.p, (uintptr_t)s->flags.p, (uintptr_t)s->bdinv32.p,
            (uintptr_t)s->dinv32.p, (uintptr_t)s->bptr.p, (uintptr_t)s->bcol.p, (uintptr_t)s->bval32.p,
            (uintptr_t)s->row_ptr.p, (uintptr_t)s->col.p, (uintptr_t)s->a_op32.p, (uintptr_t)s->bq.p, (uintptr_t)s->bq64.p,
            (uintptr_t)s->lat_err.p, (uintptr_t)s->lat_mode, (uintptr_t)s->lat[0], (uintptr_t)s->lat[1], (uintptr_t)s->lat[2],
            (uintptr_t)s->pmap_ptr, (uintptr_t)crs.agg_ptr.p, (uintptr_t)crs.agg_nodes.p, (uintptr_t)crs.mode.p,
            (uintptr_t)crs.c32.p, (uintptr_t)crs.e32.p, (uintptr_t)crs.a32.p, (uintptr_t)crs.node_agg.p,
            (uintptr_t)crs.nagg, (uintptr_t)crs.nc, (uintptr_t)crs.dof};
        if (!g.exec || g.key != key) {
            g.reset();
            if (g.failed_key == key) return false;  // this configuration could not be captured: eager
            cudaStream_t st;
            SFC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            const cudaStream_t keep = ctx->stream;
            const int64_t l0 = ctx->launches;
            cudaGraph_t graph = nullptr;
            const char *where = "cudaStreamBeginCapture";
            cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                ctx->stream = st;
                try {
                    for (int j = 0; j < check; ++j) iterate(j);
                } catch (...) {
                    ctx->stream = keep;
                    cudaStreamEndCapture(st, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    cudaStreamDestroy(st);
                    ctx->launches = l0;
                    throw;
                }
                ctx->stream = keep;
                where = "cudaStreamEndCapture";
                e = cudaStreamEndCapture(st, &graph);
            }
            cudaStreamDestroy(st);
            const int64_t captured = ctx->launches - l0;
            ctx->launches = l0;
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) {
                where = "cudaGraphInstantiate";
                e = cudaGraphInstantiate(&exec, graph, 0);
            }
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                // not fatal: the same launches go out one by one; the reason
                // is kept as the context's message (sfc_last_error)
                cudaGetLastError();
                g.failed_key = key;
                ctx->err = std::string("block solver graph not used: ") + where + ": " + cudaGetErrorString(e);
                if (debug) std::fprintf(stderr, "[sfc] %s\n", ctx->err.c_str());
                return false;
            }
            g.exec = exec;
            g.key = key;
            g.kernels = captured;
        }
        SFC_CK(cudaGraphLaunch(g.exec, ctx->stream));
        ctx->launches += g.kernels;
        ++ctx->graph_replays;
        return true;
    };
    // Reliable-update mixed-precision block PCG.  Each column is scaled to
    // ||b|| = 1 and iterated in FP32; whenever every active column's recurrence
    // residual has dropped by a decade since the last update (or has fallen
    // below its freeze threshold), x32 is folded into the FP64 solution, the
    // true residual b - S x is recomputed in FP64 and replaces r in the FP32
    // iteration while the search direction p is kept (no Krylov restart).
    // Columns whose true residual meets tol are frozen; a column whose
    // recurrence fell below its threshold while the true residual did not
    // restarts from p = z with a tighter threshold.
    std::vector<double> hb(K), hs(K), hn(K), ht(K), rr_last(K), rr_now(K), rn(K);
    std::vector<int> hrestart(K);
    int max_inner = 0, max_updates = 0;
    double worst = 0.0;
    bool all_conv = true;
    for (int c0 = 0; c0 < nrhs; c0 += K) {
        const int kb = std::min(K, nrhs - c0);
        k_gather_cols<<<grid_for(N * K, 256), 256, 0, ctx->stream>>>(B, ld, c0, kb, K, N, b64.p);
        SFC_CK(cudaMemsetAsync(x64.p, 0, N * K * 8, ctx->stream));
        SFC_CK(cudaMemsetAsync(cs.p, 0, 6 * K * 8, ctx->stream));
        SFC_CK(cudaMemsetAsync(s->scal.p, 0, nsc * 8, ctx->stream));
        SFC_CK(cudaMemsetAsync(s->flags.p, 0, (2 + K) * sizeof(int), ctx->stream));
        std::fill(nbreak.begin(), nbreak.end(), 0);
        std::fill(fallback.begin(), fallback.end(), 0);
        std::fill(nstall.begin(), nstall.end(), 0);
        int it_update = 0, last_interval = 0;
        count_launch(ctx);
        {  // x = 0: r64 = b, ||b_c||^2
            ProfScope ps(ctx, "resid64", 16.0 * N * K);
            k_bcopy_norm64<V><<<gw, 256, 0, ctx->stream>>>(b64.p, r64.p, N, bn2);
            count_launch(ctx);
        }
        download(ctx, hb.data(), bn2, K);
        std::vector<bool> active(K);
        int nactive = 0;
        for (int c = 0; c < K; ++c) {
            const double bn = std::sqrt(hb[c]);
            active[c] = c < kb && bn > 0.0;
            nactive += active[c];
            hs[c] = active[c] ? 1.0 / bn : 0.0;
            hn[c] = active[c] ? bn : 0.0;
            ht[c] = active[c] ? (0.1 * tol) * (0.1 * tol) : INFINITY;
            rr_last[c] = 1.0;
            rn[c] = active[c] ? bn : 0.0;
            hrestart[c] = 1;
        }
        int it = 0, updates = 0, real_it = 0;
        if (nactive > 0) {
            SFC_CK(cudaMemcpyAsync(scale, hs.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
            SFC_CK(cudaMemcpyAsync(norm, hn.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
            SFC_CK(cudaMemcpyAsync(thr, ht.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
            SFC_CK(cudaMemcpyAsync(restart.p, hrestart.data(), K * 4, cudaMemcpyHostToDevice, ctx->stream));
            init32(sl(0) + K, sl(0) + 2 * K);
        }
        while (nactive > 0) {
            const int it0 = it - it % check;  // first iteration of this check interval
            bool ran_graph = false;
            if (it % check == 0 && use_graph && it + check <= max_iter && launch_chunk_graph()) {
                it += check;
                ran_graph = true;
            } else {
                iterate(it);
                ++it;
            }
            double *rz1 = sl(it) + K, *rr1 = sl(it) + 2 * K;
            const bool at_cap = it >= max_iter;
            if (!ran_graph && it % check != 0 && !at_cap) continue;
            download(ctx, hflags.data(), s->flags.p, 2 + K);
            // `it` counts whole intervals (the ring and the captured graph
            // follow it); the iterations that ran end at it0 + ran, whose
            // slot no later (returning) iteration of the interval zeroes
            const int ran_now = hflags[1 + K] > 0 ? hflags[1 + K] : it - it0;
            real_it += ran_now;
            download(ctx, rr_now.data(), sl(it0 + ran_now) + 2 * K, K);
            bool update = hflags[0] || at_cap;
            for (int c = 0; c < K; ++c)
                if (active[c] && hflags[1 + c]) {
                    // a breakdown restarts the column at the next update; a
                    // column that keeps breaking down (p^T S p lost in FP32
                    // rounding near the end of a tight solve) leaves the FP32
                    // iteration and is finished by FP64 Jacobi-PCG below
                    if (++nbreak[c] > 4) fallback[c] = 1;
                    update = true;
                }
            if (!update) {
                update = true;
                for (int c = 0; c < K; ++c)
                    if (active[c] && rr_now[c] > ht[c] && rr_now[c] > 1e-2 * rr_last[c]) update = false;
            }
            // a column whose FP32 recurrence stagnates (p^T S p dominated by
            // rounding on ill-conditioned smooth modes) would hold the whole
            // block back: force the update after three times the previous
            // interval (at least 512 iterations)
            if (!update && it - it_update >= std::max(512, 3 * last_interval)) update = true;
            if (!update) continue;
            last_interval = it - it_update;
            it_update = it;
            // reliable update: x64 += ||b|| x32, true FP64 residual
            k_bacc64<V><<<grid_for(N * K, 256), 256, 0, ctx->stream>>>(x64.p, xr, norm, N);
            count_launch(ctx);
            SFC_CK(cudaMemsetAsync(rn2, 0, K * 8, ctx->stream));
            resid(x64.p, b64.p, r64.p, rn2);
            download(ctx, rn.data(), rn2, K);
            ++updates;
            if (debug) {
                double wr = 0, wrec = 0;
                int nb = 0;
                for (int c = 0; c < K; ++c)
                    if (active[c]) {
                        wr = std::max(wr, std::sqrt(rn[c]) / hn[c]);
                        wrec = std::max(wrec, std::sqrt(rr_now[c]));
                        nb += hflags[1 + c];
                    }
                std::fprintf(stderr, "[sfc block %d] it %d update %d: max true rel %.3e max recurrence %.3e breakdowns %d\n",
                             c0, it, updates, wr, wrec, nb);
            }
            nactive = 0;
            for (int c = 0; c < K; ++c) {
                hrestart[c] = 0;
                if (!active[c]) continue;
                const double bn = hn[c], r = std::sqrt(rn[c]);
                if (r <= tol * bn) {
                    active[c] = false;
                    ht[c] = INFINITY;
                    continue;
                }
                // no progress of the true residual over three updates in a
                // row: FP32 cannot resolve this column any further
                if ((r / bn) * (r / bn) >= 0.25 * rr_last[c]) {
                    if (++nstall[c] >= 3) fallback[c] = 1;
                } else {
                    nstall[c] = 0;
                }
                if (fallback[c]) {
                    active[c] = false;
                    ht[c] = INFINITY;
                    continue;
                }
                ++nactive;
                if (rr_now[c] <= ht[c]) {  // recurrence converged, true residual not
                    ht[c] = std::max(ht[c] * 1e-2, 1e-30);
                    hrestart[c] = 1;
                }
                if (hflags[1 + c]) hrestart[c] = 1;
                // Keeping p after the residual replacement is only consistent
                // when the FP32 recurrence still tracks the true residual; when
                // they have drifted apart (fast convergence between checks),
                // the column restarts from p = z instead.
                const double rec = std::sqrt(rr_now[c]), tru = r / bn;
                if (!(tru <= 1.5 * rec && rec <= 1.5 * tru)) hrestart[c] = 1;
                rr_last[c] = (r / bn) * (r / bn);
            }
            if (nactive == 0 || at_cap) break;
            SFC_CK(cudaMemcpyAsync(thr, ht.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
            SFC_CK(cudaMemcpyAsync(restart.p, hrestart.data(), K * 4, cudaMemcpyHostToDevice, ctx->stream));
            SFC_CK(cudaMemsetAsync(sl(it), 0, (size_t)3 * K * 8, ctx->stream));
            SFC_CK(cudaMemsetAsync(s->flags.p, 0, (2 + K) * sizeof(int), ctx->stream));
            // r32 <- scaled true residual, x32 <- 0, p kept (restarted columns: p = z)
            init32(rz1, rr1);
        }
        // FP64 fallback: S d = r_c (the column's true residual) by Jacobi-PCG
        // to tol ||b_c|| / ||r_c||, then x_c += d
        bool any_fb = false;
        for (int c = 0; c < kb; ++c) {
            if (!fallback[c]) continue;
            any_fb = true;
            ++n_fallback;
            s->tmpN.reserve(N);
            s->tmpN2.reserve(N);
            k_gather_cols<<<grid_for(N, 256), 256, 0, ctx->stream>>>(r64.p, K, c, 1, 1, N, s->tmpN.p);
            count_launch(ctx);
            const double bn = std::sqrt(hb[c]), r = std::sqrt(rn[c]);
            if (r > tol * bn) {
                PcgResult pr = pcg64(s, s->tmpN.p, s->tmpN2.p, tol * bn / r, max_iter, check, two_any);
                if (!pr.converged) all_conv = false;
                if (debug)
                    std::fprintf(stderr, "[sfc block %d] column %d: FP64 fallback from rel %.3e, %d iterations%s\n", c0,
                                 c, r / bn, pr.iters, pr.converged ? "" : " (not converged)");
                k_add_col<<<grid_for(N, 256), 256, 0, ctx->stream>>>(x64.p, K, c, s->tmpN2.p, N);
                count_launch(ctx);
            }
        }
        if (any_fb) {
            SFC_CK(cudaMemsetAsync(rn2, 0, K * 8, ctx->stream));
            resid(x64.p, b64.p, r64.p, rn2);
            download(ctx, rn.data(), rn2, K);
        }
        for (int c = 0; c < kb; ++c) {
            const double bn = std::sqrt(hb[c]);
            if (bn > 0) worst = std::max(worst, std::sqrt(rn[c]) / bn);
        }
        if (nactive > 0) {
            all_conv = false;
            if (debug)
                std::fprintf(stderr, "[sfc block %d] %d columns still open after %d iterations\n", c0, nactive, real_it);
        }
        k_scatter_cols<<<grid_for(N * kb, 256), 256, 0, ctx->stream>>>(x64.p, ld, c0, kb, K, N, X);
        count_launch(ctx);
        max_inner = std::max(max_inner, real_it);
        max_updates = std::max(max_updates, updates);
    }
    SFC_CK(cudaStreamSynchronize(ctx->stream));
    lattice_check(s);
    st.iterations = max_inner;
    st.refinements = max_updates;
    st.num_rhs = nrhs;
    st.max_rel_residual = worst;
    st.converged = all_conv ? 1 : 0;
    st.fallback_columns = n_fallback;
    st.coarse_dofs = two_any ? (int32_t)(crs.nc - crs.dropped) : 0;
    st.spmm_kernel = !bsr ? 1
                     : s->has_lattice && s->lat_mode == 2 ? 4
                     : s->has_lattice && s->lat_mode == 1 && K >= 64 ? 3
                                                                    : 2;
}

}  // namespace

// y = S x with the FP64 operator (used by the flexible solver in mpnn.cu)
void spmv_op64(sfc_system *s, const double *x, double *y) { launch_spmv64(s, x, y, nullptr, nullptr); }
void spmv_op64_lanes(sfc_system *s, int lanes, const double *x, double *y)
{
    const int keep = s->spmv_lanes;
    s->spmv_lanes = lanes;
    launch_spmv64(s, x, y, nullptr, nullptr);
    s->spmv_lanes = keep;
}
void spmv_op64_dot(sfc_system *s, const double *x, double *y, double *xy, const int *done)
{
    launch_spmv64(s, x, y, xy, done);
}

// lifted right-hand side b = F - K_fc u_c (see k_lift)
void lifted_rhs(sfc_system *s, double *b)
{
    k_lift<<<grid_for(s->N, 256), 256, 0, s->ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_ref.p, s->mask.p,
                                                           s->F.p, s->N, b);
    count_launch(s->ctx);
}

PcgStats pcg64_public(sfc_system *s, const double *b, double *x, double tol, int max_iter, int check)
{
    PcgResult r = pcg64(s, b, x, tol, max_iter, check, false);
    return {r.iters, r.converged};
}

double device_dot(sfc_ctx *ctx, const double *a, const double *b, int64_t n)
{
    struct {
        double *p;
    } d{ctx->dsmall.p + 4};
    SFC_CK(cudaMemsetAsync(d.p, 0, sizeof(double), ctx->stream));
    k_dot<<<grid_for(n, kRedThreads, ctx->sm_count * 4), kRedThreads, 0, ctx->stream>>>(a, b, n, d.p);
    count_launch(ctx);
    double h = 0;
    download(ctx, &h, d.p, 1);
    return h;
}

// X = A^-1 F into s->X
void solve_forward(sfc_system *s)
{
    sfc_ctx *ctx = s->ctx;
    if (s->opt.method == SFC_SOLVER_FCG_MPNN) {
        ProfScope ps(ctx, "phase:forward_solve", 0.0);
        solve_forward_fcg(s);
        return;
    }
    build_operator(s);
    const int64_t N = s->N;
    s->X.alloc(N);
    s->fwd_rhs.reserve(N);
    DBuf<double> &b = s->fwd_rhs;
    k_lift<<<grid_for(N, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_ref.p, s->mask.p, s->F.p,
                                                      N, b.p);
    count_launch(ctx);
    const auto &o = s->opt;
    const int max_iter = o.max_iter > 0 ? o.max_iter : 20000;
    const int check = o.check_every > 0 ? o.check_every : 16;
    const double tol = o.tol > 0 ? o.tol : 1e-8;
    s->solve_ev.ensure();
    cudaEvent_t e0 = s->solve_ev.a, e1 = s->solve_ev.b;
    SFC_CK(cudaEventRecord(e0, ctx->stream));
    PcgResult r;
    bool two = false;
    {
        ProfScope ps(ctx, "phase:forward_solve", 0.0);
        two = use_two_level(s);
        r = pcg64(s, b.p, s->X.p, tol, max_iter, check, two);
    }
    SFC_CK(cudaEventRecord(e1, ctx->stream));
    const double rel = true_rel_residual(s, b.p, s->X.p);
    float ms = 0;
    SFC_CK(cudaEventSynchronize(e1));
    SFC_CK(cudaEventElapsedTime(&ms, e0, e1));
    s->stats = {};
    s->stats.iterations = r.iters;
    s->stats.num_rhs = 1;
    s->stats.converged = r.converged ? 1 : 0;
    s->stats.max_rel_residual = rel;
    s->stats.device_ms = ms;
    s->stats.coarse_dofs = two ? (int32_t)(s->coarse.nc - s->coarse.dropped) : 0;
    if (!r.converged) fail(SFC_ERR_NOT_CONVERGED, "PCG did not converge within max_iter");
}

// S X = B for nrhs columns of the [N][ld] arrays (free-dof part of A^T solves;
// constrained rows come out as B_c / scalar, fixed up by transpose_fixup)
void solve_block(sfc_system *s, const double *B, double *X, int nrhs, int ld)
{
    sfc_ctx *ctx = s->ctx;
    build_operator(s);
    const int64_t N = s->N;
    s->solve_ev.ensure();
    cudaEvent_t e0 = s->solve_ev.a, e1 = s->solve_ev.b;
    SFC_CK(cudaEventRecord(e0, ctx->stream));
    sfc_solve_stats_t st{};
    const auto &o = s->opt;
    if (o.method == SFC_SOLVER_PCG_MIXED) {
        int bw = o.block_width > 0 ? o.block_width : (nrhs > 64 ? 128 : 64);
        if (nrhs <= 32) bw = 32;
        if (bw <= 32)
            block_mixed<1>(s, B, X, nrhs, ld, st);
        else if (bw <= 64)
            block_mixed<2>(s, B, X, nrhs, ld, st);
        else
            block_mixed<4>(s, B, X, nrhs, ld, st);
    } else {
        const int max_iter = o.max_iter > 0 ? o.max_iter : 20000;
        const int check = o.check_every > 0 ? o.check_every : 16;
        const double tol = o.tol > 0 ? o.tol : 1e-8;
        s->tmpN.reserve(N);
        s->blk64.reserve(N);
        DBuf<double> &b = s->tmpN, &x = s->blk64;
        const bool two = use_two_level(s);
        st.converged = 1;
        st.coarse_dofs = two ? (int32_t)(s->coarse.nc - s->coarse.dropped) : 0;
        for (int a = 0; a < nrhs; ++a) {
            k_gather_cols<<<grid_for(N, 256), 256, 0, ctx->stream>>>(B, ld, a, 1, 1, N, b.p);
            count_launch(ctx);
            PcgResult r = pcg64(s, b.p, x.p, tol, max_iter, check, two);
            st.iterations = std::max(st.iterations, r.iters);
            if (!r.converged) st.converged = 0;
            k_scatter_cols<<<grid_for(N, 256), 256, 0, ctx->stream>>>(x.p, ld, a, 1, 1, N, X);
            count_launch(ctx);
        }
        st.num_rhs = nrhs;
        st.refinements = 0;
        st.max_rel_residual = -1.0;  // recurrence residual below tol for each RHS
    }
    SFC_CK(cudaEventRecord(e1, ctx->stream));
    float ms = 0;
    SFC_CK(cudaEventSynchronize(e1));
    SFC_CK(cudaEventElapsedTime(&ms, e0, e1));
    st.device_ms = ms;
    s->stats = st;
    if (!st.converged) fail(SFC_ERR_NOT_CONVERGED, "block PCG did not converge within max_iter");
}

// A X = B for nrhs interleaved columns with the reference's row-zeroed A:
// constrained rows give x_c = b_c / a_cc, the free rows solve
// S x_f = b_f - K_fc x_c (one block solve of the lifted right-hand sides)
void solve_multi(sfc_system *s, const double *B, double *X, int nrhs, int ld)
{
    sfc_ctx *ctx = s->ctx;
    build_operator(s);
    if (!s->any_constraint) {
        solve_block(s, B, X, nrhs, ld);
        return;
    }
    const int64_t N = s->N;
    s->fix.reserve(N * (int64_t)ld);
    k_lift_block<<<grid_for(N * nrhs, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_ref.p,
                                                                   s->mask.p, B, ld, nrhs, N, s->fix.p);
    count_launch(ctx);
    solve_block(s, s->fix.p, X, nrhs, ld);
}

void transpose_fixup(sfc_system *s, const double *B, double *X, int nrhs, int ld)
{
    if (!s->any_constraint) return;
    sfc_ctx *ctx = s->ctx;
    const int64_t N = s->N;
    if (s->pattern_mesh) {  // element couplings: the pattern is symmetric
        k_fix_gather<<<grid_for(N * 32, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_ref.p,
                                                                      s->mask.p, B, ld, nrhs, N, X);
        count_launch(ctx);
        return;
    }
    s->fix.reserve(N * (int64_t)nrhs);
    SFC_CK(cudaMemsetAsync(s->fix.p, 0, N * (int64_t)nrhs * 8, ctx->stream));
    k_fix_accum<<<grid_for(N * nrhs, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->a_ref.p, s->mask.p, X,
                                                                   ld, nrhs, N, s->fix.p);
    k_fix_apply<<<grid_for(N * nrhs, 256), 256, 0, ctx->stream>>>(s->diag.p, s->a_ref.p, s->mask.p, B, s->fix.p, ld,
                                                                  nrhs, N, X);
    count_launch(ctx, 2);
}

}  // namespace sfc
