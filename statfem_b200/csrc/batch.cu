// Batched statFEM posterior for many independent 2-D Poisson instances of
// uneven size (MCMC proposals): one persistent kernel, launched as a CUDA
// graph, solves every instance's adjoint system and evaluates its marginal
// log-likelihood and sensor-space posterior.
//
// Reference path per instance (what one cluster computes):
//   ForwardGaussRHS::updateSolution   statX/infer/ForwardGaussRHS.hpp:95-139
//     R = rows of A^-T P^T (ns solves), mean = R F, C_s = R C_f R^T
//     + (sigma_f reg)^2 P P^T
//   CovarianceForcing::giveProjectedCovar  statX/infer/CovarianceForcing.ipp:38-109
//     (C_f)_ij = phibar_i k(x_i, x_j) phibar_j, k squared-exponential
//   LikelihoodKOH::giveLogLikelihood  statX/infer/LikelihoodKOH.ipp:75-120
//   LikelihoodKOH::giveProjFEconditionedData  statX/infer/LikelihoodKOH.ipp:311-361
//
// Layout: the instances are the disjoint blocks of one union mesh, so one
// CSR (block diagonal) and one assembly serve the whole batch.  Instance i
// owns dofs [row0[i], row0[i+1]), an (s_i+1)^2 tensor grid of the unit
// square (x fastest), homogeneous Dirichlet on its boundary.  The ns <= 32
// adjoint right-hand sides of an instance are the columns of an interleaved
// [dof][32] block (one lane per column).
//
// Work distribution: the grid is a set of thread-block clusters; a cluster
// takes the next instance from an atomic queue (instances ordered by
// decreasing cost) and its CTAs split the instance's rows.  Column
// reductions go through distributed shared memory and cluster barriers, the
// only waits in the kernel (hardware barriers among co-scheduled CTAs).
//
// Solve: FP32 block Jacobi-PCG inner iterations; at the start of each cycle
// the FP64 residual b - S x64 replaces the recurrence residual (reliable
// update: the search direction is kept unless the recurrence drifted);
// converged columns are frozen; the instance stops when every column meets
// the true relative residual tol.  With homogeneous constraints the
// constrained rows of S are diagonal and phibar and F vanish there, so the
// transposed-constraint terms of the reference's A^T solve do not reach
// any output.
//
// Covariance: k is separable on the grid, K = Ky (x) Kx with Toeplitz
// factors k1d[|a - a'|], so Z = K W (W = diag(phibar) R^T) costs two passes
// of O((s+1)^3 ns) and C_s = sigma^2 W^T Z.
// Workspace per dof: R^T (then Z) and W, T in FP64 [dof][32] (W holds the
// dense right-hand sides during the solve); the FP32 solver vectors x, r,
// p, q [dof][32].

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <new>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace sfc {
namespace {

constexpr int BK = 32;        // columns (sensors) per instance
constexpr int BT = 256;       // threads per CTA
constexpr int BW = BT / 32;   // warps per CTA
constexpr int kDense = 3 * BK * BK;  // doubles of the dense sensor-space stage

struct BatchArgs {
    // union operator
    const int32_t *rp, *col;
    const double *a64;
    const float *a32, *dinv32;
    const double *phibar, *F;
    // instances
    int n_inst;
    const int64_t *row0;     // n_inst + 1
    const int32_t *side;     // s
    const int32_t *order;    // processing order
    const int32_t *ns;       // sensors per instance
    const int32_t *sdof;     // n_inst x 32 x 3 global dofs (-1: none)
    const double *sw;        // n_inst x 32 x 3 weights
    const double *scoord;    // n_inst x 32 x 2
    const double *y;         // n_inst x 32 x n_o
    int n_o;
    const double *hp;        // n_inst x 6: sigma_f, length_f, rho, sigma_d, length_d, eps
    double reg;
    // workspace
    double *x64, *W, *T;
    float *x32, *r32, *p32, *q32;
    int *queue;
    int k1d_len;
    // controls
    double tol, itol;
    int max_iter, max_cycles;
    // outputs
    double *loglik, *mean_s, *cov_s, *pmean, *pcov;
    int *status, *iters;
};

struct Smem {
    double *sred;   // [3][64] reduction slots, read by the other CTAs of the cluster
    double *sres;   // [64]
    double *swp;    // [BW][64]
    double *scs;    // [32*32] C_s partial, read by CTA 0
    double *sub;    // [32] prior mean at the sensors
    double *k1d;    // [k1d_len]
    double *dense;  // [3*32*32] dense stage / [2*32*32] row tiles
    int *sinst;
};

// Column sums over the whole cluster of per-lane values v0, v1 (lane c holds
// column c's partial): results in s.sres[c] and s.sres[32 + c] of every CTA,
// summed in the same order everywhere.  Global-memory writes made before the
// call are visible to the whole cluster after it.
__device__ void cluster_sum2(cg::cluster_group &cl, const Smem &s, int &slot, double v0, double v1)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *red = s.sred + 64 * slot;
    slot = slot == 2 ? 0 : slot + 1;
    s.swp[warp * 64 + lane] = v0;
    s.swp[warp * 64 + 32 + lane] = v1;
    __syncthreads();
    if (threadIdx.x < 64) {
        double t = 0.0;
        for (int w = 0; w < BW; ++w) t += s.swp[w * 64 + threadIdx.x];
        red[threadIdx.x] = t;
    }
    __threadfence();
    cl.sync();
    if (threadIdx.x < 64) {
        double t = 0.0;
        const unsigned cs = cl.num_blocks();
        for (unsigned r = 0; r < cs; ++r) t += cl.map_shared_rank(red, r)[threadIdx.x];
        s.sres[threadIdx.x] = t;
    }
    __syncthreads();
}

// The same for the quad layout: lane (g, fl) holds partials of columns
// 4 fl .. 4 fl + 3 for its rows; the 4 row groups are combined first.
__device__ void cluster_sum_q(cg::cluster_group &cl, const Smem &s, int &slot, const double (&v0)[4],
                              const double (&v1)[4])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, fl = lane & 7;
    double *red = s.sred + 64 * slot;
    slot = slot == 2 ? 0 : slot + 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double a = v0[q], b = v1[q];
        a += __shfl_xor_sync(0xffffffffu, a, 8);
        a += __shfl_xor_sync(0xffffffffu, a, 16);
        b += __shfl_xor_sync(0xffffffffu, b, 8);
        b += __shfl_xor_sync(0xffffffffu, b, 16);
        if (lane < 8) {
            s.swp[warp * 64 + 4 * fl + q] = a;
            s.swp[warp * 64 + 32 + 4 * fl + q] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x < 64) {
        double t = 0.0;
        for (int w = 0; w < BW; ++w) t += s.swp[w * 64 + threadIdx.x];
        red[threadIdx.x] = t;
    }
    __threadfence();
    cl.sync();
    if (threadIdx.x < 64) {
        double t = 0.0;
        const unsigned cs = cl.num_blocks();
        for (unsigned r = 0; r < cs; ++r) t += cl.map_shared_rank(red, r)[threadIdx.x];
        s.sres[threadIdx.x] = t;
    }
    __syncthreads();
}

__device__ __forceinline__ void cluster_barrier(cg::cluster_group &cl)
{
    __threadfence();
    cl.sync();
}

// lower Cholesky of the n x n matrix A (row-major, stride 32) into L by one
// warp; returns 0 or k+1 when pivot k is not positive
__device__ int warp_chol(const double *A, double *L, int n)
{
    const int lane = threadIdx.x & 31;
    int info = 0;
    for (int j = 0; j < n; ++j) {
        double v = 0.0;
        if (lane >= j && lane < n) {
            v = A[lane * BK + j];
            for (int k = 0; k < j; ++k) v -= L[lane * BK + k] * L[j * BK + k];
        }
        const double d = __shfl_sync(0xffffffffu, v, j);
        if (!(d > 0.0)) {
            info = j + 1;
            break;
        }
        const double sd = sqrt(d);
        if (lane < n) L[lane * BK + j] = lane == j ? sd : (lane > j ? v / sd : 0.0);
        __syncwarp();
    }
    return info;
}

// in place X := L^-1 X for an n x m block X (row-major stride 32), lane = column
__device__ void warp_trsm(const double *L, double *X, int n, int m)
{
    const int lane = threadIdx.x & 31;
    if (lane < m)
        for (int j = 0; j < n; ++j) {
            double v = X[j * BK + lane];
            for (int k = 0; k < j; ++k) v -= L[j * BK + k] * X[k * BK + lane];
            X[j * BK + lane] = v / L[j * BK + j];
        }
    __syncwarp();
}

__global__ void __launch_bounds__(BT, 4) k_batch(BatchArgs a)
{
    cg::cluster_group cl = cg::this_cluster();
    const unsigned CS = cl.num_blocks(), rank = cl.block_rank();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    extern __shared__ __align__(16) double smem[];
    Smem s;
    s.sred = smem;
    s.sres = s.sred + 3 * 64;
    s.swp = s.sres + 64;
    s.scs = s.swp + BW * 64;
    s.sub = s.scs + BK * BK;
    s.k1d = s.sub + BK;
    s.dense = s.k1d + a.k1d_len;
    s.sinst = reinterpret_cast<int *>(s.dense + kDense);
    int slot = 0;

    for (;;) {
        if (rank == 0 && threadIdx.x == 0) *s.sinst = atomicAdd(a.queue, 1);
        cl.sync();
        const int qi = *cl.map_shared_rank(s.sinst, 0);
        cl.sync();  // every CTA has read the id before CTA 0 takes the next
        if (qi >= a.n_inst) break;
        const int inst = a.order[qi];
        const int64_t r0 = a.row0[inst];
        const int n = (int)(a.row0[inst + 1] - r0);
        const int side = a.side[inst];
        const int nsens = a.ns[inst];
        const int chunk = (n + (int)CS - 1) / (int)CS;
        const int64_t my0 = r0 + min(n, (int)rank * chunk), my1 = r0 + min(n, ((int)rank + 1) * chunk);
        int status = 0, total_it = 0;

        // ---------------- solve: FP64 refinement around FP32 block PCG ----------------
        // Quad layout: a warp works on 4 rows at once, 8 lanes per row, each
        // lane on 4 adjacent columns (16-byte vectors): four rows' loads are
        // in flight per instruction.  Lane (g, fl): row i0 + g, columns 4 fl .. 4 fl + 3.
        const int g = lane >> 3, fl = lane & 7;
        float4 *X4 = reinterpret_cast<float4 *>(a.x32), *R4 = reinterpret_cast<float4 *>(a.r32);
        float4 *P4 = reinterpret_cast<float4 *>(a.p32), *Q4 = reinterpret_cast<float4 *>(a.q32);
        // right-hand sides b = P^T, dense in W (W is free until the statistics)
        for (int64_t i = my0 + warp; i < my1; i += BW) {
            a.x64[i * BK + lane] = 0.0;
            a.W[i * BK + lane] = 0.0;
        }
        cluster_barrier(cl);
        if (rank == 0 && warp == 0 && lane < nsens)
            for (int k = 0; k < 3; ++k) {
                const int d = a.sdof[((int64_t)inst * BK + lane) * 3 + k];
                if (d >= r0 && d < r0 + n) a.W[(int64_t)d * BK + lane] += a.sw[((int64_t)inst * BK + lane) * 3 + k];
            }
        cluster_barrier(cl);
        // per column, across cycles: r.z the current direction was built
        // from, and the recurrence residual norm^2 when the column stopped
        double rzd[4] = {0, 0, 0, 0}, rrl[4] = {0, 0, 0, 0};
        for (int cycle = 0;; ++cycle) {
            double prr[4] = {0, 0, 0, 0}, pbb[4] = {0, 0, 0, 0};
            for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                const int64_t i = i0 + g;
                if (i >= my1) continue;
                const double2 *b2 = reinterpret_cast<const double2 *>(a.W + i * BK + 4 * fl);
                const double2 b01 = b2[0], b23 = b2[1];
                double r[4] = {b01.x, b01.y, b23.x, b23.y};
                const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
                if (cycle > 0)
                    for (int32_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
                        const double av = a.a64[k];
                        const double2 *x2 = reinterpret_cast<const double2 *>(a.x64 + (int64_t)a.col[k] * BK + 4 * fl);
                        const double2 x01 = x2[0], x23 = x2[1];
                        r[0] -= av * x01.x;
                        r[1] -= av * x01.y;
                        r[2] -= av * x23.x;
                        r[3] -= av * x23.y;
                    }
                R4[i * 8 + fl] = make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]);
                X4[i * 8 + fl] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    prr[q] += r[q] * r[q];
                    pbb[q] += bv[q] * bv[q];
                }
            }
            cluster_sum_q(cl, s, slot, prr, pbb);
            double rr0[4], bb[4];
            bool done[4], bad = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                rr0[q] = s.sres[4 * fl + q];
                bb[q] = s.sres[32 + 4 * fl + q];
                bad = bad || !(rr0[q] == rr0[q]) || !(bb[q] == bb[q]);
                done[q] = bb[q] == 0.0 || rr0[q] <= a.tol * a.tol * bb[q];
            }
            if (__any_sync(0xffffffffu, bad)) {
                status = SFC_ERR_NOT_SPD;
                break;
            }
            if (__all_sync(0xffffffffu, done[0] && done[1] && done[2] && done[3])) break;
            if (cycle >= a.max_cycles || total_it >= a.max_iter) {
                status = SFC_ERR_NOT_CONVERGED;
                break;
            }
            // inner FP32 PCG on S d = r for the open columns
            bool act[4];
            double thr[4], rz[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                act[q] = !done[q];
                thr[q] = a.itol * a.itol * rr0[q];
            }
            {
                // reliable update: the FP64 residual replaces the recurrence
                // one and the search direction is kept, p = z + (r.z / rzd) p,
                // unless the recurrence had drifted from the true residual by
                // more than a factor 1.5 (then, and in the first cycle, p = z)
                double prz[4] = {0, 0, 0, 0}, zero[4] = {0, 0, 0, 0};
                for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                    const int64_t i = i0 + g;
                    if (i >= my1) continue;
                    const float4 r = R4[i * 8 + fl];
                    const float d = a.dinv32[i];
                    prz[0] += (double)r.x * (d * r.x);
                    prz[1] += (double)r.y * (d * r.y);
                    prz[2] += (double)r.z * (d * r.z);
                    prz[3] += (double)r.w * (d * r.w);
                }
                cluster_sum_q(cl, s, slot, prz, zero);
                bool cont[4];
                float b0[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    rz[q] = s.sres[4 * fl + q];
                    cont[q] = cycle > 0 && act[q] && rzd[q] > 0.0 && rr0[q] <= 2.25 * rrl[q] &&
                              rr0[q] * 2.25 >= rrl[q];
                    b0[q] = cont[q] ? (float)(rz[q] / rzd[q]) : 0.f;
                }
                for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                    const int64_t i = i0 + g;
                    if (i >= my1) continue;
                    const float4 r = R4[i * 8 + fl];
                    const float d = a.dinv32[i];
                    float4 pv = make_float4(d * r.x, d * r.y, d * r.z, d * r.w);
                    if (cont[0] || cont[1] || cont[2] || cont[3]) {  // P holds a previous direction
                        const float4 po = P4[i * 8 + fl];
                        if (cont[0]) pv.x = fmaf(b0[0], po.x, pv.x);
                        if (cont[1]) pv.y = fmaf(b0[1], po.y, pv.y);
                        if (cont[2]) pv.z = fmaf(b0[2], po.z, pv.z);
                        if (cont[3]) pv.w = fmaf(b0[3], po.w, pv.w);
                    }
                    P4[i * 8 + fl] = pv;
                }
                cluster_barrier(cl);
            }
            bool inner_bad = false;
            for (; total_it < a.max_iter; ++total_it) {
                double ppq[4] = {0, 0, 0, 0}, zero[4] = {0, 0, 0, 0};
                for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                    const int64_t i = i0 + g;
                    if (i >= my1) continue;
                    const int32_t kb = a.rp[i], ke = a.rp[i + 1];
                    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (int32_t k = kb; k < ke; k += 4) {
                        // four independent neighbour loads (padding: weight 0 on the last entry)
                        const int32_t k1 = min(k + 1, ke - 1), k2 = min(k + 2, ke - 1), k3 = min(k + 3, ke - 1);
                        const float a0 = a.a32[k], a1 = k + 1 < ke ? a.a32[k1] : 0.f,
                                    a2 = k + 2 < ke ? a.a32[k2] : 0.f, a3 = k + 3 < ke ? a.a32[k3] : 0.f;
                        const float4 p0 = P4[(int64_t)a.col[k] * 8 + fl], p1 = P4[(int64_t)a.col[k1] * 8 + fl],
                                     p2 = P4[(int64_t)a.col[k2] * 8 + fl], p3 = P4[(int64_t)a.col[k3] * 8 + fl];
                        acc.x = fmaf(a0, p0.x, fmaf(a1, p1.x, fmaf(a2, p2.x, fmaf(a3, p3.x, acc.x))));
                        acc.y = fmaf(a0, p0.y, fmaf(a1, p1.y, fmaf(a2, p2.y, fmaf(a3, p3.y, acc.y))));
                        acc.z = fmaf(a0, p0.z, fmaf(a1, p1.z, fmaf(a2, p2.z, fmaf(a3, p3.z, acc.z))));
                        acc.w = fmaf(a0, p0.w, fmaf(a1, p1.w, fmaf(a2, p2.w, fmaf(a3, p3.w, acc.w))));
                    }
                    Q4[i * 8 + fl] = acc;
                    const float4 pi = P4[i * 8 + fl];
                    ppq[0] += (double)pi.x * acc.x;
                    ppq[1] += (double)pi.y * acc.y;
                    ppq[2] += (double)pi.z * acc.z;
                    ppq[3] += (double)pi.w * acc.w;
                }
                cluster_sum_q(cl, s, slot, ppq, zero);
                float alpha[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double pq = s.sres[4 * fl + q];
                    if (act[q] && !(pq > 0.0)) {
                        act[q] = false;
                        inner_bad = true;
                    }
                    alpha[q] = act[q] ? (float)(rz[q] / pq) : 0.f;
                }
                double prz2[4] = {0, 0, 0, 0}, prr2[4] = {0, 0, 0, 0};
                for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                    const int64_t i = i0 + g;
                    if (i >= my1) continue;
                    const int64_t o = i * 8 + fl;
                    const float4 pv = P4[o], qv = Q4[o];
                    float4 xv = X4[o], rv = R4[o];
                    const float d = a.dinv32[i];
                    xv.x = fmaf(alpha[0], pv.x, xv.x);
                    xv.y = fmaf(alpha[1], pv.y, xv.y);
                    xv.z = fmaf(alpha[2], pv.z, xv.z);
                    xv.w = fmaf(alpha[3], pv.w, xv.w);
                    rv.x = fmaf(-alpha[0], qv.x, rv.x);
                    rv.y = fmaf(-alpha[1], qv.y, rv.y);
                    rv.z = fmaf(-alpha[2], qv.z, rv.z);
                    rv.w = fmaf(-alpha[3], qv.w, rv.w);
                    X4[o] = xv;
                    R4[o] = rv;
                    prz2[0] += (double)rv.x * (d * rv.x);
                    prz2[1] += (double)rv.y * (d * rv.y);
                    prz2[2] += (double)rv.z * (d * rv.z);
                    prz2[3] += (double)rv.w * (d * rv.w);
                    prr2[0] += (double)rv.x * rv.x;
                    prr2[1] += (double)rv.y * rv.y;
                    prr2[2] += (double)rv.z * rv.z;
                    prr2[3] += (double)rv.w * rv.w;
                }
                cluster_sum_q(cl, s, slot, prz2, prr2);
                float beta[4];
                bool any = false;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double rzn = s.sres[4 * fl + q], rrn = s.sres[32 + 4 * fl + q];
                    if (!(rrn == rrn)) {
                        act[q] = false;
                        inner_bad = true;
                    }
                    const bool was = act[q];
                    act[q] = act[q] && rrn > thr[q];
                    if (was && !act[q]) {  // stops here: keep its direction for the next cycle
                        rzd[q] = rz[q];
                        rrl[q] = rrn;
                    }
                    beta[q] = act[q] ? (float)(rzn / rz[q]) : 0.f;
                    if (act[q]) rz[q] = rzn;
                    any = any || act[q];
                }
                if (!__any_sync(0xffffffffu, any)) {
                    ++total_it;
                    break;
                }
                for (int64_t i0 = my0 + 4 * warp; i0 < my1; i0 += 4 * BW) {
                    const int64_t i = i0 + g;
                    if (i >= my1) continue;
                    const int64_t o = i * 8 + fl;
                    const float4 rv = R4[o];
                    float4 pv = P4[o];
                    const float d = a.dinv32[i];
                    // stopped columns keep their direction
                    if (act[0]) pv.x = fmaf(beta[0], pv.x, d * rv.x);
                    if (act[1]) pv.y = fmaf(beta[1], pv.y, d * rv.y);
                    if (act[2]) pv.z = fmaf(beta[2], pv.z, d * rv.z);
                    if (act[3]) pv.w = fmaf(beta[3], pv.w, d * rv.w);
                    P4[o] = pv;
                }
                cluster_barrier(cl);
            }
            status = __any_sync(0xffffffffu, inner_bad) ? SFC_ERR_NOT_SPD : 0;
            for (int64_t i = my0 + warp; i < my1; i += BW) a.x64[i * BK + lane] += (double)a.x32[i * BK + lane];
            cluster_barrier(cl);
            if (status) break;
        }

        // ---------------- sensor-space statistics ----------------
        const double *h = a.hp + (int64_t)inst * 6;
        const double sf = h[0], lf = h[1], rho = h[2], sdm = h[3], ldm = h[4], eps = h[5];
        const int m = side + 1;
        // W = phibar * R^T, prior mean at the sensors R F
        double pu = 0.0;
        for (int64_t i = my0 + warp; i < my1; i += BW) {
            const double x = a.x64[i * BK + lane];
            a.W[i * BK + lane] = a.phibar[i] * x;
            pu += x * a.F[i];
        }
        // Toeplitz factor of the separable kernel on the grid
        for (int t = threadIdx.x; t < m; t += BT) {
            const double d = (double)t / (double)side;
            s.k1d[t] = exp(-d * d / (2.0 * lf * lf));
        }
        cluster_sum2(cl, s, slot, pu, 0.0);  // also publishes W to the cluster
        if (threadIdx.x < 32) s.sub[threadIdx.x] = s.sres[threadIdx.x];
        // x pass: T[a][b] = sum_b' k1d[|b - b'|] W[a][b']
        for (int64_t i = my0 + warp; i < my1; i += BW) {
            const int ra = (int)((i - r0) / m), b = (int)((i - r0) % m);
            const double *wl = a.W + (r0 + (int64_t)ra * m) * BK + lane;
            double acc = 0.0;
            for (int b2 = 0; b2 < m; ++b2) acc += s.k1d[abs(b - b2)] * wl[(int64_t)b2 * BK];
            a.T[i * BK + lane] = acc;
        }
        cluster_barrier(cl);
        // y pass: Z[a][b] = sum_a' k1d[|a - a'|] T[a'][b], into x64 (R^T is no longer needed)
        for (int64_t i = my0 + warp; i < my1; i += BW) {
            const int ra = (int)((i - r0) / m), b = (int)((i - r0) % m);
            const double *tl = a.T + (r0 + b) * BK + lane;
            double acc = 0.0;
            for (int a2 = 0; a2 < m; ++a2) acc += s.k1d[abs(ra - a2)] * tl[(int64_t)a2 * m * BK];
            a.x64[i * BK + lane] = acc;
        }
        __syncthreads();
        // C_s partial = W^T Z over this CTA's rows, 32-row tiles
        {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            double *tw = s.dense, *tz = s.dense + BK * BK;
            for (int64_t t0 = my0; t0 < my1; t0 += BK) {
                for (int t = threadIdx.x; t < BK * BK; t += BT) {
                    const int64_t i = t0 + t / BK;
                    const bool ok = i < my1;
                    tw[t] = ok ? a.W[i * BK + (t % BK)] : 0.0;
                    tz[t] = ok ? a.x64[i * BK + (t % BK)] : 0.0;
                }
                __syncthreads();
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int o = threadIdx.x + k * BT, c = o / BK, d = o % BK;
                    double v = acc[k];
                    for (int rrow = 0; rrow < BK; ++rrow) v += tw[rrow * BK + c] * tz[rrow * BK + d];
                    acc[k] = v;
                }
                __syncthreads();
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) s.scs[threadIdx.x + k * BT] = acc[k];
        }
        cluster_barrier(cl);
        // dense stage on CTA 0
        if (rank == 0) {
            // C_s overwrites this CTA's own partial element by element (each
            // element is read and written by the same thread; only CTA 0 reads
            // the partials)
            double *Cs = s.scs, *Ks = s.dense, *L = Ks + BK * BK, *V = L + BK * BK, *L2 = L;
            const int ns = nsens;
            const int *sdi = a.sdof + (int64_t)inst * BK * 3;
            const double *swi = a.sw + (int64_t)inst * BK * 3;
            const double reg2 = (sf * a.reg) * (sf * a.reg);
            for (int t = threadIdx.x; t < BK * BK; t += BT) {
                double v = 0.0;
                for (unsigned r = 0; r < CS; ++r) v += cl.map_shared_rank(s.scs, r)[t];  // rank order
                const int c = t / BK, d = t % BK;
                v *= sf * sf;
                if (c < ns && d < ns) {
                    double pp = 0.0;
                    for (int k = 0; k < 3; ++k)
                        for (int l = 0; l < 3; ++l)
                            if (sdi[c * 3 + k] >= 0 && sdi[c * 3 + k] == sdi[d * 3 + l])
                                pp += swi[c * 3 + k] * swi[d * 3 + l];
                    v += reg2 * pp;
                } else {
                    v = 0.0;
                }
                Cs[t] = v;
                const double *xc = a.scoord + ((int64_t)inst * BK + c) * 2, *xd = a.scoord + ((int64_t)inst * BK + d) * 2;
                const double dx = xc[0] - xd[0], dy = xc[1] - xd[1];
                Ks[t] = (c < ns && d < ns) ? sdm * sdm * exp(-(dx * dx + dy * dy) / (2.0 * ldm * ldm)) +
                                                 (c == d ? eps * eps : 0.0)
                                           : 0.0;
            }
            __syncthreads();
            for (int t = threadIdx.x; t < BK * BK; t += BT) {
                a.cov_s[(int64_t)inst * BK * BK + t] = Cs[t];
                V[t] = Ks[t] + rho * rho * Cs[t];  // total covariance C = K_s + rho^2 C_s
            }
            if (threadIdx.x < BK) a.mean_s[(int64_t)inst * BK + threadIdx.x] = threadIdx.x < ns ? s.sub[threadIdx.x] : 0.0;
            __syncthreads();
            if (warp == 0) {
                int info = warp_chol(V, L, ns);
                double ll = 0.0;
                if (info == 0) {
                    // log p = n_o (-ns/2 log 2 pi - sum log L_ii) - 1/2 sum_k |L^-1 (y_k - rho mean)|^2
                    double ld = 0.0;
                    for (int j = 0; j < ns; ++j) ld += log(L[j * BK + j]);
                    double quad = 0.0;
                    for (int k = 0; k < a.n_o; ++k) {
                        double v = 0.0;  // lane j holds component j of L^-1 d_k
                        for (int j = 0; j < ns; ++j) {
                            double t = a.y[((int64_t)inst * BK + j) * a.n_o + k] - rho * s.sub[j];
                            for (int q = 0; q < j; ++q) t -= L[j * BK + q] * __shfl_sync(0xffffffffu, v, q);
                            t /= L[j * BK + j];
                            if (lane == j) v = t;
                        }
                        double sq = lane < ns ? v * v : 0.0;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
                        quad += sq;
                    }
                    ll = a.n_o * (-0.5 * ns * log(2.0 * 3.14159265358979323846) - ld) - 0.5 * quad;
                }
                // posterior at the sensors: G = C_s + K_s / (rho^2 n_o),
                // mean = mu + C_s G^-1 (ybar / rho - mu), cov = C_s - C_s G^-1 C_s
                int info2 = 0;
                if (info == 0) {
                    const double f = 1.0 / (rho * rho * a.n_o);
                    for (int c = 0; c < ns; ++c)
                        if (lane < ns) V[c * BK + lane] = Cs[c * BK + lane] + f * Ks[c * BK + lane];
                    __syncwarp();
                    info2 = warp_chol(V, L2, ns);
                }
                if (info == 0 && info2 == 0) {
                    for (int c = 0; c < ns; ++c)
                        if (lane < ns) V[c * BK + lane] = Cs[c * BK + lane];
                    __syncwarp();
                    warp_trsm(L2, V, ns, ns);  // V = L2^-1 C_s
                    // w = L2^-1 (ybar / rho - mu), lane j holds w_j
                    double w = 0.0;
                    for (int j = 0; j < ns; ++j) {
                        double yb = 0.0;
                        for (int k = 0; k < a.n_o; ++k) yb += a.y[((int64_t)inst * BK + j) * a.n_o + k];
                        double t = yb / (a.n_o * rho) - s.sub[j];
                        for (int q = 0; q < j; ++q) t -= L2[j * BK + q] * __shfl_sync(0xffffffffu, w, q);
                        t /= L2[j * BK + j];
                        if (lane == j) w = t;
                    }
                    double pm = 0.0;
                    for (int j = 0; j < ns; ++j) pm += V[j * BK + lane] * __shfl_sync(0xffffffffu, w, j);
                    if (lane < BK) a.pmean[(int64_t)inst * BK + lane] = lane < ns ? s.sub[lane] + pm : 0.0;
                    for (int c = 0; c < BK; ++c) {
                        double v = 0.0;
                        if (c < ns && lane < ns) {
                            v = Cs[c * BK + lane];
                            for (int j = 0; j < ns; ++j) v -= V[j * BK + c] * V[j * BK + lane];
                        }
                        a.pcov[((int64_t)inst * BK + c) * BK + lane] = v;
                    }
                }
                if (lane == 0) {
                    a.loglik[inst] = info == 0 ? ll : NAN;
                    int st = status;
                    if (!st && (info || info2)) st = SFC_ERR_NOT_SPD;
                    a.status[inst] = st;
                    a.iters[inst] = total_it;
                }
            }
        }
        cluster_barrier(cl);  // CTA 0's shared memory stays live until the others are done reading
    }
}

}  // namespace
}  // namespace sfc

struct sfc_batch {
    sfc_ctx *ctx = nullptr;
    const sfc_mesh *mesh = nullptr;
    sfc_system *sys = nullptr;
    int n = 0, n_o = 1, smax = 0;
    double f = 1.0, reg = 1e-3;
    int64_t nbc = 0;
    sfc::DBuf<int64_t> row0;
    sfc::DBuf<int32_t> side, order, ns, sdof, status, iters, queue;
    sfc::DBuf<double> sw, scoord, y, hp, phibar, x64, W, T, loglik, mean_s, cov_s, pmean, pcov, bc_zero;
    sfc::DBuf<float> x32, r32, p32, q32;
    sfc::DBuf<uint32_t> bc_idx;
    bool have_y = false, have_hp = false;
    // launch
    int cluster = 0, grid = 0;
    size_t smem = 0;
    sfc::BatchArgs args{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    double tol = 1e-8, itol = 1e-2;
    int max_iter = 50000, max_cycles = 200;
    ~sfc_batch()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        delete sys;
    }
};

namespace sfc {

namespace {

void batch_release_graph(sfc_batch *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

size_t batch_smem(int smax)
{
    const int k1d = ((smax + 1) + 1) & ~1;
    return sizeof(double) * (3 * 64 + 64 + BW * 64 + BK * BK + BK + k1d + kDense) + 16;
}

// cluster size and persistent grid: the largest cluster size (of those
// tried, in preference order) that the device can co-schedule
void batch_configure(sfc_batch *b, int want_cluster)
{
    const size_t smem = batch_smem(b->smax);
    SFC_CK(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SFC_CK(cudaFuncSetAttribute(k_batch, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    const int tries[] = {want_cluster, 8, 4, 2, 1};
    for (int cs : tries) {
        if (cs < 1 || cs > 16) continue;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(cs, 1, 1);
        cfg.blockDim = dim3(BT, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, k_batch, &cfg);
        if (e != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (nclusters > 0) {
            b->cluster = cs;
            b->grid = cs * std::min(nclusters, std::max(1, b->n));
            b->smem = smem;
            return;
        }
    }
    fail(SFC_ERR_TOO_LARGE, "no cluster shape of the batch kernel fits on this device");
}

void batch_launch(sfc_batch *b, cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = b->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(b->grid, 1, 1);
    cfg.blockDim = dim3(BT, 1, 1);
    cfg.dynamicSmemBytes = b->smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SFC_CK(cudaLaunchKernelEx(&cfg, k_batch, b->args));
}

__global__ void k_zero_at(double *v, const uint32_t *idx, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        v[idx[t]] = 0.0;
}

// assembly of the union system (not captured: it reads status words)
void batch_assemble(sfc_batch *b)
{
    sfc_ctx *ctx = b->ctx;
    sfc_system *s = b->sys;
    assemble_matrix(s, b->mesh);
    const int64_t N = s->N;
    s->F.alloc(N);
    assemble_load(ctx, b->mesh, &b->f, s->F.p, true);
    const double one = 1.0;
    assemble_load(ctx, b->mesh, &one, b->phibar.p, true);
    k_zero_at<<<grid_for(b->nbc, 256), 256, 0, ctx->stream>>>(b->phibar.p, b->bc_idx.p, b->nbc);
    count_launch(ctx);
    apply_constraints_dev(s, b->bc_idx.p, b->bc_zero.p, b->nbc, 1.0, 1.0);
    build_operator(s, false);  // a bad instance fails alone, in the kernel
}

void batch_build_args(sfc_batch *b)
{
    sfc_system *s = b->sys;
    BatchArgs &a = b->args;
    a = {};
    a.rp = s->row_ptr.p;
    a.col = s->col.p;
    a.a64 = s->a_op.p;
    a.a32 = s->a_op32.p;
    a.dinv32 = s->dinv32.p;
    a.phibar = b->phibar.p;
    a.F = s->F.p;
    a.n_inst = b->n;
    a.row0 = b->row0.p;
    a.side = b->side.p;
    a.order = b->order.p;
    a.ns = b->ns.p;
    a.sdof = b->sdof.p;
    a.sw = b->sw.p;
    a.scoord = b->scoord.p;
    a.y = b->y.p;
    a.n_o = b->n_o;
    a.hp = b->hp.p;
    a.reg = b->reg;
    a.x64 = b->x64.p;
    a.W = b->W.p;
    a.T = b->T.p;
    a.x32 = b->x32.p;
    a.r32 = b->r32.p;
    a.p32 = b->p32.p;
    a.q32 = b->q32.p;
    a.queue = b->queue.p;
    a.k1d_len = ((b->smax + 1) + 1) & ~1;
    a.tol = b->tol;
    a.itol = b->itol;
    a.max_iter = b->max_iter;
    a.max_cycles = b->max_cycles;
    a.loglik = b->loglik.p;
    a.mean_s = b->mean_s.p;
    a.cov_s = b->cov_s.p;
    a.pmean = b->pmean.p;
    a.pcov = b->pcov.p;
    a.status = b->status.p;
    a.iters = b->iters.p;
}

// the captured step: reset the queue, run the persistent kernel
void batch_capture(sfc_batch *b)
{
    batch_release_graph(b);
    batch_build_args(b);
    cudaStream_t st;
    SFC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaMemsetAsync(b->queue.p, 0, sizeof(int), st);
        try {
            batch_launch(b, st);
        } catch (const Error &) {
            cudaGraph_t g;
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(st);
            throw;
        }
        e = cudaStreamEndCapture(st, &b->graph);
    }
    cudaStreamDestroy(st);
    SFC_CK(e);
    SFC_CK(cudaGraphInstantiate(&b->gexec, b->graph, 0));
}

}  // namespace

void batch_run(sfc_batch *b)
{
    sfc_ctx *ctx = b->ctx;
    SFC_REQUIRE(b->have_y && b->have_hp, "set readings and hyperparameters before running the batch");
    {
        ProfScope ps(ctx, "phase:batch_assembly", 0.0);
        batch_assemble(b);
    }
    if (!b->gexec) batch_capture(b);
    ProfScope ps(ctx, "phase:batch_solve_likelihood", 0.0);
    SFC_CK(cudaGraphLaunch(b->gexec, ctx->stream));
    count_launch(ctx);
    ++ctx->graph_replays;
}

}  // namespace sfc

using namespace sfc;

namespace sfc {
namespace {
int bguard(sfc_ctx *ctx, const std::function<void()> &fn)
{
    try {
        SFC_CK(cudaSetDevice(ctx->device));
        fn();
        return SFC_OK;
    } catch (const Error &e) {
        ctx->err = e.msg;
        if (e.code == SFC_ERR_CUDA) cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->err = "host allocation failed";
        return SFC_ERR_NO_MEMORY;
    }
}
}  // namespace
}  // namespace sfc

extern "C" {

int32_t sfc_batch_create(sfc_ctx_t *ctx, const sfc_mesh_t *mesh, int32_t num_instances, const int64_t *dof_offset,
                         const int32_t *grid_side, const uint32_t *bc_dofs, int64_t num_bc,
                         const int32_t *num_sensors, const int32_t *sensor_dofs, const double *sensor_weights,
                         const double *sensor_coords, double forcing_mean, int32_t cluster_size, sfc_batch_t **out)
{
    if (!ctx || !mesh || num_instances <= 0 || !dof_offset || !grid_side || (num_bc > 0 && !bc_dofs) || num_bc < 0 ||
        !num_sensors || !sensor_dofs || !sensor_weights || !sensor_coords || !out)
        return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_batch *b = new (std::nothrow) sfc_batch();
    if (!b) return SFC_ERR_NO_MEMORY;
    int rc = bguard(ctx, [&] {
        SFC_REQUIRE(mesh->ctx == ctx, "mesh belongs to another context");
        SFC_REQUIRE(mesh->kind == SFC_ELEM_TRI3_POISSON, "the batch path takes 2-D Poisson triangle meshes");
        const int n = num_instances;
        SFC_REQUIRE(dof_offset[0] == 0 && dof_offset[n] == mesh->num_dofs,
                    "dof_offset must start at 0 and end at the mesh's dof count");
        // every instance is an (s+1)^2 grid of the unit square, x fastest
        int smax = 0;
        for (int i = 0; i < n; ++i) {
            const int s = grid_side[i];
            SFC_REQUIRE(s >= 1 && s <= 4096, "grid side out of range");
            const int64_t m = (int64_t)s + 1;
            SFC_REQUIRE(dof_offset[i + 1] - dof_offset[i] == m * m, "instance dof count is not (side+1)^2");
            for (int64_t k = 0; k < m * m; ++k) {
                const double *x = &mesh->h_coords[(dof_offset[i] + k) * 3];
                const double ex = (double)(k % m) / s, ey = (double)(k / m) / s;
                SFC_REQUIRE(std::fabs(x[0] - ex) < 1e-12 && std::fabs(x[1] - ey) < 1e-12,
                            "instance nodes are not the (side+1)^2 grid of the unit square, x fastest");
            }
            SFC_REQUIRE(num_sensors[i] >= 1 && num_sensors[i] <= BK, "1..32 sensors per instance");
            smax = std::max(smax, s);
        }
        for (int64_t t = 0; t < (int64_t)n * BK * 3; ++t)
            SFC_REQUIRE(sensor_dofs[t] >= -1 && sensor_dofs[t] < mesh->num_dofs, "sensor dof out of range");
        b->ctx = ctx;
        b->mesh = mesh;
        b->n = n;
        b->smax = smax;
        b->f = forcing_mean;
        b->sys = new sfc_system();
        b->sys->ctx = ctx;
        b->sys->N = mesh->num_dofs;
        const int64_t N = mesh->num_dofs;
        upload(ctx, b->row0, dof_offset, n + 1);
        upload(ctx, b->side, grid_side, n);
        upload(ctx, b->ns, num_sensors, n);
        upload(ctx, b->sdof, sensor_dofs, (size_t)n * BK * 3);
        upload(ctx, b->sw, sensor_weights, (size_t)n * BK * 3);
        upload(ctx, b->scoord, sensor_coords, (size_t)n * BK * 2);
        // most expensive first: cost ~ dofs x iterations ~ s^3
        std::vector<int32_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int p, int q) { return grid_side[p] > grid_side[q]; });
        upload(ctx, b->order, ord.data(), n);
        b->nbc = num_bc;
        if (num_bc) {
            upload(ctx, b->bc_idx, bc_dofs, num_bc);
            std::vector<double> z(num_bc, 0.0);
            upload(ctx, b->bc_zero, z.data(), num_bc);
        }
        b->phibar.alloc(N);
        b->x64.alloc(N * BK);
        b->W.alloc(N * BK);
        b->T.alloc(N * BK);
        b->x32.alloc(N * BK);
        b->r32.alloc(N * BK);
        b->p32.alloc(N * BK);
        b->q32.alloc(N * BK);
        b->queue.alloc(1);
        b->loglik.alloc(n);
        b->mean_s.alloc((size_t)n * BK);
        b->cov_s.alloc((size_t)n * BK * BK);
        b->pmean.alloc((size_t)n * BK);
        b->pcov.alloc((size_t)n * BK * BK);
        b->status.alloc(n);
        b->iters.alloc(n);
        b->hp.alloc((size_t)n * 6);
        batch_configure(b, cluster_size > 0 ? cluster_size : 8);
    });
    if (rc != SFC_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return SFC_OK;
}

int32_t sfc_batch_destroy(sfc_batch_t *b)
{
    if (!b) return SFC_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return SFC_OK;
}

int32_t sfc_batch_cluster_size(const sfc_batch_t *b, int32_t *cluster, int32_t *grid)
{
    if (!b) return SFC_ERR_BAD_ARG;
    if (cluster) *cluster = b->cluster;
    if (grid) *grid = b->grid;
    return SFC_OK;
}

int32_t sfc_batch_set_solver(sfc_batch_t *b, double tol, double inner_tol, int32_t max_iter)
{
    if (!b || !(tol > 0) || !(inner_tol > 0 && inner_tol < 1) || max_iter <= 0) return SFC_ERR_BAD_ARG;
    b->tol = tol;
    b->itol = inner_tol;
    b->max_iter = max_iter;
    batch_release_graph(b);
    return SFC_OK;
}

int32_t sfc_batch_set_coefficients(sfc_batch_t *b, const double *elem_coeff)
{
    if (!b) return SFC_ERR_BAD_ARG;
    return sfc_mesh_set_coefficients(const_cast<sfc_mesh_t *>(b->mesh), elem_coeff, 1.0, 0.3);
}

int32_t sfc_batch_set_hparams(sfc_batch_t *b, const sfc_hparams_t *hp, double reg)
{
    if (!b || !hp) return SFC_ERR_BAD_ARG;
    return bguard(b->ctx, [&] {
        std::vector<double> h((size_t)b->n * 6);
        for (int i = 0; i < b->n; ++i) {
            const sfc_hparams_t &p = hp[i];
            SFC_REQUIRE(p.forcing_sigma >= 0 && p.forcing_length > 0 && p.mismatch_length > 0 && p.rho != 0,
                        "invalid hyperparameters");
            h[i * 6 + 0] = p.forcing_sigma;
            h[i * 6 + 1] = p.forcing_length;
            h[i * 6 + 2] = p.rho;
            h[i * 6 + 3] = p.mismatch_sigma;
            h[i * 6 + 4] = p.mismatch_length;
            h[i * 6 + 5] = p.mismatch_sensor_eps;
        }
        upload(b->ctx, b->hp, h.data(), h.size());
        if (b->reg != reg) batch_release_graph(b);
        b->reg = reg;
        b->have_hp = true;
    });
}

int32_t sfc_batch_set_readings(sfc_batch_t *b, const double *y, int32_t num_readings)
{
    if (!b || !y || num_readings < 1 || num_readings > 64) return SFC_ERR_BAD_ARG;
    return bguard(b->ctx, [&] {
        if (num_readings != b->n_o || !b->y.p) batch_release_graph(b);
        b->n_o = num_readings;
        upload(b->ctx, b->y, y, (size_t)b->n * BK * num_readings);
        b->have_y = true;
    });
}

int32_t sfc_batch_run(sfc_batch_t *b)
{
    if (!b) return SFC_ERR_BAD_ARG;
    return bguard(b->ctx, [&] { batch_run(b); });
}

int32_t sfc_batch_autotune(sfc_batch_t *b, int32_t remeasure, int32_t *cluster)
{
    if (!b) return SFC_ERR_BAD_ARG;
    return bguard(b->ctx, [&] {
        SFC_REQUIRE(b->have_y && b->have_hp, "set readings and hyperparameters before tuning the batch");
        int smax_log = 0;
        for (int v = b->smax; v > 1; v >>= 1) ++smax_log;
        int nlog = 0;
        for (int v = b->n; v > 1; v >>= 1) ++nlog;
        const std::string key = "batch:" + tune_device_key(b->ctx) + ":i" + std::to_string(nlog) + ":s" +
                                std::to_string(smax_log);
        std::string v;
        if (!remeasure && tune_lookup(key, v)) {
            batch_release_graph(b);
            batch_configure(b, std::atoi(v.c_str()));
        } else {
            sfc_ctx *ctx = b->ctx;
            batch_assemble(b);
            double best_ms = 1e300;
            int best = b->cluster;
            for (int cs : {1, 2, 4, 8, 16}) {
                batch_release_graph(b);
                batch_configure(b, cs);
                if (b->cluster != cs) continue;  // not co-schedulable on this device
                batch_capture(b);
                SFC_CK(cudaGraphLaunch(b->gexec, ctx->stream));  // warm
                cudaEvent_t e0, e1;
                SFC_CK(cudaEventCreate(&e0));
                SFC_CK(cudaEventCreate(&e1));
                SFC_CK(cudaEventRecord(e0, ctx->stream));
                SFC_CK(cudaGraphLaunch(b->gexec, ctx->stream));
                SFC_CK(cudaEventRecord(e1, ctx->stream));
                SFC_CK(cudaEventSynchronize(e1));
                float ms = 0;
                SFC_CK(cudaEventElapsedTime(&ms, e0, e1));
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                count_launch(ctx, 2);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = cs;
                }
            }
            batch_release_graph(b);
            batch_configure(b, best);
            tune_store(key, std::to_string(best));
        }
        if (cluster) *cluster = b->cluster;
    });
}

int32_t sfc_batch_results(sfc_batch_t *b, double *loglik, double *mean_s, double *cov_s, double *post_mean,
                          double *post_cov, int32_t *status, int32_t *iterations)
{
    if (!b) return SFC_ERR_BAD_ARG;
    return bguard(b->ctx, [&] {
        const size_t n = b->n;
        if (loglik) download(b->ctx, loglik, b->loglik.p, n);
        if (mean_s) download(b->ctx, mean_s, b->mean_s.p, n * BK);
        if (cov_s) download(b->ctx, cov_s, b->cov_s.p, n * BK * BK);
        if (post_mean) download(b->ctx, post_mean, b->pmean.p, n * BK);
        if (post_cov) download(b->ctx, post_cov, b->pcov.p, n * BK * BK);
        if (status) download(b->ctx, status, b->status.p, n);
        if (iterations) download(b->ctx, iterations, b->iters.p, n);
        SFC_CK(cudaStreamSynchronize(b->ctx->stream));
    });
}

}  // extern "C"
