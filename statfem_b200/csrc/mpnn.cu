// Learned preconditioner: a message-passing network on the mesh graph, its
// training on residual/error pairs from plain Jacobi-PCG, and flexible CG.
// (No reference counterpart: the reference solves with Eigen::SparseLU.)
//
// Scaled operator  Ahat = D^-1/2 S D^-1/2  (unit diagonal, FP32 CSR values on
// the matrix pattern; S is the symmetric elimination used by every solver).
// For a residual r:  rhat = D^-1/2 r,  s = rms(rhat),  x0 = rhat / s,
//   H0 = relu(E [x0, Ahat x0] + e)                    encoder, 2 -> 64
//   Hl = relu(Wl [H(l-1) ; Ahat H(l-1)] + bl)         l = 1..3, 128 -> 64
//   y  = w . H3 + c                                   decoder, 64 -> 1
//   M(r) = s D^-1/2 (x0 + y) = D^-1 r + s D^-1/2 y    Jacobi + learned correction
// (y = 0 on constrained dofs, whose rows of S are diagonal: Jacobi is exact).
// The RMS normalisation keeps the node features O(1) whatever the mesh size.
// The aggregation Ahat H is a 64-column SpMM on the operator's pattern.  The
// dense transforms run on the 5th-generation tensor cores (tcgen05.mma,
// BF16 x BF16 -> FP32 in tensor memory): k_layer_tc in inference (gather
// fused), k_dense_fwd_tc and k_dense_bwd_x_tc in training, with the inputs
// rounded to BF16 on the fly, and the weight gradient k_dense_bwd_w_tc as the
// transposed product accumulated over a CTA's node tiles; SFC_MPNN_TC=0
// selects the earlier forms (mma.sync k_layer_inf, k_dense_fwd,
// k_dense_bwd_x, and the FP32 reduction k_dense_bwd_w) for comparison.
// Activations in training, master weights, gradients and Adam state are FP32.
//
// Training pair (r, e) with S e = r: target t = D^1/2 e / s, d = x0 + y - t,
// loss L = d^T Ahat d / N (the S-norm of the error of M(r) scaled by 1/(N s^2)).
// Pairs come from x_k of Jacobi-PCG started at 0: r_k = b - S x_k,
// e_k = x* - x_k, x* the converged solution.

#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <new>
#include <random>
#include <vector>

#include "common.cuh"

namespace {

constexpr int H = 64;                 // hidden width
constexpr int LAYERS = 3;             // message-passing layers
constexpr int OFF_EW = 0;             // encoder weights [64][2]
constexpr int OFF_EB = OFF_EW + 2 * H;
constexpr int OFF_L = OFF_EB + H;     // layer l: W [64][128] then b [64]
constexpr int LSZ = H * 2 * H + H;
constexpr int OFF_DW = OFF_L + LAYERS * LSZ;
constexpr int OFF_DB = OFF_DW + H;
constexpr int NPARAM = OFF_DB + 1;

}  // namespace

struct sfc_mpnn {
    sfc_ctx *ctx = nullptr;
    int64_t step = 0;
    sfc::DBuf<float> params, grads, adam_m, adam_v;
    sfc::DBuf<__nv_bfloat16> wbf;  // LAYERS x [64][128] BF16 copies
    // operator-dependent data (for the system the network was last used on)
    const sfc_system *op_sys = nullptr;
    int64_t N = 0;
    sfc::DBuf<float> ahat, sdinv;
    // activations and gradients
    sfc::DBuf<float> x0, ax0, yhat, tgt, dvec, qvec, H[LAYERS + 1], Y[LAYERS + 1], dH0, dH1, dY;
    sfc::DBuf<__nv_bfloat16> hb[2];  // inference activations (BF16, ping-pong)
    sfc::DBuf<int> tc_err;           // bounded-wait status of the tensor-core layers
    sfc::DBuf<double> fcg_sc;        // flexible-CG scalars, per iteration
    sfc::DBuf<int> fcg_flags;        // done, breakdown
    sfc::DBuf<double> scal;  // [0]: N s^2 = |D^-1/2 r|^2, [1]: loss
    // training pairs (FP64, N each)
    sfc::DBuf<double> pr, pe;
    std::vector<double> pw;  // per-pair loss weights
    int npairs = 0;
};

namespace sfc {
namespace {

__device__ __forceinline__ float warp_sumf(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low half) = lo
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// D (16x8, f32) += A (16x16, bf16, row) * B (16x8, bf16, col)
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---- operator scaling --------------------------------------------------------
__global__ void k_scale_op(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                           const int32_t *__restrict__ diag, const double *__restrict__ a, int64_t N,
                           float *__restrict__ ahat, float *__restrict__ sdinv)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double si = 1.0 / sqrt(a[diag[i]]);
        sdinv[i] = (float)si;
        for (int32_t s = rp[i]; s < rp[i + 1]; ++s) {
            const int32_t j = col[s];
            ahat[s] = (float)(a[s] * si / sqrt(a[diag[j]]));
        }
    }
}

// y = Ahat x (one column), warp per row
__global__ void k_spmv32(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                         const float *__restrict__ v, const float *__restrict__ x, float *__restrict__ y, int64_t N)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        float s = 0.f;
        for (int32_t k = rp[i] + lane; k < rp[i + 1]; k += 32) s = fmaf(v[k], x[col[k]], s);
        s = warp_sumf(s);
        if (lane == 0) y[i] = s;
    }
}

// Y (+)= Ahat X for 64 feature columns, warp per row, two features per lane
__global__ void k_agg64(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                        const float *__restrict__ v, const float *__restrict__ X, float *__restrict__ Y, int64_t N,
                        int accumulate)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        float2 acc = make_float2(0.f, 0.f);
        const int32_t b = rp[i], e = rp[i + 1];
        for (int32_t s0 = b; s0 < e; s0 += 32) {
            const int32_t s = s0 + lane;
            const float av = s < e ? v[s] : 0.f;
            const int32_t cv = s < e ? col[s] : 0;
            const int n = min(32, e - s0);
            for (int j = 0; j < n; ++j) {
                const float aj = __shfl_sync(0xffffffffu, av, j);
                const int32_t cj = __shfl_sync(0xffffffffu, cv, j);
                const float2 xv = *reinterpret_cast<const float2 *>(X + (int64_t)cj * H + 2 * lane);
                acc.x = fmaf(aj, xv.x, acc.x);
                acc.y = fmaf(aj, xv.y, acc.y);
            }
        }
        float2 *out = reinterpret_cast<float2 *>(Y + i * H + 2 * lane);
        if (accumulate) {
            const float2 o = *out;
            acc.x += o.x;
            acc.y += o.y;
        }
        *out = acc;
    }
}

// x0 = D^-1/2 r / s  (N s^2 in scal[0])
__global__ void k_x0(const double *__restrict__ r, const float *__restrict__ sdinv, const double *scal, int64_t N,
                     float *__restrict__ x0)
{
    const double inv = scal[0] > 0 ? 1.0 / sqrt(scal[0] / (double)N) : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        x0[i] = (float)(r[i] * (double)sdinv[i] * inv);
}

// scal[slot] += sum (D^-1/2 v)^2
// (and rhat = FP32(D^-1/2 v) when rhat != NULL)
__global__ void k_scaled_norm2(const double *__restrict__ v, const float *__restrict__ sdinv, int64_t N, double *out,
                               float *__restrict__ rhat = nullptr)
{
    __shared__ double sh[32];
    double s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double t = v[i] * (double)sdinv[i];
        s += t * t;
        if (rhat) rhat[i] = (float)t;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

__global__ void k_encoder(const float *__restrict__ x0, const float *__restrict__ ax0, const float *__restrict__ P,
                          int64_t N, float *__restrict__ H0)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * H; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / H;
        const int k = (int)(t - i * H);
        const float z = fmaf(P[OFF_EW + 2 * k], x0[i], fmaf(P[OFF_EW + 2 * k + 1], ax0[i], P[OFF_EB + k]));
        H0[t] = fmaxf(z, 0.f);
    }
}

// Hout = relu([Hin | Yin] W^T + b), 16 nodes per warp, BF16 mma, FP32 accumulate
__global__ void __launch_bounds__(256) k_dense_fwd(const float *__restrict__ Hin, const float *__restrict__ Yin,
                                                   const __nv_bfloat16 *__restrict__ W, const float *__restrict__ bias,
                                                   int64_t N, float *__restrict__ Hout)
{
    __shared__ __align__(16) __nv_bfloat16 sW[H * 2 * H];
    for (int t = threadIdx.x; t < H * 2 * H; t += blockDim.x) sW[t] = W[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int64_t tiles = (N + 15) / 16;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t tile = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; tile < tiles; tile += warps) {
        const int64_t r0 = tile * 16 + gid, r1 = r0 + 8;
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
            const float *src = ks < 4 ? Hin : Yin;
            const int c0 = (ks & 3) * 16 + tig * 2, c1 = c0 + 8;
            float2 v00 = make_float2(0.f, 0.f), v01 = v00, v10 = v00, v11 = v00;
            if (r0 < N) {
                v00 = *reinterpret_cast<const float2 *>(src + r0 * H + c0);
                v01 = *reinterpret_cast<const float2 *>(src + r0 * H + c1);
            }
            if (r1 < N) {
                v10 = *reinterpret_cast<const float2 *>(src + r1 * H + c0);
                v11 = *reinterpret_cast<const float2 *>(src + r1 * H + c1);
            }
            const uint32_t a[4] = {pack_bf16(v00.x, v00.y), pack_bf16(v10.x, v10.y), pack_bf16(v01.x, v01.y),
                                   pack_bf16(v11.x, v11.y)};
            const int k = ks * 16 + tig * 2;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int n = nt * 8 + gid;
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&sW[n * 2 * H + k]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&sW[n * 2 * H + k + 8]);
                mma16816(acc[nt], a, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int c = nt * 8 + tig * 2;
            const float b0 = bias[c], b1 = bias[c + 1];
            if (r0 < N)
                *reinterpret_cast<float2 *>(Hout + r0 * H + c) =
                    make_float2(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
            if (r1 < N)
                *reinterpret_cast<float2 *>(Hout + r1 * H + c) =
                    make_float2(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
        }
    }
}

// yhat = x0 + (w . H3 + c) on free dofs, x0 on constrained ones; warp per node
__global__ void k_decoder(const float *__restrict__ H3, const float *__restrict__ P, const float *__restrict__ x0,
                          const unsigned char *__restrict__ mask, int64_t N, float *__restrict__ yhat)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float w0 = P[OFF_DW + 2 * lane], w1 = P[OFF_DW + 2 * lane + 1], c = P[OFF_DB];
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const float2 h = *reinterpret_cast<const float2 *>(H3 + i * H + 2 * lane);
        const float s = warp_sumf(fmaf(w0, h.x, w1 * h.y));
        if (lane == 0) yhat[i] = mask[i] ? x0[i] : x0[i] + s + c;
    }
}

// target t = D^1/2 e / s
__global__ void k_target(const double *__restrict__ e, const float *__restrict__ sdinv, const double *scal, int64_t N,
                         float *__restrict__ t)
{
    const double inv = scal[0] > 0 ? 1.0 / sqrt(scal[0] / (double)N) : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        t[i] = (float)(e[i] / (double)sdinv[i] * inv);
}

__global__ void k_sub(const float *__restrict__ a, const float *__restrict__ b, int64_t N, float *__restrict__ d)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = a[i] - b[i];
}

// loss += w d . q / N ; g = 2 w q / N (in place)
__global__ void k_loss(const float *__restrict__ d, float *__restrict__ q, int64_t N, double w, double *loss)
{
    __shared__ double sh[32];
    double s = 0;
    const float g2 = (float)(2.0 * w / (double)N);
    const double invn = w / (double)N;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        s += (double)d[i] * (double)q[i] * invn;
        q[i] *= g2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(loss, s);
    }
}

// decoder backward: dH3 = g w ; dw += sum_i g_i H3_i ; dc += sum g_i
__global__ void k_decoder_bwd(const float *__restrict__ g, const float *__restrict__ H3, const float *__restrict__ P,
                              const unsigned char *__restrict__ mask, int64_t N, float *__restrict__ dH3,
                              float *__restrict__ G)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float w0 = P[OFF_DW + 2 * lane], w1 = P[OFF_DW + 2 * lane + 1];
    float a0 = 0.f, a1 = 0.f, ac = 0.f;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const float gi = mask[i] ? 0.f : g[i];
        const float2 h = *reinterpret_cast<const float2 *>(H3 + i * H + 2 * lane);
        *reinterpret_cast<float2 *>(dH3 + i * H + 2 * lane) = make_float2(gi * w0, gi * w1);
        a0 = fmaf(gi, h.x, a0);
        a1 = fmaf(gi, h.y, a1);
        ac += gi;
    }
    atomicAdd(&G[OFF_DW + 2 * lane], a0);
    atomicAdd(&G[OFF_DW + 2 * lane + 1], a1);
    if (lane == 0) atomicAdd(&G[OFF_DB], ac);
}

// input gradient of a dense layer: dZ = dH * (Hl > 0) (BF16),
// [dHprev | dY] = dZ W  (16 nodes per warp, mma, FP32 accumulate)
__global__ void __launch_bounds__(256) k_dense_bwd_x(const float *__restrict__ dH, const float *__restrict__ Hl,
                                                     const __nv_bfloat16 *__restrict__ W, int64_t N,
                                                     float *__restrict__ dHprev, float *__restrict__ dY)
{
    __shared__ __align__(16) __nv_bfloat16 sW[H * 2 * H];
    for (int t = threadIdx.x; t < H * 2 * H; t += blockDim.x) sW[t] = W[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int64_t tiles = (N + 15) / 16;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t tile = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; tile < tiles; tile += warps) {
        const int64_t r0 = tile * 16 + gid, r1 = r0 + 8;
        float acc[16][4];
#pragma unroll
        for (int nt = 0; nt < 16; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const int c0 = ks * 16 + tig * 2, c1 = c0 + 8;
            float v[4][2] = {};
            if (r0 < N) {
                const float2 d0 = *reinterpret_cast<const float2 *>(dH + r0 * H + c0);
                const float2 d1 = *reinterpret_cast<const float2 *>(dH + r0 * H + c1);
                const float2 h0 = *reinterpret_cast<const float2 *>(Hl + r0 * H + c0);
                const float2 h1 = *reinterpret_cast<const float2 *>(Hl + r0 * H + c1);
                v[0][0] = h0.x > 0.f ? d0.x : 0.f;
                v[0][1] = h0.y > 0.f ? d0.y : 0.f;
                v[2][0] = h1.x > 0.f ? d1.x : 0.f;
                v[2][1] = h1.y > 0.f ? d1.y : 0.f;
            }
            if (r1 < N) {
                const float2 d0 = *reinterpret_cast<const float2 *>(dH + r1 * H + c0);
                const float2 d1 = *reinterpret_cast<const float2 *>(dH + r1 * H + c1);
                const float2 h0 = *reinterpret_cast<const float2 *>(Hl + r1 * H + c0);
                const float2 h1 = *reinterpret_cast<const float2 *>(Hl + r1 * H + c1);
                v[1][0] = h0.x > 0.f ? d0.x : 0.f;
                v[1][1] = h0.y > 0.f ? d0.y : 0.f;
                v[3][0] = h1.x > 0.f ? d1.x : 0.f;
                v[3][1] = h1.y > 0.f ? d1.y : 0.f;
            }
            const uint32_t a[4] = {pack_bf16(v[0][0], v[0][1]), pack_bf16(v[1][0], v[1][1]),
                                   pack_bf16(v[2][0], v[2][1]), pack_bf16(v[3][0], v[3][1])};
            const int k = ks * 16 + tig * 2;  // output-feature index of W rows
#pragma unroll
            for (int nt = 0; nt < 16; ++nt) {
                const int n = nt * 8 + gid;  // input-feature index (0..127)
                const uint32_t b0 = (uint32_t) * reinterpret_cast<const uint16_t *>(&sW[k * 2 * H + n]) |
                                    ((uint32_t) * reinterpret_cast<const uint16_t *>(&sW[(k + 1) * 2 * H + n]) << 16);
                const uint32_t b1 =
                    (uint32_t) * reinterpret_cast<const uint16_t *>(&sW[(k + 8) * 2 * H + n]) |
                    ((uint32_t) * reinterpret_cast<const uint16_t *>(&sW[(k + 9) * 2 * H + n]) << 16);
                mma16816(acc[nt], a, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 16; ++nt) {
            const int c = nt * 8 + tig * 2;
            float *dst = c < H ? dHprev : dY;
            const int cc = c < H ? c : c - H;
            if (r0 < N) *reinterpret_cast<float2 *>(dst + r0 * H + cc) = make_float2(acc[nt][0], acc[nt][1]);
            if (r1 < N) *reinterpret_cast<float2 *>(dst + r1 * H + cc) = make_float2(acc[nt][2], acc[nt][3]);
        }
    }
}

// weight gradient of a dense layer: dW[o][j] += sum_i dZ[i][o] Xc[i][j] with
// dZ and Xc = [Hin | Yin] rounded to BF16 (the operands of the tensor-core
// products), db[o] += sum_i dZ[i][o] unrounded; FP32 accumulate
constexpr int kTN = 32;
__global__ void __launch_bounds__(256) k_dense_bwd_w(const float *__restrict__ dH, const float *__restrict__ Hl,
                                                     const float *__restrict__ Hin, const float *__restrict__ Yin,
                                                     int64_t N, float *__restrict__ GW, float *__restrict__ Gb)
{
    __shared__ float sZ[kTN][H];
    __shared__ float sX[kTN][2 * H + 1];
    const int o = threadIdx.x >> 2, jq = threadIdx.x & 3;  // 64 outputs x 4 interleaved input groups
    float acc[32];
#pragma unroll
    for (int u = 0; u < 32; ++u) acc[u] = 0.f;
    float accb = 0.f;
    for (int64_t n0 = (int64_t)blockIdx.x * kTN; n0 < N; n0 += (int64_t)gridDim.x * kTN) {
        __syncthreads();
        for (int t = threadIdx.x; t < kTN * H; t += blockDim.x) {
            const int ii = t / H, k = t % H;
            const int64_t i = n0 + ii;
            float z = 0.f;
            if (i < N) z = Hl[i * H + k] > 0.f ? dH[i * H + k] : 0.f;
            sZ[ii][k] = z;
        }
        for (int t = threadIdx.x; t < kTN * 2 * H; t += blockDim.x) {
            const int ii = t / (2 * H), j = t % (2 * H);
            const int64_t i = n0 + ii;
            float x = 0.f;
            if (i < N) x = j < H ? Hin[i * H + j] : Yin[i * H + j - H];
            sX[ii][j] = bf16r(x);
        }
        __syncthreads();
        for (int ii = 0; ii < kTN; ++ii) {
            const float z0 = sZ[ii][o], z = bf16r(z0);
            if (jq == 0) accb += z0;
#pragma unroll
            for (int u = 0; u < 32; ++u) acc[u] = fmaf(z, sX[ii][u * 4 + jq], acc[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < 32; ++u) atomicAdd(&GW[o * 2 * H + u * 4 + jq], acc[u]);
    if (jq == 0) atomicAdd(&Gb[o], accb);
}

__global__ void k_encoder_bwd(const float *__restrict__ dH0, const float *__restrict__ H0, const float *__restrict__ x0,
                              const float *__restrict__ ax0, int64_t N, float *__restrict__ G)
{
    // thread owns feature k = threadIdx.x & 63 for its node stride
    const int k = threadIdx.x & (H - 1);
    float a0 = 0.f, a1 = 0.f, ab = 0.f;
    const int64_t lanes = (int64_t)gridDim.x * (blockDim.x / H);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / H; i < N; i += lanes) {
        const float z = H0[i * H + k] > 0.f ? dH0[i * H + k] : 0.f;
        a0 = fmaf(z, x0[i], a0);
        a1 = fmaf(z, ax0[i], a1);
        ab += z;
    }
    atomicAdd(&G[OFF_EW + 2 * k], a0);
    atomicAdd(&G[OFF_EW + 2 * k + 1], a1);
    atomicAdd(&G[OFF_EB + k], ab);
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       float clip)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        float g = fminf(fmaxf(G[t], -clip), clip);
        m[t] = b1 * m[t] + (1.f - b1) * g;
        v[t] = b2 * v[t] + (1.f - b2) * g * g;
        P[t] -= lr * (m[t] / c1) / (sqrtf(v[t] / c2) + eps);
    }
}

__global__ void k_to_bf16(const float *__restrict__ P, __nv_bfloat16 *__restrict__ wbf)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < LAYERS * H * 2 * H; t += gridDim.x * blockDim.x) {
        const int l = t / (H * 2 * H), r = t % (H * 2 * H);
        wbf[t] = __float2bfloat16_rn(P[OFF_L + l * LSZ + r]);
    }
}

// ---- inference: BF16 activations, gather fused with the dense transform --------
// The stored activations are the BF16 values the tensor-core products round
// them to anyway; the aggregation reads them (half the gather traffic of
// FP32) and accumulates in FP32.
constexpr int kLS = 68;  // shared-memory row stride in 32-bit words (136 BF16): conflict-free fragments

__device__ __forceinline__ float2 bf16x2_to_f2(uint32_t u)
{
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(v);
}

// x0 = rhat / s, H0 = BF16(relu(E [x0, Ahat x0] + e)) with Ahat x0 =
// (Ahat rhat) / s; 8 lanes per node (8 features each), 4 nodes per warp trip
__global__ void k_encoder_inf(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                              const float *__restrict__ v, const float *__restrict__ rhat, const double *scal,
                              const float *__restrict__ P, int64_t N, float *__restrict__ x0, uint4 *__restrict__ H0)
{
    const int lane = threadIdx.x & 31, sub = lane >> 3, fl = lane & 7;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float inv = scal[0] > 0 ? (float)(1.0 / sqrt(scal[0] / (double)N)) : 0.f;
    float e0[8], e1[8], eb[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        e0[q] = P[OFF_EW + 2 * (fl * 8 + q)];
        e1[q] = P[OFF_EW + 2 * (fl * 8 + q) + 1];
        eb[q] = P[OFF_EB + fl * 8 + q];
    }
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 4; base < N; base += nwarps * 4) {
        const int64_t i = base + sub;
        const bool valid = i < N;
        float acc = 0.f;
        if (valid)
            for (int32_t k = rp[i] + fl; k < rp[i + 1]; k += 8) acc = fmaf(v[k], rhat[col[k]], acc);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        if (!valid) continue;
        const float xi = rhat[i] * inv, ax = acc * inv;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            w[q] = pack_bf16(fmaxf(fmaf(e0[2 * q], xi, fmaf(e1[2 * q], ax, eb[2 * q])), 0.f),
                             fmaxf(fmaf(e0[2 * q + 1], xi, fmaf(e1[2 * q + 1], ax, eb[2 * q + 1])), 0.f));
        H0[i * 8 + fl] = make_uint4(w[0], w[1], w[2], w[3]);
        if (fl == 0) x0[i] = xi;
    }
}

// One message-passing layer, 16 nodes per warp: gather Ahat Hin for the
// tile's rows into shared memory beside the rows of Hin, then
// [Hin | Ahat Hin] W^T on BF16 mma fragments (FP32 accumulate), bias, relu.
// DECODE (last layer): instead of storing H, z = s D^-1/2 (x0 + w . H + c)
// (x0 alone on constrained dofs).
template <bool DECODE>
__global__ void __launch_bounds__(128) k_layer_inf(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                   const float *__restrict__ v, const uint32_t *__restrict__ Hin,
                                                   const __nv_bfloat16 *__restrict__ W, const float *__restrict__ bias,
                                                   int64_t N, uint32_t *__restrict__ Hout,
                                                   const float *__restrict__ P, const float *__restrict__ x0,
                                                   const float *__restrict__ sdinv,
                                                   const unsigned char *__restrict__ mask, const double *scal,
                                                   double *__restrict__ z)
{
    __shared__ __align__(16) uint32_t sW[H * kLS];
    __shared__ __align__(16) uint32_t sA[4][16 * kLS];
    const uint32_t *W32 = reinterpret_cast<const uint32_t *>(W);
    for (int t = threadIdx.x; t < H * H; t += blockDim.x) sW[(t / H) * kLS + (t % H)] = W32[t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    uint32_t *tileA = sA[warp];
    const int64_t tiles = (N + 15) / 16;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t tile = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp; tile < tiles; tile += nwarps) {
        // gather: 8 lanes per row (8 features = 16 bytes each), 4 rows at a
        // time, 8 neighbours per trip with independent loads
        const int sub = lane >> 3, fl = lane & 7;
        const uint4 *Hin4 = reinterpret_cast<const uint4 *>(Hin);
        for (int pass = 0; pass < 4; ++pass) {
            const int rr = pass * 4 + sub;
            const int64_t i = tile * 16 + rr;
            const bool valid = i < N;
            const int32_t b = valid ? rp[i] : 0;
            const int len = valid ? rp[i + 1] - b : 0;
            int maxlen = len;
            maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, 8));
            maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, 16));
            float acc[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[q] = 0.f;
            for (int s0 = 0; s0 < maxlen; s0 += 8) {
                const int sl = s0 + fl;
                const int32_t cv = sl < len ? col[b + sl] : 0;  // padding: row 0 with weight 0
                const float av = sl < len ? v[b + sl] : 0.f;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int32_t cj = __shfl_sync(0xffffffffu, cv, j, 8);
                    const float aj = __shfl_sync(0xffffffffu, av, j, 8);
                    const uint4 u = Hin4[(int64_t)cj * 8 + fl];
                    const float2 f0 = bf16x2_to_f2(u.x), f1 = bf16x2_to_f2(u.y), f2 = bf16x2_to_f2(u.z),
                                 f3 = bf16x2_to_f2(u.w);
                    acc[0] = fmaf(aj, f0.x, acc[0]);
                    acc[1] = fmaf(aj, f0.y, acc[1]);
                    acc[2] = fmaf(aj, f1.x, acc[2]);
                    acc[3] = fmaf(aj, f1.y, acc[3]);
                    acc[4] = fmaf(aj, f2.x, acc[4]);
                    acc[5] = fmaf(aj, f2.y, acc[5]);
                    acc[6] = fmaf(aj, f3.x, acc[6]);
                    acc[7] = fmaf(aj, f3.y, acc[7]);
                }
            }
            const uint4 hv = valid ? Hin4[i * 8 + fl] : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(&tileA[rr * kLS + fl * 4]) = hv;
            *reinterpret_cast<uint4 *>(&tileA[rr * kLS + 32 + fl * 4]) =
                make_uint4(pack_bf16(acc[0], acc[1]), pack_bf16(acc[2], acc[3]), pack_bf16(acc[4], acc[5]),
                           pack_bf16(acc[6], acc[7]));
        }
        __syncwarp();
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
            const int kw = ks * 8 + tig;  // 32-bit word of columns (k, k+1), k = ks*16 + 2*tig
            const uint32_t a[4] = {tileA[gid * kLS + kw], tileA[(gid + 8) * kLS + kw], tileA[gid * kLS + kw + 4],
                                   tileA[(gid + 8) * kLS + kw + 4]};
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int n = nt * 8 + gid;
                mma16816(acc[nt], a, sW[n * kLS + kw], sW[n * kLS + kw + 4]);
            }
        }
        __syncwarp();
        if constexpr (!DECODE) {
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int c = nt * 8 + tig * 2;
                const float b0 = bias[c], b1 = bias[c + 1];
                tileA[gid * kLS + c / 2] = pack_bf16(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
                tileA[(gid + 8) * kLS + c / 2] = pack_bf16(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
            }
            __syncwarp();
            for (int rr = 0; rr < 16; ++rr) {
                const int64_t i = tile * 16 + rr;
                if (i < N) Hout[i * (H / 2) + lane] = tileA[rr * kLS + lane];
            }
            __syncwarp();
        } else {
            float y0 = 0.f, y1 = 0.f;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int c = nt * 8 + tig * 2;
                const float b0 = bias[c], b1 = bias[c + 1], w0 = P[OFF_DW + c], w1 = P[OFF_DW + c + 1];
                y0 = fmaf(w0, fmaxf(acc[nt][0] + b0, 0.f), fmaf(w1, fmaxf(acc[nt][1] + b1, 0.f), y0));
                y1 = fmaf(w0, fmaxf(acc[nt][2] + b0, 0.f), fmaf(w1, fmaxf(acc[nt][3] + b1, 0.f), y1));
            }
            y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
            y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
            y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
            y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
            if (tig == 0) {
                const double sc = sqrt(scal[0] / (double)N);
                const float c0 = P[OFF_DB];
                const int64_t i0 = tile * 16 + gid, i1 = i0 + 8;
                if (i0 < N) z[i0] = sc * (double)sdinv[i0] * (double)(mask[i0] ? x0[i0] : x0[i0] + y0 + c0);
                if (i1 < N) z[i1] = sc * (double)sdinv[i1] * (double)(mask[i1] ? x0[i1] : x0[i1] + y1 + c0);
            }
        }
    }
}

// ---- inference on the 5th-generation tensor cores (tcgen05) ---------------------
// A CTA of eight warps takes 128 nodes at a time: the warps gather the tile's
// [Hin | Ahat Hin] rows (BF16, K = 128) into shared memory in the canonical
// K-major layout without swizzle (8-row x 16-byte core matrices: core (row
// group g, K chunk c) at byte (16 g + c) * 128, so the next K chunk is 128
// bytes on (LBO) and the next 8-row group 2,048 bytes on (SBO)); W (64 x 128,
// K-major) sits beside it in the same layout for the whole kernel.  One thread
// issues eight tcgen05.mma (M = 128, N = 64, K = 16, BF16 x BF16 -> FP32)
// into a 64-column accumulator in tensor memory and commits them to an
// mbarrier; warps w and w + 4 then read the 32 rows of TMEM lanes 32 (w % 4)
// .. with tcgen05.ld, columns 0-31 and 32-63 respectively, add the bias, apply
// relu and store BF16 rows (or, DECODE, the decoded correction z).  The mbarrier wait is bounded: on a timeout the
// kernel sets *err, waits once more (bounded) for the MMAs in flight, frees
// its tensor memory and leaves.
constexpr int kTcRows = 128;           // nodes per tile (MMA M)
constexpr uint32_t kTcCols = 64;       // accumulator columns (MMA N), tensor-memory columns allocated
constexpr int kTcBBytes = H * 2 * H * 2;      // W: 16 KiB
constexpr int kTcABytes = kTcRows * 2 * H * 2;  // A tile: 32 KiB
constexpr size_t kTcSmem = (size_t)kTcABytes + kTcBBytes + 16;  // + mbarrier + tensor-memory address
constexpr uint32_t kTcWaitTries = 1u << 22;
// instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits
// 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kTcCols >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
static_assert(kTcIdesc == (1u << 4) + (1u << 7) + (1u << 10) + (8u << 17) + (8u << 24), "M = 128, N = 64");

// byte offset of the 16-byte piece (row, K chunk) of a K-major operand with KC
// chunks of 8 BF16 per row in the canonical layout (core matrix = 8 rows of
// one chunk, 128 bytes; next chunk +128 B; next 8-row group + 128 KC B)
template <int KC = 16>
__device__ __forceinline__ uint32_t tc_off(int row, int chunk)
{
    return (uint32_t)(((row >> 3) * KC + chunk) * 128 + (row & 7) * 16);
}

// shared-memory matrix descriptor: start address, LBO = 128 B (next K chunk),
// SBO = 128 KC B (next 8-row group), all in 16-byte units; descriptor version
// 1, no swizzle
template <int KC = 16>
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((128u * KC) >> 4) << 32) | (1ull << 46);
}

// instruction descriptor of a BF16 x BF16 -> FP32 MMA, both operands K-major
constexpr uint32_t tc_idesc(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kTcWaitTries; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t u[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
          "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(u[j]);
}

template <bool DECODE>
__global__ void __launch_bounds__(256, 4) k_layer_tc(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                     const float *__restrict__ v, const uint32_t *__restrict__ Hin,
                                                     const __nv_bfloat16 *__restrict__ W,
                                                     const float *__restrict__ bias, int64_t N,
                                                     uint32_t *__restrict__ Hout, const float *__restrict__ P,
                                                     const float *__restrict__ x0, const float *__restrict__ sdinv,
                                                     const unsigned char *__restrict__ mask, const double *scal,
                                                     double *__restrict__ z, int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *sA = tsm, *sB = tsm + kTcABytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tsm + kTcABytes + kTcBBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tsm + kTcABytes + kTcBBytes + 8);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA), sB_u = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t bar_u = (uint32_t)__cvta_generic_to_shared(bar);
    // W (row n = output feature, 16 chunks of 8 K values) into the canonical layout
    const uint4 *W4 = reinterpret_cast<const uint4 *>(W);
    for (int t = threadIdx.x; t < H * 16; t += blockDim.x)
        *reinterpret_cast<uint4 *>(sB + tc_off(t / 16, t % 16)) = W4[t];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tslot)),
                     "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // W visible to the tensor cores
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __shared__ float ypart[kTcRows];  // DECODE: the upper 32 columns' share of each row's w . H
    const uint32_t tmem = *tslot;
    // warps w and w + 4 share TMEM lanes 32 (w % 4) ..: w < 4 reads columns 0-31, w >= 4 columns 32-63
    const int quad = warp & 3, half = warp >> 2;
    const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16) + 32u * half;
    const int64_t tiles = (N + kTcRows - 1) / kTcRows;
    const uint4 *Hin4 = reinterpret_cast<const uint4 *>(Hin);
    const int sub = lane >> 3, fl = lane & 7;
    uint32_t parity = 0;
    bool ok = !(*err), pending = false;  // pending: MMAs committed and not yet waited for
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // gather: warp w fills rows 16 w .. 16 w + 15, four rows per pass, 8 lanes per row
        for (int pass = 0; pass < 4; ++pass) {
            const int rr = 16 * warp + pass * 4 + sub;
            const int64_t i = tile * kTcRows + rr;
            const bool valid = i < N;
            const int32_t b = valid ? rp[i] : 0;
            const int len = valid ? rp[i + 1] - b : 0;
            int maxlen = len;
            maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, 8));
            maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, 16));
            float acc[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[q] = 0.f;
            for (int s0 = 0; s0 < maxlen; s0 += 8) {
                const int sl = s0 + fl;
                const int32_t cv = sl < len ? col[b + sl] : 0;  // padding: row 0 with weight 0
                const float av = sl < len ? v[b + sl] : 0.f;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int32_t cj = __shfl_sync(0xffffffffu, cv, j, 8);
                    const float aj = __shfl_sync(0xffffffffu, av, j, 8);
                    const uint4 u = Hin4[(int64_t)cj * 8 + fl];
                    const float2 f0 = bf16x2_to_f2(u.x), f1 = bf16x2_to_f2(u.y), f2 = bf16x2_to_f2(u.z),
                                 f3 = bf16x2_to_f2(u.w);
                    acc[0] = fmaf(aj, f0.x, acc[0]);
                    acc[1] = fmaf(aj, f0.y, acc[1]);
                    acc[2] = fmaf(aj, f1.x, acc[2]);
                    acc[3] = fmaf(aj, f1.y, acc[3]);
                    acc[4] = fmaf(aj, f2.x, acc[4]);
                    acc[5] = fmaf(aj, f2.y, acc[5]);
                    acc[6] = fmaf(aj, f3.x, acc[6]);
                    acc[7] = fmaf(aj, f3.y, acc[7]);
                }
            }
            const uint4 hv = valid ? Hin4[i * 8 + fl] : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(sA + tc_off(rr, fl)) = hv;
            *reinterpret_cast<uint4 *>(sA + tc_off(rr, 8 + fl)) =
                make_uint4(pack_bf16(acc[0], acc[1]), pack_bf16(acc[2], acc[3]), pack_bf16(acc[4], acc[5]),
                           pack_bf16(acc[6], acc[7]));
        }
        // the tile is visible to the tensor cores, and every warp has read the
        // previous tile's accumulator
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (threadIdx.x == 0) {
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint64_t da = tc_desc(sA_u + 256u * ks), db = tc_desc(sB_u + 256u * ks);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(kTcIdesc), "r"(ks), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_u)
                         : "memory");
        }
        pending = true;
        ok = __syncthreads_and(tc_wait(bar_u, parity));
        if (!ok) break;
        pending = false;
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int64_t i = tile * kTcRows + 32 * quad + lane;  // this thread's row
        const int c0 = 32 * half;                              // and its first column
        float y = 0.f;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            float d[16];
            tc_ld16(trow + 16u * part, d);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int cb = c0 + 16 * part;
            if constexpr (!DECODE) {
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    w[j] = pack_bf16(fmaxf(d[2 * j] + bias[cb + 2 * j], 0.f),
                                     fmaxf(d[2 * j + 1] + bias[cb + 2 * j + 1], 0.f));
                if (i < N) {
                    uint4 *dst = reinterpret_cast<uint4 *>(Hout + i * (H / 2) + cb / 2);
                    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) y = fmaf(P[OFF_DW + cb + j], fmaxf(d[j] + bias[cb + j], 0.f), y);
            }
        }
        if constexpr (DECODE) {
            if (half) ypart[32 * quad + lane] = y;
            __syncthreads();
            if (!half && i < N) {
                y += ypart[32 * quad + lane];
                const double sc = sqrt(scal[0] / (double)N);
                z[i] = sc * (double)sdinv[i] * (double)(mask[i] ? x0[i] : x0[i] + y + P[OFF_DB]);
            }
        }
    }
    if (!ok && pending) {
        // a wait gave up: record it and let the MMAs in flight finish (bounded)
        if (threadIdx.x == 0) atomicExch(err, 1);
        tc_wait(bar_u, parity);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
}

// ---- training products on tcgen05 --------------------------------------------------
// Shared steps of the tensor-core kernels below: warp 0 allocates NCOLS
// tensor-memory columns and thread 0 initialises the mbarrier; tc_product
// makes the staged operands visible to the tensor cores, lets thread 0 issue
// the KS K-steps (16 each) and commit them, and waits for them (bounded);
// tc_finish frees the tensor memory after a last bounded wait when a product
// is still in flight.
template <uint32_t NCOLS>
__device__ __forceinline__ uint32_t tc_setup(uint32_t *tslot, uint32_t bar_u)
{
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tslot)),
                     "r"(NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return *tslot;
}

template <int KCA, int KCB, int KS, uint32_t IDESC>
__device__ __forceinline__ bool tc_product(uint32_t sA_u, uint32_t sB_u, uint32_t tmem, uint32_t bar_u,
                                           uint32_t parity)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const uint64_t da = tc_desc<KCA>(sA_u + 256u * ks), db = tc_desc<KCB>(sB_u + 256u * ks);
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                :
                : "r"(tmem), "l"(da), "l"(db), "r"(IDESC), "r"(ks), "r"(0u)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_u)
                     : "memory");
    }
    const bool ok = __syncthreads_and(tc_wait(bar_u, parity));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return ok;
}

template <uint32_t NCOLS>
__device__ __forceinline__ void tc_finish(uint32_t tmem, uint32_t bar_u, uint32_t parity, bool ok, bool pending,
                                          int *err)
{
    if (!ok && pending) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        tc_wait(bar_u, parity);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS));
}

// Hout = relu([Hin | Yin] W^T + b) on tcgen05: 128 nodes per tile, the FP32
// inputs rounded to BF16 into the canonical K-major layout (K = 128), W
// (64 x 128) staged once; M = 128, N = 64, eight K-steps into 64 TMEM columns.
// Eight warps; warps w and w + 4 read back TMEM lanes 32 (w % 4) .., columns
// 0-31 and 32-63.
constexpr size_t kTcFwdSmem = (size_t)kTcABytes + kTcBBytes + 16;

__global__ void __launch_bounds__(256, 4) k_dense_fwd_tc(const float *__restrict__ Hin, const float *__restrict__ Yin,
                                                         const __nv_bfloat16 *__restrict__ W,
                                                         const float *__restrict__ bias, int64_t N,
                                                         float *__restrict__ Hout, int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *sA = tsm, *sB = tsm + kTcABytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tsm + kTcABytes + kTcBBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tsm + kTcABytes + kTcBBytes + 8);
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA), sB_u = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t bar_u = (uint32_t)__cvta_generic_to_shared(bar);
    const uint4 *W4 = reinterpret_cast<const uint4 *>(W);
    for (int t = threadIdx.x; t < H * 16; t += blockDim.x) *reinterpret_cast<uint4 *>(sB + tc_off(t / 16, t % 16)) = W4[t];
    const uint32_t tmem = tc_setup<64>(tslot, bar_u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, quad = warp & 3, half = warp >> 2;
    const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16) + 32u * half;
    const int64_t tiles = (N + kTcRows - 1) / kTcRows;
    uint32_t parity = 0;
    bool ok = !(*err), pending = false;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // 128 rows x 16 pieces of 8 inputs: 8 pieces per thread
        for (int t = threadIdx.x; t < kTcRows * 16; t += blockDim.x) {
            const int rr = t >> 4, c = t & 15;
            const int64_t i = tile * kTcRows + rr;
            uint4 u = make_uint4(0, 0, 0, 0);
            if (i < N) {
                const float4 *src = reinterpret_cast<const float4 *>((c < 8 ? Hin : Yin) + i * H + (c & 7) * 8);
                const float4 a = src[0], b = src[1];
                u = make_uint4(pack_bf16(a.x, a.y), pack_bf16(a.z, a.w), pack_bf16(b.x, b.y), pack_bf16(b.z, b.w));
            }
            *reinterpret_cast<uint4 *>(sA + tc_off(rr, c)) = u;
        }
        pending = true;
        ok = tc_product<16, 16, 8, tc_idesc(128, 64)>(sA_u, sB_u, tmem, bar_u, parity);
        if (!ok) break;
        pending = false;
        parity ^= 1u;
        const int64_t i = tile * kTcRows + 32 * quad + lane;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            float d[16];
            tc_ld16(trow + 16u * part, d);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int cb = 32 * half + 16 * part;
            if (i < N) {
                float4 *dst = reinterpret_cast<float4 *>(Hout + i * H + cb);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dst[q] = make_float4(fmaxf(d[4 * q] + bias[cb + 4 * q], 0.f),
                                         fmaxf(d[4 * q + 1] + bias[cb + 4 * q + 1], 0.f),
                                         fmaxf(d[4 * q + 2] + bias[cb + 4 * q + 2], 0.f),
                                         fmaxf(d[4 * q + 3] + bias[cb + 4 * q + 3], 0.f));
            }
        }
    }
    tc_finish<64>(tmem, bar_u, parity, ok, pending, err);
}

// [dHprev | dY] = dZ W with dZ = dH * (Hl > 0) on tcgen05: A = dZ rounded to
// BF16 (128 x 64, K = 64 over the layer's outputs), B = W^T (128 x 64, staged
// once from W by columns); M = 128, N = 128, four K-steps into 128 TMEM
// columns.  Warps w and w + 4 read back TMEM lanes 32 (w % 4) .., columns
// 0-63 (dHprev) and 64-127 (dY).
constexpr int kTcXABytes = kTcRows * H * 2;   // 16 KiB
constexpr int kTcXBBytes = 2 * H * H * 2;     // 16 KiB
constexpr size_t kTcBwdSmem = (size_t)kTcXABytes + kTcXBBytes + 16;

__global__ void __launch_bounds__(256, 4) k_dense_bwd_x_tc(const float *__restrict__ dH, const float *__restrict__ Hl,
                                                           const __nv_bfloat16 *__restrict__ W, int64_t N,
                                                           float *__restrict__ dHprev, float *__restrict__ dY,
                                                           int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *sA = tsm, *sB = tsm + kTcXABytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tsm + kTcXABytes + kTcXBBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tsm + kTcXABytes + kTcXBBytes + 8);
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA), sB_u = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t bar_u = (uint32_t)__cvta_generic_to_shared(bar);
    // B[j][o] = W[o][j]: 128 rows j x 8 pieces of 8 outputs o
    const uint16_t *W16 = reinterpret_cast<const uint16_t *>(W);
    for (int t = threadIdx.x; t < 2 * H * 8; t += blockDim.x) {
        const int j = t >> 3, c = t & 7;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            w[q] = (uint32_t)W16[(8 * c + 2 * q) * 2 * H + j] | ((uint32_t)W16[(8 * c + 2 * q + 1) * 2 * H + j] << 16);
        *reinterpret_cast<uint4 *>(sB + tc_off<8>(j, c)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    const uint32_t tmem = tc_setup<128>(tslot, bar_u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, quad = warp & 3, half = warp >> 2;
    const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16) + 64u * half;
    float *out = half ? dY : dHprev;
    const int64_t tiles = (N + kTcRows - 1) / kTcRows;
    uint32_t parity = 0;
    bool ok = !(*err), pending = false;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // 128 rows x 8 pieces of 8 outputs: 4 pieces per thread
        for (int t = threadIdx.x; t < kTcRows * 8; t += blockDim.x) {
            const int rr = t >> 3, c = t & 7;
            const int64_t i = tile * kTcRows + rr;
            uint4 u = make_uint4(0, 0, 0, 0);
            if (i < N) {
                const float4 *d4 = reinterpret_cast<const float4 *>(dH + i * H + 8 * c);
                const float4 *h4 = reinterpret_cast<const float4 *>(Hl + i * H + 8 * c);
                const float4 a = d4[0], b = d4[1], ha = h4[0], hb = h4[1];
                u = make_uint4(pack_bf16(ha.x > 0.f ? a.x : 0.f, ha.y > 0.f ? a.y : 0.f),
                               pack_bf16(ha.z > 0.f ? a.z : 0.f, ha.w > 0.f ? a.w : 0.f),
                               pack_bf16(hb.x > 0.f ? b.x : 0.f, hb.y > 0.f ? b.y : 0.f),
                               pack_bf16(hb.z > 0.f ? b.z : 0.f, hb.w > 0.f ? b.w : 0.f));
            }
            *reinterpret_cast<uint4 *>(sA + tc_off<8>(rr, c)) = u;
        }
        pending = true;
        ok = tc_product<8, 8, 4, tc_idesc(128, 128)>(sA_u, sB_u, tmem, bar_u, parity);
        if (!ok) break;
        pending = false;
        parity ^= 1u;
        const int64_t i = tile * kTcRows + 32 * quad + lane;
#pragma unroll
        for (int part = 0; part < 4; ++part) {
            float d[16];
            tc_ld16(trow + 16u * part, d);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (i < N) {
                float4 *dst = reinterpret_cast<float4 *>(out + i * H + 16 * part);
#pragma unroll
                for (int q = 0; q < 4; ++q) dst[q] = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
            }
        }
    }
    tc_finish<128>(tmem, bar_u, parity, ok, pending, err);
}

// dW[o][j] += sum_i dZ[i][o] Xc[i][j] (Xc = [Hin | Yin]) and db[o] += sum_i
// dZ[i][o] on tcgen05: the transposed product dW^T = Xc^T dZ with M = 128 (the
// inputs j), N = 64 (the outputs o) and K = the 128 nodes of a tile, both
// operands MN-major as they lie in memory (a node's 8 consecutive features
// are one 16-byte piece: piece (feature group g, node group kg) at byte
// (16 g + kg) * 128 + (node % 8) * 16, so the next node group is 128 B on
// (LBO) and the next feature group 2,048 B on (SBO)), rounded to BF16 like
// the forward products.  A CTA accumulates all its tiles in 64 TMEM columns
// and adds the result to GW once; db (unrounded dZ) is summed on the way.
constexpr uint32_t kTcIdescWgrad = tc_idesc(128, 64) | (1u << 15) | (1u << 16);  // A and B MN-major

__global__ void __launch_bounds__(256, 4) k_dense_bwd_w_tc(const float *__restrict__ dH, const float *__restrict__ Hl,
                                                           const float *__restrict__ Hin,
                                                           const float *__restrict__ Yin, int64_t N,
                                                           float *__restrict__ GW, float *__restrict__ Gb, int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *sA = tsm, *sB = tsm + kTcABytes;  // Xc^T: 128 x 128 (32 KiB); dZ^T: 64 x 128 (16 KiB)
    uint64_t *bar = reinterpret_cast<uint64_t *>(tsm + kTcABytes + kTcBBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tsm + kTcABytes + kTcBBytes + 8);
    __shared__ float sdb[H];
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA), sB_u = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t bar_u = (uint32_t)__cvta_generic_to_shared(bar);
    for (int t = threadIdx.x; t < H; t += blockDim.x) sdb[t] = 0.f;
    const uint32_t tmem = tc_setup<64>(tslot, bar_u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, quad = warp & 3, half = warp >> 2;
    const int64_t tiles = (N + kTcRows - 1) / kTcRows;
    uint32_t parity = 0;
    bool ok = !(*err), pending = false, any = false;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // Xc: 128 nodes x 16 feature groups; dZ: 128 nodes x 8 output groups
        for (int t = threadIdx.x; t < kTcRows * 24; t += blockDim.x) {
            const int node = t / 24, g = t % 24;
            const int64_t i = tile * kTcRows + node;
            uint4 u = make_uint4(0, 0, 0, 0);
            if (i < N) {
                float4 a, b;
                if (g < 16) {
                    const float4 *src = reinterpret_cast<const float4 *>((g < 8 ? Hin : Yin) + i * H + (g & 7) * 8);
                    a = src[0];
                    b = src[1];
                } else {
                    const float4 *d4 = reinterpret_cast<const float4 *>(dH + i * H + (g - 16) * 8);
                    const float4 *h4 = reinterpret_cast<const float4 *>(Hl + i * H + (g - 16) * 8);
                    const float4 da = d4[0], dbv = d4[1], ha = h4[0], hb = h4[1];
                    a = make_float4(ha.x > 0.f ? da.x : 0.f, ha.y > 0.f ? da.y : 0.f, ha.z > 0.f ? da.z : 0.f,
                                    ha.w > 0.f ? da.w : 0.f);
                    b = make_float4(hb.x > 0.f ? dbv.x : 0.f, hb.y > 0.f ? dbv.y : 0.f, hb.z > 0.f ? dbv.z : 0.f,
                                    hb.w > 0.f ? dbv.w : 0.f);
                    // db: unrounded dZ, one shared-memory add per output and piece
                    const int o0 = (g - 16) * 8;
                    atomicAdd(&sdb[o0], a.x);
                    atomicAdd(&sdb[o0 + 1], a.y);
                    atomicAdd(&sdb[o0 + 2], a.z);
                    atomicAdd(&sdb[o0 + 3], a.w);
                    atomicAdd(&sdb[o0 + 4], b.x);
                    atomicAdd(&sdb[o0 + 5], b.y);
                    atomicAdd(&sdb[o0 + 6], b.z);
                    atomicAdd(&sdb[o0 + 7], b.w);
                }
                u = make_uint4(pack_bf16(a.x, a.y), pack_bf16(a.z, a.w), pack_bf16(b.x, b.y), pack_bf16(b.z, b.w));
            }
            const uint32_t off = (uint32_t)((((g < 16 ? g : g - 16) * 16) + (node >> 3)) * 128 + (node & 7) * 16);
            *reinterpret_cast<uint4 *>((g < 16 ? sA : sB) + off) = u;
        }
        pending = true;
        // K-steps of 16 nodes: the descriptors advance by two node groups (256 B);
        // the first tile's first step overwrites the accumulator
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (threadIdx.x == 0) {
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint64_t da = tc_desc<16>(sA_u + 256u * ks), dbd = tc_desc<16>(sB_u + 256u * ks);
                const uint32_t acc = (any || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(dbd), "r"(kTcIdescWgrad), "r"(acc), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_u)
                         : "memory");
        }
        ok = __syncthreads_and(tc_wait(bar_u, parity));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok) break;
        pending = false;
        any = true;
        parity ^= 1u;
    }
    if (ok && any) {
        // D[j][o]: warps w and w + 4 hold inputs j = 32 (w % 4) + lane, outputs 0-31 / 32-63
        const int j = 32 * quad + lane;
        const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16) + 32u * half;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            float d[16];
            tc_ld16(trow + 16u * part, d);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) atomicAdd(&GW[(32 * half + 16 * part + q) * 2 * H + j], d[q]);
        }
    }
    __syncthreads();
    if (ok && any)
        for (int t = threadIdx.x; t < H; t += blockDim.x) atomicAdd(&Gb[t], sdb[t]);
    tc_finish<64>(tmem, bar_u, parity, ok, pending, err);
}

// ---- host side -------------------------------------------------------------------
// the tensor-core (tcgen05) kernels unless SFC_MPNN_TC=0 selects the mma.sync ones
bool use_tc()
{
    static int m = -1;
    if (m < 0) {
        const char *e = std::getenv("SFC_MPNN_TC");
        m = (e && e[0] == '0') ? 0 : 1;
    }
    return m == 1;
}

// grid of the tensor-core kernels (four CTAs per SM by their resources, at
// most 4 x 128 tensor-memory columns; the grid-stride loops take any number of
// tiles); sets their attributes and the error word on first use
unsigned tc_grid(sfc_mpnn *m, int64_t N)
{
    sfc_ctx *ctx = m->ctx;
    if (!m->tc_err.p) {
        m->tc_err.alloc(1);
        SFC_CK(cudaMemsetAsync(m->tc_err.p, 0, sizeof(int), ctx->stream));
    }
    static bool attr = false;
    if (!attr) {
        const std::pair<const void *, size_t> ks[] = {{(const void *)k_layer_tc<false>, kTcSmem},
                                                      {(const void *)k_layer_tc<true>, kTcSmem},
                                                      {(const void *)k_dense_fwd_tc, kTcFwdSmem},
                                                      {(const void *)k_dense_bwd_x_tc, kTcBwdSmem},
                                                      {(const void *)k_dense_bwd_w_tc, kTcFwdSmem}};
        for (const auto &k : ks) {
            SFC_CK(cudaFuncSetAttribute(k.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.second));
            SFC_CK(cudaFuncSetAttribute(k.first, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        }
        attr = true;
    }
    return (unsigned)std::min<int64_t>((N + kTcRows - 1) / kTcRows, (int64_t)ctx->sm_count * 4);
}

// after a batch of applications: a tensor-core layer whose bounded wait gave
// up fails the call
void check_tc(sfc_mpnn *m)
{
    if (!m->tc_err.p) return;
    int h = 0;
    download(m->ctx, &h, m->tc_err.p, 1);
    if (h) {
        SFC_CK(cudaMemsetAsync(m->tc_err.p, 0, sizeof(int), m->ctx->stream));
        fail(SFC_ERR_TIMEOUT, "learned preconditioner: a bounded wait for the tensor-core products gave up");
    }
}

void refresh_bf16(sfc_mpnn *m)
{
    k_to_bf16<<<64, 256, 0, m->ctx->stream>>>(m->params.p, m->wbf.p);
    count_launch(m->ctx);
}

// bind the network to a system's operator (scaled copy of its FP64 values)
void bind(sfc_mpnn *m, sfc_system *s)
{
    sfc_ctx *ctx = m->ctx;
    flush_staged(s);
    build_operator(s);
    const int64_t N = s->N;
    if (m->N != N) {
        m->N = N;
        m->sdinv.alloc(N);
        m->x0.alloc(N);
        m->ax0.alloc(N);
        m->yhat.alloc(N);
        m->tgt.alloc(N);
        m->dvec.alloc(N);
        m->qvec.alloc(N);
        for (int l = 0; l <= LAYERS; ++l) {
            m->H[l].alloc(N * H);
            m->Y[l].alloc(N * H);
        }
        m->hb[0].alloc(N * H);
        m->hb[1].alloc(N * H);
        m->dH0.alloc(N * H);
        m->dH1.alloc(N * H);
        m->dY.alloc(N * H);
    }
    m->ahat.reserve(s->nnz);
    k_scale_op<<<grid_for(N, 128), 128, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_op.p, N, m->ahat.p,
                                                         m->sdinv.p);
    count_launch(ctx);
    m->op_sys = s;
}

unsigned gwarp(sfc_ctx *ctx) { return (unsigned)(ctx->sm_count * 8); }

// forward pass on residual r (device FP64): fills x0, ax0, H[], Y[], yhat
void forward(sfc_mpnn *m, const double *r)
{
    sfc_ctx *ctx = m->ctx;
    const sfc_system *s = m->op_sys;
    const int64_t N = m->N;
    ProfScope ps(ctx, "mpnn_forward", 0.0);
    SFC_CK(cudaMemsetAsync(m->scal.p, 0, sizeof(double), ctx->stream));
    k_scaled_norm2<<<grid_for(N, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(r, m->sdinv.p, N, m->scal.p);
    count_launch(ctx);
    k_x0<<<grid_for(N, 256), 256, 0, ctx->stream>>>(r, m->sdinv.p, m->scal.p, N, m->x0.p);
    k_spmv32<<<gwarp(ctx), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, m->x0.p, m->ax0.p, N);
    k_encoder<<<grid_for(N * H, 256), 256, 0, ctx->stream>>>(m->x0.p, m->ax0.p, m->params.p, N, m->H[0].p);
    count_launch(ctx, 3);
    for (int l = 1; l <= LAYERS; ++l) {
        k_agg64<<<gwarp(ctx), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, m->H[l - 1].p, m->Y[l].p, N, 0);
        if (use_tc())
            k_dense_fwd_tc<<<tc_grid(m, N), 256, kTcFwdSmem, ctx->stream>>>(
                m->H[l - 1].p, m->Y[l].p, m->wbf.p + (l - 1) * H * 2 * H, m->params.p + OFF_L + (l - 1) * LSZ + H * 2 * H,
                N, m->H[l].p, m->tc_err.p);
        else
            k_dense_fwd<<<gwarp(ctx), 256, 0, ctx->stream>>>(m->H[l - 1].p, m->Y[l].p, m->wbf.p + (l - 1) * H * 2 * H,
                                                            m->params.p + OFF_L + (l - 1) * LSZ + H * 2 * H, N,
                                                            m->H[l].p);
        count_launch(ctx, 2);
    }
    k_decoder<<<gwarp(ctx), 256, 0, ctx->stream>>>(m->H[LAYERS].p, m->params.p, m->x0.p, s->mask.p, N, m->yhat.p);
    count_launch(ctx);
}

// residual-dependent quantities of a pair: s, x0, target t, d = yhat - t,
// q = 2 w Ahat d / N (the gradient w.r.t. yhat) and the weighted loss in
// scal[1]; yhat is the network output, or x0 alone for the Jacobi loss
void pair_residual(sfc_mpnn *m, const double *e, const float *yhat, double w)
{
    sfc_ctx *ctx = m->ctx;
    const sfc_system *s = m->op_sys;
    const int64_t N = m->N;
    SFC_CK(cudaMemsetAsync(m->scal.p + 1, 0, sizeof(double), ctx->stream));
    k_target<<<grid_for(N, 256), 256, 0, ctx->stream>>>(e, m->sdinv.p, m->scal.p, N, m->tgt.p);
    k_sub<<<grid_for(N, 256), 256, 0, ctx->stream>>>(yhat, m->tgt.p, N, m->dvec.p);
    k_spmv32<<<gwarp(ctx), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, m->dvec.p, m->qvec.p, N);
    k_loss<<<grid_for(N, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(m->dvec.p, m->qvec.p, N, w, m->scal.p + 1);
    count_launch(ctx, 4);
}

// loss of the Jacobi preconditioner (zero network output) for pair (r, e)
double jacobi_loss(sfc_mpnn *m, const double *r, const double *e)
{
    sfc_ctx *ctx = m->ctx;
    const int64_t N = m->N;
    SFC_CK(cudaMemsetAsync(m->scal.p, 0, sizeof(double), ctx->stream));
    k_scaled_norm2<<<grid_for(N, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(r, m->sdinv.p, N, m->scal.p);
    k_x0<<<grid_for(N, 256), 256, 0, ctx->stream>>>(r, m->sdinv.p, m->scal.p, N, m->x0.p);
    count_launch(ctx, 2);
    pair_residual(m, e, m->x0.p, 1.0);
    double hl = 0;
    download(ctx, &hl, m->scal.p + 1, 1);
    check_tc(m);
    return hl;
}

// weighted loss w * L and its parameter gradient for pair (r, e) (device
// FP64); gradients accumulate into grads; returns w * L
double loss_grad(sfc_mpnn *m, const double *r, const double *e, double w)
{
    sfc_ctx *ctx = m->ctx;
    const sfc_system *s = m->op_sys;
    const int64_t N = m->N;
    forward(m, r);
    ProfScope ps(ctx, "mpnn_backward", 0.0);
    pair_residual(m, e, m->yhat.p, w);
    // qvec = dL/dyhat
    float *dHa = m->dH0.p, *dHb = m->dH1.p;
    k_decoder_bwd<<<gwarp(ctx), 256, 0, ctx->stream>>>(m->qvec.p, m->H[LAYERS].p, m->params.p, s->mask.p, N, dHa,
                                                       m->grads.p);
    count_launch(ctx);
    for (int l = LAYERS; l >= 1; --l) {
        const __nv_bfloat16 *W = m->wbf.p + (l - 1) * H * 2 * H;
        float *GW = m->grads.p + OFF_L + (l - 1) * LSZ;
        if (use_tc())
            k_dense_bwd_w_tc<<<tc_grid(m, N), 256, kTcFwdSmem, ctx->stream>>>(dHa, m->H[l].p, m->H[l - 1].p,
                                                                               m->Y[l].p, N, GW, GW + H * 2 * H,
                                                                               m->tc_err.p);
        else
            k_dense_bwd_w<<<(unsigned)(ctx->sm_count * 2), 256, 0, ctx->stream>>>(dHa, m->H[l].p, m->H[l - 1].p,
                                                                                  m->Y[l].p, N, GW, GW + H * 2 * H);
        if (use_tc())
            k_dense_bwd_x_tc<<<tc_grid(m, N), 256, kTcBwdSmem, ctx->stream>>>(dHa, m->H[l].p, W, N, dHb, m->dY.p,
                                                                               m->tc_err.p);
        else
            k_dense_bwd_x<<<gwarp(ctx), 256, 0, ctx->stream>>>(dHa, m->H[l].p, W, N, dHb, m->dY.p);
        // dH(l-1) += Ahat^T dY (Ahat is symmetric)
        k_agg64<<<gwarp(ctx), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, m->dY.p, dHb, N, 1);
        count_launch(ctx, 3);
        std::swap(dHa, dHb);
    }
    k_encoder_bwd<<<grid_for(N * H, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(dHa, m->H[0].p, m->x0.p,
                                                                                     m->ax0.p, N, m->grads.p);
    count_launch(ctx);
    double hl = 0;
    download(ctx, &hl, m->scal.p + 1, 1);
    check_tc(m);
    return hl;
}

// z = M(r) (device FP64 vectors): the inference kernels, no host synchronisation
void apply(sfc_mpnn *m, const double *r, double *z)
{
    sfc_ctx *ctx = m->ctx;
    const sfc_system *s = m->op_sys;
    const int64_t N = m->N;
    ProfScope ps(ctx, "mpnn_apply", 0.0);
    SFC_CK(cudaMemsetAsync(m->scal.p, 0, sizeof(double), ctx->stream));
    k_scaled_norm2<<<grid_for(N, 256, ctx->sm_count * 4), 256, 0, ctx->stream>>>(r, m->sdinv.p, N, m->scal.p,
                                                                                   m->ax0.p);
    k_encoder_inf<<<gwarp(ctx), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, m->ax0.p, m->scal.p,
                                                       m->params.p, N, m->x0.p, reinterpret_cast<uint4 *>(m->hb[0].p));
    count_launch(ctx, 2);
    if (use_tc()) {
        const unsigned gt = tc_grid(m, N);
        for (int l = 0; l < LAYERS; ++l) {
            const uint32_t *hin = reinterpret_cast<const uint32_t *>(m->hb[l & 1].p);
            uint32_t *hout = reinterpret_cast<uint32_t *>(m->hb[(l + 1) & 1].p);
            const __nv_bfloat16 *W = m->wbf.p + l * H * 2 * H;
            const float *b = m->params.p + OFF_L + l * LSZ + H * 2 * H;
            if (l + 1 < LAYERS)
                k_layer_tc<false><<<gt, 256, kTcSmem, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, hin, W, b, N,
                                                                     hout, m->params.p, m->x0.p, m->sdinv.p,
                                                                     s->mask.p, m->scal.p, nullptr, m->tc_err.p);
            else
                k_layer_tc<true><<<gt, 256, kTcSmem, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, hin, W, b, N,
                                                                    nullptr, m->params.p, m->x0.p, m->sdinv.p,
                                                                    s->mask.p, m->scal.p, z, m->tc_err.p);
            count_launch(ctx);
        }
        return;
    }
    const unsigned g = (unsigned)std::min<int64_t>((N + 63) / 64, (int64_t)ctx->sm_count * 12);
    for (int l = 0; l < LAYERS; ++l) {
        const uint32_t *hin = reinterpret_cast<const uint32_t *>(m->hb[l & 1].p);
        uint32_t *hout = reinterpret_cast<uint32_t *>(m->hb[(l + 1) & 1].p);
        const __nv_bfloat16 *W = m->wbf.p + l * H * 2 * H;
        const float *b = m->params.p + OFF_L + l * LSZ + H * 2 * H;
        if (l + 1 < LAYERS)
            k_layer_inf<false><<<g, 128, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, hin, W, b, N, hout,
                                                           m->params.p, m->x0.p, m->sdinv.p, s->mask.p, m->scal.p,
                                                           nullptr);
        else
            k_layer_inf<true><<<g, 128, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, m->ahat.p, hin, W, b, N, nullptr,
                                                          m->params.p, m->x0.p, m->sdinv.p, s->mask.p, m->scal.p, z);
        count_launch(ctx);
    }
}

void adam_step(sfc_mpnn *m, double lr)
{
    ++m->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    k_adam<<<64, 256, 0, m->ctx->stream>>>(m->params.p, m->grads.p, m->adam_m.p, m->adam_v.p, NPARAM, (float)lr, b1, b2,
                                           1e-8f, c1, c2, 1.0f);
    count_launch(m->ctx);
    refresh_bf16(m);
}

__global__ void k_resid_pair(const double *__restrict__ b, const double *__restrict__ Sx, const double *__restrict__ xs,
                             const double *__restrict__ x, int64_t N, double *__restrict__ r, double *__restrict__ e)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        r[i] = b[i] - Sx[i];
        e[i] = xs[i] - x[i];
    }
}

// Residual/error pairs from Jacobi-PCG on the system's right-hand side b:
// x* converged to 1e-12; x_k = k iterations of PCG from 0, for k = 0 and
// max_pairs - 1 values spaced geometrically up to the iteration at which
// |r_k| / |b| first drops below `floor` (later iterates carry too few digits
// of their error).  Each pair's weight is 1 / (its Jacobi loss) when
// `normalize`, else 1.
void make_pairs(sfc_mpnn *m, sfc_system *s, int max_pairs, double floor, bool normalize)
{
    sfc_ctx *ctx = m->ctx;
    const int64_t N = s->N;
    DBuf<double> b, xs, xk, t;
    b.alloc(N);
    xs.alloc(N);
    xk.alloc(N);
    t.alloc(N);
    lifted_rhs(s, b.p);
    const PcgStats ref = pcg64_public(s, b.p, xs.p, 1e-12, 200000, 32);
    SFC_REQUIRE(ref.converged, "Jacobi-PCG did not converge while generating training pairs");
    const PcgStats fl = pcg64_public(s, b.p, xk.p, floor, 200000, 1);
    const int kmax = std::max(1, fl.iters);
    std::vector<int> ks{0};
    for (int j = 1; j < max_pairs; ++j) {
        const int k = (int)std::lround(std::pow((double)kmax, (double)j / (double)std::max(1, max_pairs - 1)));
        if (k > ks.back()) ks.push_back(k);
    }
    const int np = (int)ks.size();
    m->pr.reserve(N * np);
    m->pe.reserve(N * np);
    m->pw.assign(np, 1.0);
    for (int j = 0; j < np; ++j) {
        if (ks[j] == 0)
            SFC_CK(cudaMemsetAsync(xk.p, 0, N * 8, ctx->stream));
        else
            pcg64_public(s, b.p, xk.p, 1e-300, ks[j], 1 << 30);
        spmv_op64(s, xk.p, t.p);
        k_resid_pair<<<grid_for(N, 256), 256, 0, ctx->stream>>>(b.p, t.p, xs.p, xk.p, N, m->pr.p + j * N,
                                                               m->pe.p + j * N);
        count_launch(ctx);
        if (normalize) {
            const double lj = jacobi_loss(m, m->pr.p + j * N, m->pe.p + j * N);
            m->pw[j] = lj > 0 ? 1.0 / lj : 1.0;
        }
    }
    m->npairs = np;
    SFC_CK(cudaStreamSynchronize(ctx->stream));
}

__global__ void k_resid(const double *__restrict__ b, const double *__restrict__ Sx, int64_t n, double *__restrict__ r)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - Sx[i];
}

__device__ double block_sum_d(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    if (threadIdx.x < 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;  // valid in thread 0
}

// *out += a . b unless *done
__global__ void k_dot_done(const double *__restrict__ a, const double *__restrict__ b, int64_t n, double *out,
                           const int *done)
{
    __shared__ double sh[32];
    if (done && *done) return;
    double v = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v += a[i] * b[i];
    v = block_sum_d(v, sh);
    if (threadIdx.x == 0) atomicAdd(out, v);
}

__global__ void k_axpy(double *__restrict__ y, const double *__restrict__ x, double a, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

// alpha = (p.r)/(p.q); x += alpha p; r -= alpha q; rr' += r.r
__global__ void k_fcg_update(double *__restrict__ x, double *__restrict__ r, const double *__restrict__ p,
                             const double *__restrict__ q, int64_t n, const double *pq, const double *pr,
                             double *rr_next, const int *done, int *err)
{
    __shared__ double sh[32];
    if (*done) return;
    const double den = *pq;
    if (!(den > 0.0)) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    const double alpha = *pr / den;
    double c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        c += ri * ri;
    }
    c = block_sum_d(c, sh);
    if (threadIdx.x == 0) atomicAdd(rr_next, c);
}

__global__ void k_fcg_check(const double *rr, double thr, int it, int *done, const int *err)
{
    if (!*done && !*err && *rr <= thr) *done = it;
}

// beta = -(z.q)/(p.q); p = z + beta p; pr' += p.r
__global__ void k_fcg_pupdate(double *__restrict__ p, const double *__restrict__ z, const double *__restrict__ r,
                              int64_t n, const double *zq, const double *pq, double *pr_next, const int *done,
                              const int *err)
{
    __shared__ double sh[32];
    if (*done || *err) return;
    const double beta = -*zq / *pq;
    double c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double pi = z[i] + beta * p[i];
        p[i] = pi;
        c += pi * r[i];
    }
    c = block_sum_d(c, sh);
    if (threadIdx.x == 0) atomicAdd(pr_next, c);
}

}  // namespace

// Flexible CG (FCG(1), Notay 2000) with z = M(r) from the network, with
// plain Jacobi-PCG as the fallback when the network stalls or breaks down:
// alpha = p.r / p.Sp, p' = z - (z.Sp / p.Sp) p.  The scalars live on the
// device (one slot per iteration) and the host reads the flags every
// check_every iterations, so the iteration issues no synchronisation.  When
// the recurrence residual meets tol, the true FP64 residual ||b - S x|| is
// computed; if it misses tol, the method restarts from it.
void solve_forward_fcg(sfc_system *s)
{
    sfc_ctx *ctx = s->ctx;
    SFC_REQUIRE(s->mpnn, "no learned preconditioner set (sfc_system_set_mpnn)");
    sfc_mpnn *m = s->mpnn;
    bind(m, s);  // the operator's values may have changed since the last use
    const int64_t N = s->N;
    const auto &o = s->opt;
    const int max_iter = o.max_iter > 0 ? o.max_iter : 20000;
    const int check = o.check_every > 0 ? o.check_every : 8;
    const double tol = o.tol > 0 ? o.tol : 1e-8;
    s->X.alloc(N);
    s->blk64.reserve(6 * N);
    double *b = s->blk64.p, *r = b + N, *z = r + N, *p = z + N, *q = p + N, *t = q + N;
    const int64_t slots = (int64_t)max_iter + 2;
    m->fcg_sc.reserve(4 * slots);
    double *pq = m->fcg_sc.p, *pr = pq + slots, *rr = pr + slots, *zq = rr + slots;
    m->fcg_flags.reserve(2);
    int *done = m->fcg_flags.p, *err = done + 1;
    cudaEvent_t e0, e1;
    SFC_CK(cudaEventCreate(&e0));
    SFC_CK(cudaEventCreate(&e1));
    SFC_CK(cudaEventRecord(e0, ctx->stream));
    SFC_CK(cudaMemsetAsync(m->fcg_sc.p, 0, 4 * slots * sizeof(double), ctx->stream));
    SFC_CK(cudaMemsetAsync(done, 0, 2 * sizeof(int), ctx->stream));
    lifted_rhs(s, b);
    SFC_CK(cudaMemsetAsync(s->X.p, 0, N * 8, ctx->stream));
    SFC_CK(cudaMemcpyAsync(r, b, N * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    const double bb = device_dot(ctx, b, b, N);
    const double thr = tol * tol * bb;
    const unsigned g = grid_for(N, 256, ctx->sm_count * 4);
    auto true_residual = [&]() {  // r = b - S x, returns |r| / |b|
        spmv_op64(s, s->X.p, t);
        k_resid<<<grid_for(N, 256), 256, 0, ctx->stream>>>(b, t, N, r);
        count_launch(ctx);
        return std::sqrt(device_dot(ctx, r, r, N) / bb);
    };
    auto start = [&](int slot) {  // direction from the current residual
        apply(m, r, z);
        SFC_CK(cudaMemcpyAsync(p, z, N * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        spmv_op64_dot(s, p, q, pq + slot, nullptr);
        k_dot_done<<<g, 256, 0, ctx->stream>>>(p, r, N, pr + slot, nullptr);
        count_launch(ctx);
    };
    int it = 0, iters = 0, fallback = 0, mark_it = 0;
    constexpr int kStall = 400;
    double mark_rr = bb;
    bool conv = bb == 0.0;
    double rel = 0.0;
    if (!conv) {
        ProfScope ps(ctx, "fcg_iterations", 0.0);
        start(0);
        for (it = 0; it < max_iter; ++it) {
            k_fcg_update<<<g, 256, 0, ctx->stream>>>(s->X.p, r, p, q, N, pq + it, pr + it, rr + it + 1, done, err);
            k_fcg_check<<<1, 1, 0, ctx->stream>>>(rr + it + 1, thr, it + 1, done, err);
            count_launch(ctx, 2);
            apply(m, r, z);
            k_dot_done<<<g, 256, 0, ctx->stream>>>(z, q, N, zq + it, done);
            k_fcg_pupdate<<<g, 256, 0, ctx->stream>>>(p, z, r, N, zq + it, pq + it, pr + it + 1, done, err);
            count_launch(ctx, 2);
            spmv_op64_dot(s, p, q, pq + it + 1, done);
            if ((it + 1) % check == 0 || it + 1 == max_iter) {
                int hf[2];
                download(ctx, hf, done, 2);
                bool give_up = hf[1] != 0;  // breakdown (p^T S p <= 0)
                if (!give_up && hf[0]) {
                    iters = hf[0];
                    rel = true_residual();
                    if (rel <= tol) {
                        conv = true;
                        break;
                    }
                    // the recurrence drifted: restart from the true residual
                    SFC_CK(cudaMemsetAsync(done, 0, sizeof(int), ctx->stream));
                    if (it + 1 < max_iter) start(it + 1);
                    mark_it = it + 1;
                } else if (!give_up) {
                    // stagnation: no 100-fold reduction of the recurrence
                    // residual^2 (10-fold of the residual) within kStall iterations
                    double rr_now = 0;
                    download(ctx, &rr_now, rr + it + 1, 1);
                    if (rr_now < 0.01 * mark_rr) {
                        mark_rr = rr_now;
                        mark_it = it + 1;
                    } else if (it + 1 - mark_it > kStall) {
                        give_up = true;
                    }
                }
                if (give_up) break;
            }
        }
        if (!conv) {
            // the network failed this system (stagnation, breakdown or the
            // iteration cap): plain FP64 Jacobi-PCG finishes from the current
            // x on the true residual, S d = b - S x, x += d
            iters = std::max(iters, std::min(it + 1, max_iter));
            rel = true_residual();
            if (rel > tol) {
                fallback = 1;
                const PcgStats pr = pcg64_public(s, r, z, tol / rel, max_iter, 32);
                k_axpy<<<g, 256, 0, ctx->stream>>>(s->X.p, z, 1.0, N);
                count_launch(ctx);
                iters += pr.iters;
                rel = true_residual();
            }
            conv = rel <= tol * (1.0 + 1e-9);
        }
    }
    SFC_CK(cudaEventRecord(e1, ctx->stream));
    float ms = 0;
    SFC_CK(cudaEventSynchronize(e1));
    SFC_CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_tc(m);
    s->stats = {};
    s->stats.iterations = iters;
    s->stats.num_rhs = 1;
    s->stats.converged = conv ? 1 : 0;
    s->stats.max_rel_residual = rel;
    s->stats.device_ms = ms;
    s->stats.fallback_columns = fallback;
    if (!conv) fail(SFC_ERR_NOT_CONVERGED, "flexible CG (and the Jacobi-PCG fallback) did not converge within max_iter");
}

}  // namespace sfc

using namespace sfc;

namespace {
int mguard(sfc_ctx *ctx, const std::function<void()> &fn)
{
    try {
        SFC_CK(cudaSetDevice(ctx->device));
        fn();
        return SFC_OK;
    } catch (const Error &e) {
        ctx->err = e.msg;
        if (e.code == SFC_ERR_CUDA) cudaGetLastError();
        return e.code;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return SFC_ERR_BAD_ARG;
    }
}
}  // namespace

extern "C" {

int64_t sfc_mpnn_num_params(void) { return NPARAM; }

int32_t sfc_mpnn_create(sfc_ctx_t *ctx, uint64_t seed, sfc_mpnn_t **out)
{
    if (!ctx || !out) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_mpnn *m = new (std::nothrow) sfc_mpnn();
    if (!m) return SFC_ERR_NO_MEMORY;
    int rc = mguard(ctx, [&] {
        m->ctx = ctx;
        std::vector<float> p(NPARAM, 0.f);
        std::mt19937_64 gen(seed);
        std::normal_distribution<float> nd(0.f, 1.f);
        for (int k = 0; k < 2 * H; ++k) p[OFF_EW + k] = nd(gen) * 0.7f;
        for (int k = 0; k < H; ++k) p[OFF_EB + k] = 0.05f;
        for (int l = 0; l < LAYERS; ++l)
            for (int k = 0; k < H * 2 * H; ++k) p[OFF_L + l * LSZ + k] = nd(gen) * std::sqrt(2.f / (2 * H));
        // decoder starts at zero: the untrained network is exactly Jacobi
        m->params.alloc(NPARAM);
        m->grads.alloc(NPARAM);
        m->adam_m.alloc(NPARAM);
        m->adam_v.alloc(NPARAM);
        m->wbf.alloc(LAYERS * H * 2 * H);
        m->scal.alloc(4);
        upload(ctx, m->params, p.data(), NPARAM);
        SFC_CK(cudaMemsetAsync(m->adam_m.p, 0, NPARAM * 4, ctx->stream));
        SFC_CK(cudaMemsetAsync(m->adam_v.p, 0, NPARAM * 4, ctx->stream));
        refresh_bf16(m);
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    });
    if (rc != SFC_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return SFC_OK;
}

int32_t sfc_mpnn_destroy(sfc_mpnn_t *m)
{
    if (!m) return SFC_OK;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    delete m;
    return SFC_OK;
}

int32_t sfc_mpnn_get_params(const sfc_mpnn_t *m, float *out, int64_t n)
{
    if (!m || !out || n != NPARAM) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] { download(m->ctx, out, m->params.p, NPARAM); });
}

int32_t sfc_mpnn_set_params(sfc_mpnn_t *m, const float *in, int64_t n)
{
    if (!m || !in || n != NPARAM) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] {
        upload(m->ctx, m->params, in, NPARAM);
        refresh_bf16(m);
        SFC_CK(cudaStreamSynchronize(m->ctx->stream));
    });
}

int32_t sfc_mpnn_save(const sfc_mpnn_t *m, const char *path)
{
    if (!m || !path) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] {
        std::vector<float> buf(3 * (size_t)NPARAM);
        download(m->ctx, buf.data(), m->params.p, NPARAM);
        download(m->ctx, buf.data() + NPARAM, m->adam_m.p, NPARAM);
        download(m->ctx, buf.data() + 2 * NPARAM, m->adam_v.p, NPARAM);
        FILE *f = std::fopen(path, "wb");
        SFC_REQUIRE(f, std::string("cannot open ") + path);
        const int64_t hdr[3] = {0x53464d50, NPARAM, m->step};  // "SFMP"
        bool ok = std::fwrite(hdr, sizeof hdr, 1, f) == 1 && std::fwrite(buf.data(), 4, buf.size(), f) == buf.size();
        std::fclose(f);
        SFC_REQUIRE(ok, "checkpoint write failed");
    });
}

int32_t sfc_mpnn_load(sfc_mpnn_t *m, const char *path)
{
    if (!m || !path) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] {
        FILE *f = std::fopen(path, "rb");
        SFC_REQUIRE(f, std::string("cannot open ") + path);
        int64_t hdr[3] = {};
        std::vector<float> buf(3 * (size_t)NPARAM);
        bool ok = std::fread(hdr, sizeof hdr, 1, f) == 1 && hdr[0] == 0x53464d50 && hdr[1] == NPARAM &&
                  std::fread(buf.data(), 4, buf.size(), f) == buf.size();
        std::fclose(f);
        SFC_REQUIRE(ok, "not a checkpoint of this network");
        upload(m->ctx, m->params, buf.data(), NPARAM);
        upload(m->ctx, m->adam_m, buf.data() + NPARAM, NPARAM);
        upload(m->ctx, m->adam_v, buf.data() + 2 * NPARAM, NPARAM);
        m->step = hdr[2];
        refresh_bf16(m);
        SFC_CK(cudaStreamSynchronize(m->ctx->stream));
    });
}

int32_t sfc_mpnn_loss_grad(sfc_mpnn_t *m, sfc_system_t *s, const double *r, const double *e, double *loss,
                           float *grad)
{
    if (!m || !s || !r || !e) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] {
        bind(m, s);
        DBuf<double> dr, de;
        upload(m->ctx, dr, r, s->N);
        upload(m->ctx, de, e, s->N);
        SFC_CK(cudaMemsetAsync(m->grads.p, 0, NPARAM * 4, m->ctx->stream));
        const double l = loss_grad(m, dr.p, de.p, 1.0);
        if (loss) *loss = l;
        if (grad) download(m->ctx, grad, m->grads.p, NPARAM);
    });
}

int32_t sfc_mpnn_apply(sfc_mpnn_t *m, sfc_system_t *s, const double *r, double *z)
{
    if (!m || !s || !r || !z) return SFC_ERR_BAD_ARG;
    return mguard(m->ctx, [&] {
        bind(m, s);
        DBuf<double> dr, dz;
        upload(m->ctx, dr, r, s->N);
        dz.alloc(s->N);
        apply(m, dr.p, dz.p);
        download(m->ctx, z, dz.p, s->N);
        check_tc(m);
    });
}

int32_t sfc_mpnn_default_train_options(sfc_mpnn_train_options_t *o)
{
    if (!o) return SFC_ERR_BAD_ARG;
    o->steps = 500;
    o->batch = 4;
    o->max_pairs = 16;
    o->normalize = 1;
    o->lr = 1e-3;
    o->pair_floor = 1e-6;
    o->seed = 0;
    return SFC_OK;
}

int32_t sfc_mpnn_train(sfc_mpnn_t *m, sfc_system_t *s, const sfc_mpnn_train_options_t *o, double *loss_history)
{
    if (!m || !s || !o || o->steps < 0 || o->batch < 1 || o->max_pairs < 1 || o->max_pairs > 64 || !(o->lr > 0) ||
        !(o->pair_floor > 0 && o->pair_floor < 1)) {
        if (m) m->ctx->err = "invalid training options";
        return SFC_ERR_BAD_ARG;
    }
    return mguard(m->ctx, [&] {
        bind(m, s);
        make_pairs(m, s, o->max_pairs, o->pair_floor, o->normalize != 0);
        const int64_t N = s->N;
        std::mt19937_64 gen(o->seed ^ (uint64_t)(m->step * 0x9E3779B97F4A7C15ull));
        std::uniform_int_distribution<int> pick(0, m->npairs - 1);
        for (int t = 0; t < o->steps; ++t) {
            SFC_CK(cudaMemsetAsync(m->grads.p, 0, NPARAM * 4, m->ctx->stream));
            double acc = 0;
            for (int j = 0; j < o->batch; ++j) {
                const int k = pick(gen);
                acc += loss_grad(m, m->pr.p + k * N, m->pe.p + k * N, m->pw[k] / o->batch);
            }
            adam_step(m, o->lr);
            if (loss_history) loss_history[t] = acc;
        }
        SFC_CK(cudaStreamSynchronize(m->ctx->stream));
    });
}

int32_t sfc_system_set_mpnn(sfc_system_t *s, sfc_mpnn_t *m)
{
    if (!s) return SFC_ERR_BAD_ARG;
    s->mpnn = m;
    if (m) m->op_sys = nullptr;  // rebind on next use
    return SFC_OK;
}

}  // extern "C"
