// Block SpMM Q = S P for 3-dof meshes on a structured node lattice
// (trilinear hexahedra on an nx x ny x nz grid, nodes numbered x fastest):
// the FP32 product at the heart of the mixed block PCG, replacing the sparse
// direct solve of corlib/SystemSolveEigenSparse.hpp:273-404 for the many
// adjoint right-hand sides of statX/infer/ForwardGaussRHS.hpp:104-112.
//
// S is held as each node's 27 neighbour blocks in canonical slots
// (dz, dy, dx) (zero where the lattice has no neighbour), rows padded to four
// floats so a warp reads a block with three 16-byte broadcast loads.  P and Q
// are the block solver's RHS-interleaved [N][K] FP32 arrays.  Two products
// use this view: the streamed x-line kernel k_xspmm32 (the default; described
// at the kernel) and the TMA-staged brick kernel k_lspmm32 below
// (SFC_SPMM=lattice).
//
// Staged bricks.  A work item is a brick of 4 x 2 x 2 output nodes and a
// 64-column slice of the block.  One elected thread issues a single 5-D TMA
// tensor load of the brick's halo (6 x 4 x 4 column nodes x 3 rows x 64
// columns, zero-filled outside the lattice: 72 KiB) and 1-D bulk copies of
// the brick's block rows (up to 4 x 5 KiB) into shared memory, completing on
// one mbarrier.  Each x-line of four output nodes belongs to two warps (32
// columns each, one per lane): for every column node of its 3 x 3 neighbour
// lines a warp reads the node's three P rows from shared memory once and
// applies them to every output node of the line that couples to it (up to
// three), so a P row read feeds 1.8 outputs on average.  Measured, the shared-memory load path bounds
// it: both warps of an x-line load the same block values for their two
// columns per lane.  The p.q column dots are accumulated in FP64 per lane
// across all of a CTA's work items and reduced once at the end.
//
// Two CTAs share an SM (94.5 KiB of shared memory each); each x-line is
// split over two warps by columns (8 warps per CTA) for latency hiding
// (SFC_LATTICE_WARPS=4 keeps one warp per x-line).  Waits on the mbarrier
// are bounded: a wait that gives up sets lat_err (the solver then fails with
// SFC_ERR_TIMEOUT), waits once more (bounded) for the copies in flight and
// leaves the kernel.  No multicast, no clusters: every copy reads this
// GPU's own memory.

#include <cudaTypedefs.h>

#include <cstdlib>

#include "common.cuh"

namespace sfc {
namespace {

constexpr int BX = 4, BY = 2, BZ = 2;  // output nodes per brick
constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2;
constexpr int CS = 64;                 // columns per slice (2 per lane)
constexpr int SLOT = 12;               // floats per padded 3x3 block
constexpr int NODE_FLOATS = 27 * SLOT; // 324 floats = 1296 bytes per node
constexpr int HALO_FLOATS = HZ * HY * HX * 3 * CS;
constexpr int BLK_FLOATS = BX * BY * BZ * NODE_FLOATS;
constexpr int HALO_BYTES = HALO_FLOATS * 4;                 // 73,728
constexpr size_t SMEM_BYTES = (size_t)(HALO_FLOATS + BLK_FLOATS) * 4 + 16;  // 94,480: + mbarrier
constexpr uint32_t WAIT_TRIES = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t i = 0; i < WAIT_TRIES; ++i) {
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

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1, int c2,
                                            int c3, int c4)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
                 : "memory");
}

struct Brick {
    int x0, y0, z0, nvx;
};

__device__ __forceinline__ Brick brick_of(int64_t w, int slices, int tx_n, int ty_n, int nx)
{
    const int64_t t = w / slices;
    const int tx = (int)(t % tx_n);
    const int64_t tr = t / tx_n;
    Brick b;
    b.x0 = tx * BX;
    b.y0 = (int)(tr % ty_n) * BY;
    b.z0 = (int)(tr / ty_n) * BZ;
    b.nvx = min(BX, nx - b.x0);
    return b;
}

// one thread: the brick's halo (one 5-D tensor copy) and its block rows (one
// bulk copy per x-line inside the lattice), all completing on `bar`
__device__ __forceinline__ void issue_brick(const CUtensorMap *pmap, const float *__restrict__ bq, float *halo,
                                            float *blk, uint32_t bar, const Brick &b, int slice, int nx, int ny,
                                            int nz)
{
    uint32_t bytes = HALO_BYTES;
    for (int l = 0; l < BY * BZ; ++l)
        if (b.y0 + (l & 1) < ny && b.z0 + (l >> 1) < nz) bytes += (uint32_t)b.nvx * NODE_FLOATS * 4;
    mbar_expect_tx(bar, bytes);
    tma_load_5d(smem_u32(halo), pmap, bar, slice * CS, 0, b.x0 - 1, b.y0 - 1, b.z0 - 1);
    for (int l = 0; l < BY * BZ; ++l) {
        const int y = b.y0 + (l & 1), z = b.z0 + (l >> 1);
        if (y >= ny || z >= nz) continue;
        const int64_t node = ((int64_t)z * ny + y) * nx + b.x0;
        bulk_load(smem_u32(blk + l * BX * NODE_FLOATS), bq + node * NODE_FLOATS, (uint32_t)b.nvx * NODE_FLOATS * 4,
                  bar);
    }
}

// H column groups per x-line: 4 H warps, warp (xl, g) owns x-line xl (wy =
// xl & 1, wz = xl >> 1) and V = 2 / H columns per lane of the slice's group g.
// Two CTAs per SM (94.5 KiB of shared memory each).
template <int H>
__global__ void __launch_bounds__(128 * H, 2)
    k_lspmm32(const __grid_constant__ CUtensorMap pmap, const float *__restrict__ bq, float *__restrict__ Q, int nx,
              int ny, int nz, int K, int slices, int64_t work, double *pq, const int *stop, int *err)
{
    constexpr int V = 2 / H, GC = CS / H;  // columns per lane, per group
    if (*stop) return;
    extern __shared__ __align__(128) unsigned char smem[];
    float *halo = reinterpret_cast<float *>(smem);
    float *blk = halo + HALO_FLOATS;
    uint64_t *barp = reinterpret_cast<uint64_t *>(blk + BLK_FLOATS);
    const uint32_t bar = smem_u32(barp);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int xl = warp & 3, grp = warp >> 2;
    const int wy = xl & 1, wz = xl >> 1;
    const int col = grp * GC + lane * V;  // first column of this lane within the slice
    const int tx_n = (nx + BX - 1) / BX, ty_n = (ny + BY - 1) / BY;
    const int slice = (int)(blockIdx.x % slices);  // gridDim.x is a multiple of slices
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    uint32_t parity = 0;
    for (int64_t w = blockIdx.x; w < work; w += gridDim.x) {
        const Brick b = brick_of(w, slices, tx_n, ty_n, nx);
        if (threadIdx.x == 0) issue_brick(&pmap, bq, halo, blk, bar, b, slice, nx, ny, nz);
        const bool got = mbar_wait(bar, parity);
        if (__syncthreads_or(!got)) {
            // the copies did not complete in time: record it, give the copies
            // in flight one more bounded wait, and leave (uniformly)
            if (threadIdx.x == 0) atomicExch(err, 1);
            mbar_wait(bar, parity);
            return;
        }
        parity ^= 1u;
        float acc[BX][3][V];
#pragma unroll
        for (int o = 0; o < BX; ++o)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) acc[o][r][v] = 0.f;
        const float *hb = halo + col;
        const float *bb = blk + xl * BX * NODE_FLOATS;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy) {
                const float *line = hb + ((wz + dz) * HY + (wy + dy)) * HX * 3 * CS;
#pragma unroll
                for (int cx = 0; cx < HX; ++cx) {
                    float p[3][V];
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        if constexpr (V == 2) {
                            const float2 t = *reinterpret_cast<const float2 *>(line + (cx * 3 + r) * CS);
                            p[r][0] = t.x;
                            p[r][1] = t.y;
                        } else {
                            p[r][0] = line[(cx * 3 + r) * CS];
                        }
                    }
#pragma unroll
                    for (int ox = 0; ox < BX; ++ox) {
                        const int dx = cx - ox;  // lattice offset dx - 1
                        if (dx < 0 || dx > 2) continue;
                        const float *bp = bb + ox * NODE_FLOATS + (dz * 9 + dy * 3 + dx) * SLOT;
                        const float4 bm[3] = {*reinterpret_cast<const float4 *>(bp),
                                              *reinterpret_cast<const float4 *>(bp + 4),
                                              *reinterpret_cast<const float4 *>(bp + 8)};
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int v = 0; v < V; ++v)
                                acc[ox][r][v] =
                                    fmaf(bm[r].z, p[2][v], fmaf(bm[r].y, p[1][v], fmaf(bm[r].x, p[0][v], acc[ox][r][v])));
                    }
                }
            }
        const int y = b.y0 + wy, z = b.z0 + wz;
        if (y < ny && z < nz) {
            // own rows of P sit at halo (ox + 1, wy + 1, wz + 1)
            const float *own = hb + ((wz + 1) * HY + (wy + 1)) * HX * 3 * CS;
#pragma unroll
            for (int ox = 0; ox < BX; ++ox) {
                if (ox >= b.nvx) break;
                const int64_t node = ((int64_t)z * ny + y) * nx + b.x0 + ox;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    float *q = Q + (3 * node + r) * K + slice * CS + col;
                    const float *pv = own + ((ox + 1) * 3 + r) * CS;
                    if constexpr (V == 2)
                        *reinterpret_cast<float2 *>(q) = make_float2(acc[ox][r][0], acc[ox][r][1]);
                    else
                        *q = acc[ox][r][0];
#pragma unroll
                    for (int v = 0; v < V; ++v) dacc[v] += (double)pv[v] * (double)acc[ox][r][v];
                }
            }
        }
        __syncthreads();  // every warp is done with the staged tiles before the next copies land
    }
    // column dots: red[xl][c], the four x-lines' partials of slice column c
    double *red = reinterpret_cast<double *>(smem);
#pragma unroll
    for (int v = 0; v < V; ++v) red[xl * CS + col + v] = dacc[v];
    __syncthreads();
    if (threadIdx.x < CS) {
        const double sum = red[threadIdx.x] + red[CS + threadIdx.x] + red[2 * CS + threadIdx.x] + red[3 * CS + threadIdx.x];
        atomicAdd(pq + slice * CS + threadIdx.x, sum);
    }
}

// canonical 27-slot blocks (FP32 or FP64) from the node-block (BSR) view; a
// block whose column node is not a lattice neighbour sets *err
template <typename T>
__global__ void k_lattice_fill(const int32_t *__restrict__ bptr, const int32_t *__restrict__ bcol,
                               const T *__restrict__ b32, int64_t nodes, int nx, int ny, T *__restrict__ bq,
                               int *err)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t plane = (int64_t)nx * ny;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nodes; i += warps) {
        const int32_t b0 = bptr[i], nb = bptr[i + 1] - b0;
        const int xi = (int)(i % nx), yi = (int)((i / nx) % ny), zi = (int)(i / plane);
        for (int32_t e = lane; e < 9 * nb; e += 32) {
            const int32_t t = e / 9, k = e % 9;
            const int64_t j = bcol[b0 + t];
            const int dx = (int)(j % nx) - xi, dy = (int)((j / nx) % ny) - yi, dz = (int)(j / plane) - zi;
            if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) {
                atomicExch(err, 1);
                continue;
            }
            const int slot = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
            bq[i * NODE_FLOATS + slot * SLOT + (k / 3) * 4 + k % 3] = b32[(int64_t)(b0 + t) * 9 + k];
        }
    }
}

// Streamed lattice product (the default on lattices): one warp per
// contiguous run of output nodes (numbered x fastest, so a run is a few x-line
// segments), all K = 32 V columns of the block, V per lane.  The warp walks
// each segment's column positions cx along x; at each it loads the P rows of
// the nine neighbour lines (y + dy, z + dz) once and applies them to the
// three output nodes cx - 1, cx, cx + 1 that couple to them, keeping a
// sliding window of three output nodes' accumulators in registers.  Output
// cx - 1 then has all its columns and is stored.  Every P row read from L1
// therefore feeds three outputs (against one in the node-block kernel), and a
// block's nine values (three 16-byte shared loads, the same address in every
// lane) feed 9 V FMAs per lane.
//
// Each block is read exactly once, so a load of it from global memory would
// miss L1 and stall the FMAs that follow it.  Every output node's 27 blocks
// (1296 bytes) are instead copied by cp.async into a per-warp ring of four
// rows in shared memory one position before their first use (the three rows
// in use and the one in flight), and the FMAs read them there.  Neighbour
// lines outside the lattice are clamped to a line inside it: their blocks are
// zero, so they add nothing; outputs outside the segment are computed from
// stale ring rows and never stored.  p.q column dots in FP64.
constexpr int XR = 4;  // block ring rows per warp

template <int V>
constexpr size_t xsmem()
{
    return (size_t)8 * 32 * V * sizeof(double) + (size_t)8 * XR * NODE_FLOATS * sizeof(float);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int V>
__global__ void __launch_bounds__(256, 2)
    k_xspmm32(const float *__restrict__ bq, const float *__restrict__ P, float *__restrict__ Q, int nx, int ny,
              int nz, int64_t nodes, int64_t per_warp, double *pq, const int *stop)
{
    constexpr int K = 32 * V;
    constexpr int64_t RS = 3 * (int64_t)K;  // floats per node of P and Q
    extern __shared__ __align__(16) unsigned char xs[];
    double *sh = reinterpret_cast<double *>(xs);
    if (*stop) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *ring = reinterpret_cast<float *>(xs + 8 * K * sizeof(double)) + warp * XR * NODE_FLOATS;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    const int64_t end = min(nodes, (gw + 1) * per_warp);
    const int64_t row = (int64_t)nx * RS;
    for (int64_t a = gw * per_warp; a < end;) {
        const int64_t line = a / nx;
        const int x0 = (int)(a - line * nx);
        const int x1 = (int)(min(end, (line + 1) * nx) - 1 - line * nx);
        const int y = (int)(line % ny), z = (int)(line / ny);
        // the nine neighbour lines (index z * ny + y), clamped into the lattice
        int nl[9];
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
                nl[dz * 3 + dy] = min(max(z + dz - 1, 0), nz - 1) * ny + min(max(y + dy - 1, 0), ny - 1);
        const float *pb = P + lane * V;
        const float *bl = bq + line * nx * NODE_FLOATS;
        const float *own = P + line * row + lane * V;
        float *ql = Q + line * row + lane * V;
        const int c0 = max(0, x0 - 1), c1 = min(nx - 1, x1 + 1);
        // output ox's blocks into ring row ox % XR (nothing outside the segment)
        auto fetch = [&](int ox) {
            if (ox < x0 || ox > x1) return;
            const float4 *src = reinterpret_cast<const float4 *>(bl + (int64_t)ox * NODE_FLOATS);
            float4 *dst = reinterpret_cast<float4 *>(ring + (ox % XR) * NODE_FLOATS);
            for (int t = lane; t < NODE_FLOATS / 4; t += 32) cp_async16(dst + t, src + t);
        };
        // every lane is done with the previous segment's ring; the outputs
        // that the first position needs
        __syncwarp();
        for (int ox = x0; ox <= c0 + 1; ++ox) fetch(ox);
        cp_async_commit();
        float acc[3][3][V];
#pragma unroll
        for (int o = 0; o < 3; ++o)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) acc[o][r][v] = 0.f;
        for (int cx = c0; cx <= c1; ++cx) {
            // outputs up to cx + 1 have landed; then the copy for output cx + 2
            // (into the row of output cx - 2, which no lane reads any more)
            cp_async_wait_all();
            __syncwarp();
            fetch(cx + 2);
            cp_async_commit();
#pragma unroll
            for (int l = 0; l < 9; ++l) {
                const float *pj = pb + ((int64_t)nl[l] * nx + cx) * RS;
                float p[3][V];
                ldv<V>(pj, p[0]);
                ldv<V>(pj + K, p[1]);
                ldv<V>(pj + 2 * K, p[2]);
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    // output cx - 1 + o couples to column cx at dx = 1 - o (slot 2 - o)
                    const int slot = (cx - 1 + o + XR) % XR;  // cx - 1 + o >= -1
                    const float4 *bp =
                        reinterpret_cast<const float4 *>(ring + slot * NODE_FLOATS + (l * 3 + 2 - o) * SLOT);
                    const float4 m[3] = {bp[0], bp[1], bp[2]};
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int v = 0; v < V; ++v)
                            acc[o][r][v] = fmaf(m[r].z, p[2][v], fmaf(m[r].y, p[1][v], fmaf(m[r].x, p[0][v], acc[o][r][v])));
                }
            }
            // output cx - 1 has all three of its column positions
            if (cx - 1 >= x0) {
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const int64_t off = (int64_t)(cx - 1) * RS + r * K;
                    stv<V>(ql + off, acc[0][r]);
                    float pv[V];
                    ldv<V>(own + off, pv);
#pragma unroll
                    for (int v = 0; v < V; ++v) dacc[v] += (double)pv[v] * (double)acc[0][r][v];
                }
            }
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    acc[0][r][v] = acc[1][r][v];
                    acc[1][r][v] = acc[2][r][v];
                    acc[2][r][v] = 0.f;
                }
        }
        if (c1 == x1) {
            // the segment ends on the lattice face: its last output is in slot 0
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int64_t off = (int64_t)x1 * RS + r * K;
                stv<V>(ql + off, acc[0][r]);
                float pv[V];
                ldv<V>(own + off, pv);
#pragma unroll
                for (int v = 0; v < V; ++v) dacc[v] += (double)pv[v] * (double)acc[0][r][v];
            }
        }
        a = line * nx + x1 + 1;
    }
    cp_async_wait_all();  // no copy outlives the kernel (they are all empty by now)
    block_cols_add<V>(dacc, sh, pq);
}

// R = B - S X in FP64 on the lattice view (the true residual of the mixed
// block solver's reliable updates; rr[c] += sum R^2 per column): the same
// streamed x-line walk as k_xspmm32 over FP64 canonical blocks (12 doubles
// per 3x3 block, rows padded to four), each run of output nodes split over H
// warps by columns (V doubles per lane) so that the FP64 accumulators fit two
// CTAs per SM; the blocks of output cx + 2 are copied by cp.async into the
// warp's ring while position cx is computed.
template <int V, int H>
constexpr size_t xrsmem()
{
    return (size_t)8 * 32 * V * H * sizeof(double) + (size_t)8 * XR * NODE_FLOATS * sizeof(double);
}

template <int V, int H>
__global__ void __launch_bounds__(256, 2)
    k_xresid64(const double *__restrict__ bq, const double *__restrict__ X, const double *__restrict__ B,
               double *__restrict__ R, int nx, int ny, int nz, int64_t nodes, int64_t per_run, double *rr)
{
    constexpr int K = 32 * V * H;
    constexpr int64_t RS = 3 * (int64_t)K;  // doubles per node of X, B and R
    extern __shared__ __align__(16) unsigned char xs[];
    double *sh = reinterpret_cast<double *>(xs);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int colv = (warp % H) * 32 * V + lane * V;  // first column of this lane
    double *ring = reinterpret_cast<double *>(xs + 8 * K * sizeof(double)) + warp * XR * NODE_FLOATS;
    const int64_t run = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) / H;
    double dacc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dacc[v] = 0.0;
    const int64_t row = (int64_t)nx * RS;
    // chunks of per_run nodes, run r taking chunks r, r + nruns, ...: the
    // chunks in flight at one time are a contiguous band of x-lines, so the
    // nine neighbour lines of a line are mostly read while L2 still holds them
    const int64_t nruns = (int64_t)gridDim.x * (8 / H);
    for (int64_t chunk = run; chunk * per_run < nodes; chunk += nruns)
    for (int64_t a = chunk * per_run, end = min(nodes, (chunk + 1) * per_run); a < end;) {
        const int64_t line = a / nx;
        const int x0 = (int)(a - line * nx);
        const int x1 = (int)(min(end, (line + 1) * nx) - 1 - line * nx);
        const int y = (int)(line % ny), z = (int)(line / ny);
        int nl[9];
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
                nl[dz * 3 + dy] = min(max(z + dz - 1, 0), nz - 1) * ny + min(max(y + dy - 1, 0), ny - 1);
        const double *xb = X + colv;
        const double *bl = bq + line * nx * NODE_FLOATS;
        const int64_t own = line * row + colv;
        const int c0 = max(0, x0 - 1), c1 = min(nx - 1, x1 + 1);
        auto fetch = [&](int ox) {
            if (ox < x0 || ox > x1) return;
            const double2 *src = reinterpret_cast<const double2 *>(bl + (int64_t)ox * NODE_FLOATS);
            double2 *dst = reinterpret_cast<double2 *>(ring + (ox % XR) * NODE_FLOATS);
            for (int t = lane; t < NODE_FLOATS / 2; t += 32) cp_async16(dst + t, src + t);
        };
        auto store = [&](int ox, const double (&acc)[3][V]) {
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int64_t off = own + (int64_t)ox * RS + r * K;
                double bv[V];
                ldv64<V>(B + off, bv);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const double rv = bv[v] - acc[r][v];
                    R[off + v] = rv;
                    dacc[v] += rv * rv;
                }
            }
        };
        __syncwarp();
        for (int ox = x0; ox <= c0 + 1; ++ox) fetch(ox);
        cp_async_commit();
        double acc[3][3][V];
#pragma unroll
        for (int o = 0; o < 3; ++o)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) acc[o][r][v] = 0.0;
        for (int cx = c0; cx <= c1; ++cx) {
            cp_async_wait_all();
            __syncwarp();
            fetch(cx + 2);
            cp_async_commit();
#pragma unroll
            for (int l = 0; l < 9; ++l) {
                const double *xj = xb + ((int64_t)nl[l] * nx + cx) * RS;
                double p[3][V];
                ldv64<V>(xj, p[0]);
                ldv64<V>(xj + K, p[1]);
                ldv64<V>(xj + 2 * K, p[2]);
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    const int slot = (cx - 1 + o + XR) % XR;
                    const double *bp = ring + slot * NODE_FLOATS + (l * 3 + 2 - o) * SLOT;
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        const double2 m01 = *reinterpret_cast<const double2 *>(bp + 4 * r);
                        const double m2 = bp[4 * r + 2];
#pragma unroll
                        for (int v = 0; v < V; ++v)
                            acc[o][r][v] = fma(m2, p[2][v], fma(m01.y, p[1][v], fma(m01.x, p[0][v], acc[o][r][v])));
                    }
                }
            }
            if (cx - 1 >= x0) store(cx - 1, acc[0]);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    acc[0][r][v] = acc[1][r][v];
                    acc[1][r][v] = acc[2][r][v];
                    acc[2][r][v] = 0.0;
                }
        }
        if (c1 == x1) store(x1, acc[0]);
        a = line * nx + x1 + 1;
    }
    cp_async_wait_all();
    // the 8 / H runs' partials of column c sit at sh[run][c]
#pragma unroll
    for (int v = 0; v < V; ++v) sh[(warp / H) * K + colv + v] = dacc[v];
    __syncthreads();
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        double sum = 0;
        for (int j = 0; j < 8 / H; ++j) sum += sh[j * K + c];
        atomicAdd(rr + c, sum);
    }
}

int g_occ = 0;     // resident CTAs per SM of the k_lspmm32 instantiation in use
int g_groups = 0;  // column groups per x-line: 2 (8 warps per CTA) or 1 (SFC_LATTICE_WARPS=4)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        SFC_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(SFC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

}  // namespace

// Installs the lattice view when the system's pattern comes from a 3-dof
// mesh whose nodes form a lattice (numbered x fastest) and every block couples
// lattice neighbours, and picks the product that uses it: the streamed
// x-line kernel by default, the TMA-staged brick kernel with SFC_SPMM=lattice
// in the environment.  SFC_SPMM=bsr, and every other mesh, keep the
// node-block (BSR) kernels.
void build_lattice_blocks(sfc_system *s)
{
    sfc_ctx *ctx = s->ctx;
    s->has_lattice = false;
    s->lat_mode = 0;
    const sfc_mesh *m = s->pattern_mesh;
    const char *e = std::getenv("SFC_SPMM");
    const std::string want = e ? e : "";
    if (want == "bsr") return;
    if (!s->has_bsr || !m || !m->is_grid || m->dim != 3 || m->dof != 3) return;
    const int nx = m->gn[0], ny = m->gn[1], nz = m->gn[2];
    if ((int64_t)nx * ny * nz != s->nodes || nx < 2 || ny < 2 || nz < 2) return;
    s->bq.alloc((size_t)s->nodes * NODE_FLOATS);  // same size on every rebuild: no reallocation
    if (!s->lat_err.p) {
        s->lat_err.alloc(1);
        SFC_CK(cudaMemsetAsync(s->lat_err.p, 0, sizeof(int), ctx->stream));
    }
    s->pmap_ptr = nullptr;  // the lattice may differ from the one the cached map was made for
    SFC_CK(cudaMemsetAsync(s->bq.p, 0, (size_t)s->nodes * NODE_FLOATS * 4, ctx->stream));
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    k_lattice_fill<float><<<grid_for(s->nodes * 32, 256), 256, 0, ctx->stream>>>(s->bptr.p, s->bcol.p, s->bval32.p,
                                                                              s->nodes, nx, ny, s->bq.p, err.p);
    // the FP64 view for the true residual (k_xresid64)
    s->bq64.alloc((size_t)s->nodes * NODE_FLOATS);
    SFC_CK(cudaMemsetAsync(s->bq64.p, 0, (size_t)s->nodes * NODE_FLOATS * 8, ctx->stream));
    k_lattice_fill<double><<<grid_for(s->nodes * 32, 256), 256, 0, ctx->stream>>>(s->bptr.p, s->bcol.p, s->bval64.p,
                                                                               s->nodes, nx, ny, s->bq64.p, err.p);
    count_launch(ctx, 2);
    int h = 0;
    download(ctx, &h, err.p, 1);
    if (h) return;
    s->lat[0] = nx;
    s->lat[1] = ny;
    s->lat[2] = nz;
    s->has_lattice = true;
    s->lat_mode = want == "lattice" ? 1 : 2;
}

// the tensor map of P and the kernel's attributes, set up outside any
// stream capture
void lattice_prepare(sfc_system *s, const float *P, int K)
{
    const int nx = s->lat[0], ny = s->lat[1], nz = s->lat[2];
    SFC_REQUIRE(K % CS == 0, "lattice SpMM needs a multiple of 64 columns");
    if (s->pmap_ptr != P || s->pmap_K != K) {
        const cuuint64_t dims[5] = {(cuuint64_t)K, 3, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
        const cuuint64_t strides[4] = {(cuuint64_t)K * 4, (cuuint64_t)3 * K * 4, (cuuint64_t)3 * K * 4 * nx,
                                       (cuuint64_t)3 * K * 4 * nx * ny};
        const cuuint32_t box[5] = {CS, 3, HX, HY, HZ};
        const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
        const CUresult r = encode_fn()(&s->pmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<float *>(P), dims,
                                       strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) fail(SFC_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
        s->pmap_ptr = P;
        s->pmap_K = K;
    }
    if (!g_groups) {
        const char *e = std::getenv("SFC_LATTICE_WARPS");
        g_groups = (e && std::string(e) == "4") ? 1 : 2;
        if (g_groups == 2) {
            SFC_CK(cudaFuncSetAttribute(k_lspmm32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
            SFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ, k_lspmm32<2>, 256, SMEM_BYTES));
        } else {
            SFC_CK(cudaFuncSetAttribute(k_lspmm32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
            SFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ, k_lspmm32<1>, 128, SMEM_BYTES));
        }
        if (g_occ < 1) g_occ = 1;
    }
}

void lattice_spmm32(sfc_system *s, const float *P, float *Q, int K, double *pq, const int *stop)
{
    sfc_ctx *ctx = s->ctx;
    const int nx = s->lat[0], ny = s->lat[1], nz = s->lat[2];
    lattice_prepare(s, P, K);
    const int occ = g_occ;
    const int slices = K / CS;
    const int64_t tiles = (int64_t)((nx + BX - 1) / BX) * ((ny + BY - 1) / BY) * ((nz + BZ - 1) / BZ);
    const int64_t work = tiles * slices;
    int64_t grid = std::min<int64_t>(work, (int64_t)occ * ctx->sm_count);
    grid = std::max<int64_t>(slices, grid - grid % slices);
    if (g_groups == 2)
        k_lspmm32<2><<<(unsigned)grid, 256, SMEM_BYTES, ctx->stream>>>(s->pmap, s->bq.p, Q, nx, ny, nz, K, slices,
                                                                       work, pq, stop, s->lat_err.p);
    else
        k_lspmm32<1><<<(unsigned)grid, 128, SMEM_BYTES, ctx->stream>>>(s->pmap, s->bq.p, Q, nx, ny, nz, K, slices,
                                                                       work, pq, stop, s->lat_err.p);
    count_launch(ctx);
}

// the streamed x-line product (k_xspmm32): contiguous runs of output nodes,
// one per warp, of equal length, over every resident warp of the GPU
template <int V>
int xline_occ()
{
    static int occ = 0;
    if (!occ) {
        SFC_CK(cudaFuncSetAttribute(k_xspmm32<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsmem<V>()));
        SFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xspmm32<V>, 256, xsmem<V>()));
        if (occ < 1) occ = 1;
    }
    return occ;
}

template <int V>
void xline_launch(sfc_system *s, const float *P, float *Q, double *pq, const int *stop)
{
    sfc_ctx *ctx = s->ctx;
    const int64_t warps = (int64_t)xline_occ<V>() * ctx->sm_count * 8;
    const int64_t per_warp = (s->nodes + warps - 1) / warps;
    const unsigned grid = (unsigned)((s->nodes + per_warp * 8 - 1) / (per_warp * 8));
    k_xspmm32<V><<<grid, 256, xsmem<V>(), ctx->stream>>>(s->bq.p, P, Q, s->lat[0], s->lat[1], s->lat[2], s->nodes,
                                                           per_warp, pq, stop);
    count_launch(ctx);
}

// kernel attributes of the streamed product for K columns, set up outside any
// stream capture
void xline_prepare(int K)
{
    if (K == 32) xline_occ<1>();
    else if (K == 64) xline_occ<2>();
    else if (K == 128) xline_occ<4>();
}

void xline_spmm32(sfc_system *s, const float *P, float *Q, int K, double *pq, const int *stop)
{
    SFC_REQUIRE(K == 32 || K == 64 || K == 128, "streamed lattice SpMM needs 32, 64 or 128 columns");
    if (K == 32) xline_launch<1>(s, P, Q, pq, stop);
    else if (K == 64) xline_launch<2>(s, P, Q, pq, stop);
    else xline_launch<4>(s, P, Q, pq, stop);
}

// the FP64 residual on the lattice view (k_xresid64): K = 128 as two
// 64-column warps per run, K = 64 and 32 as one warp
template <int V, int H>
int xresid_occ()
{
    static int occ = 0;
    if (!occ) {
        SFC_CK(cudaFuncSetAttribute(k_xresid64<V, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)xrsmem<V, H>()));
        SFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xresid64<V, H>, 256, xrsmem<V, H>()));
        if (occ < 1) occ = 1;
    }
    return occ;
}

template <int V, int H>
void xresid_launch(sfc_system *s, const double *X, const double *B, double *R, double *rr)
{
    sfc_ctx *ctx = s->ctx;
    // Chunks of nx .. nx + 2 nodes (about one x-line), dealt round-robin to
    // at most the resident runs, every run taking the same number of chunks:
    // the y and z neighbours of a node then lie in chunks that other runs
    // walk at nearly the same time, so the nine reads of an X row come close
    // together and mostly from L2.  (With the node range split evenly over
    // the resident runs, each run walked more than one line, and a row's
    // y neighbour was read by the same run one line later, after the FP64
    // rows in flight had outgrown L2: 2.6x the algorithmic DRAM bytes.)
    const int64_t cap = (int64_t)xresid_occ<V, H>() * ctx->sm_count * (8 / H);
    const int64_t nx = s->lat[0], nodes = s->nodes;
    int64_t per_run = nx, nrun = 0;
    for (int64_t len = nx; len <= nx + 2; ++len) {
        const int64_t passes = (nodes + cap * len - 1) / (cap * len);
        const int64_t r = (nodes + passes * len - 1) / (passes * len);
        if (r > nrun) {
            nrun = r;
            per_run = len;
        }
    }
    const unsigned grid = (unsigned)((nrun + (8 / H) - 1) / (8 / H));
    k_xresid64<V, H><<<grid, 256, xrsmem<V, H>(), ctx->stream>>>(s->bq64.p, X, B, R, s->lat[0], s->lat[1], s->lat[2],
                                                                   s->nodes, per_run, rr);
    count_launch(ctx);
}

void xresid_prepare(int K)
{
    if (K == 32) xresid_occ<1, 1>();
    else if (K == 64) xresid_occ<2, 1>();
    else if (K == 128) xresid_occ<2, 2>();
}

void xline_resid64(sfc_system *s, const double *X, const double *B, double *R, int K, double *rr)
{
    SFC_REQUIRE(K == 32 || K == 64 || K == 128, "lattice residual needs 32, 64 or 128 columns");
    if (K == 32) xresid_launch<1, 1>(s, X, B, R, rr);
    else if (K == 64) xresid_launch<2, 1>(s, X, B, R, rr);
    else xresid_launch<2, 2>(s, X, B, R, rr);
}

// after a solve: a staged SpMM whose bounded wait gave up fails the solve
void lattice_check(sfc_system *s)
{
    if (!s->has_lattice || !s->lat_err.p) return;
    int h = 0;
    download(s->ctx, &h, s->lat_err.p, 1);
    if (h) {
        SFC_CK(cudaMemsetAsync(s->lat_err.p, 0, sizeof(int), s->ctx->stream));
        fail(SFC_ERR_TIMEOUT, "staged SpMM: a bounded wait for its shared-memory copies gave up");
    }
}

}  // namespace sfc
