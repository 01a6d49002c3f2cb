// Internal declarations shared by the CUDA translation units of the statFEM
// B200 library.  Nothing here is part of the C ABI (include/statfem_cuda.h).
#pragma once

#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "statfem_cuda.h"

namespace sfc {

// ---------------------------------------------------------------------------
// errors: internal code throws Error; every C entry point converts it to a
// status code and stores the message on the context.
// ---------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Error{code, msg}; }

#define SFC_CK(call)                                                                   \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            ::sfc::fail(SFC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SFC_REQUIRE(cond, msg)                                                         \
    do {                                                                               \
        if (!(cond)) ::sfc::fail(SFC_ERR_BAD_ARG, msg);                                \
    } while (0)

// A size beyond a fixed limit of the implementation (32-bit index range,
// fixed scratch area): SFC_ERR_TOO_LARGE.
#define SFC_REQUIRE_SIZE(cond, msg)                                                    \
    do {                                                                               \
        if (!(cond)) ::sfc::fail(SFC_ERR_TOO_LARGE, msg);                              \
    } while (0)

// Device buffer with RAII ownership.
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // (re)allocate to exactly `count` elements when the size differs
    void alloc(size_t count)
    {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            fail(SFC_ERR_NO_MEMORY, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        n = count;
    }
    // grow only
    void reserve(size_t count)
    {
        if (count > n) alloc(count);
    }
    T *get() const { return p; }
};

}  // namespace sfc

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct sfc_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;        // kernels launched (also those inside graph replays)
    int64_t graph_replays = 0;   // graph launches (each counted once here)
    cudaEvent_t marks[16] = {};
    // pinned host scratch for small device->host reads
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    sfc::DBuf<unsigned char> scratch;  // generic device scratch (CUB temp etc.)
    // small persistent device scratch (status words, scalars): per-call
    // allocations would put cudaMalloc/cudaFree (and their implicit device
    // synchronisation) on the repeated-solve path
    sfc::DBuf<int> ierr;       // >= 16 ints
    sfc::DBuf<double> dsmall;  // >= 16 doubles
    // kernel timing (off by default): an event pair around each profiled launch
    bool prof = false;
    struct ProfRec {
        const char *name;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
};

namespace sfc {

inline void count_launch(sfc_ctx *ctx, int n = 1)
{
    ctx->launches += n;
    SFC_CK(cudaGetLastError());
}

// Records a CUDA event before and after the launches in its scope when the
// context's profiling is on; the report sums device time and algorithmic
// bytes per kernel name.
struct ProfScope {
    sfc_ctx *ctx;
    long idx = -1;
    ProfScope(sfc_ctx *c, const char *name, double bytes) : ctx(c)
    {
        if (!ctx->prof) return;
        while (ctx->ev_pool.size() < ctx->ev_used + 2) {
            cudaEvent_t e;
            SFC_CK(cudaEventCreate(&e));
            ctx->ev_pool.push_back(e);
        }
        cudaEvent_t a = ctx->ev_pool[ctx->ev_used], b = ctx->ev_pool[ctx->ev_used + 1];
        ctx->ev_used += 2;
        SFC_CK(cudaEventRecord(a, ctx->stream));
        idx = (long)ctx->prof_recs.size();
        ctx->prof_recs.push_back({name, a, b, bytes});
    }
    ~ProfScope()
    {
        if (idx >= 0) cudaEventRecord(ctx->prof_recs[idx].b, ctx->stream);
    }
};

inline unsigned grid_for(int64_t work, int block, int max_blocks = 148 * 32)
{
    int64_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (unsigned)g;
}

// copy host -> device on the context stream (synchronous w.r.t. the host
// buffer: the call returns once the data has been consumed)
template <class T>
void upload(sfc_ctx *ctx, DBuf<T> &dst, const T *src, size_t count)
{
    dst.reserve(count);
    if (count) {
        SFC_CK(cudaMemcpyAsync(dst.p, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    }
}

template <class T>
void download(sfc_ctx *ctx, T *dst, const T *src, size_t count)
{
    if (count) {
        SFC_CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    }
}

void *pinned(sfc_ctx *ctx, size_t bytes);

// a status word in the context's persistent scratch (callers memset it)
struct DevInt {
    int *p;
};
inline DevInt status_word(sfc_ctx *ctx, int k = 0) { return DevInt{ctx->ierr.p + k}; }

// ---------------------------------------------------------------------------
// quadrature tables (weights, shape values, reference gradients at the
// points), evaluated on the host with the reference's literals
// ---------------------------------------------------------------------------
constexpr int kMaxQ = 27;

struct QuadTable {
    int nq;
    double w[kMaxQ];
    double xi[kMaxQ][3];
    double phi[kMaxQ][8];
    double dphi[kMaxQ][3][8];  // d phi^K / d xi_a
};

int elem_dim(int kind);
int elem_nodes(int kind);
int elem_dofs(int kind);
void make_quadrature(int kind, int qps, QuadTable &t);

}  // namespace sfc

// ---------------------------------------------------------------------------
// coarse space of the two-level preconditioner (coarse.cu): rigid-body modes
// (3-dof meshes) or the constant (scalar meshes) of box aggregates
// ---------------------------------------------------------------------------
struct sfc_mesh;
namespace sfc {
// scratch of spd_inverse_gj (dense.cu)
struct GjScratch {
    DBuf<double> diag, rowp, colp;
    DBuf<int> word;
    struct Graph {  // captured launch sequence of one (matrix, size)
        const double *A;
        int64_t n;
        double rel;
        const double *pivots;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    GjScratch() = default;
    GjScratch(const GjScratch &) = delete;
    GjScratch &operator=(const GjScratch &) = delete;
    ~GjScratch();
    void reserve(int64_t n);
    void drop_graphs();
};

// An instantiated CUDA graph of a captured launch sequence, with the key
// (pointers and sizes baked into its launches) it was captured for.
struct GraphExec {
    std::vector<uintptr_t> key;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;  // kernel launches per replay
    std::vector<uintptr_t> failed_key;  // a configuration whose capture failed (launched eagerly)
    GraphExec() = default;
    GraphExec(const GraphExec &) = delete;
    GraphExec &operator=(const GraphExec &) = delete;
    ~GraphExec() { reset(); }
    void reset()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        kernels = 0;
    }
};

// A pair of CUDA events kept for the life of their owner (timing of repeated
// solves without creating events per call).
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() = default;
    EventPair(const EventPair &) = delete;
    EventPair &operator=(const EventPair &) = delete;
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void ensure()
    {
        if (!a) SFC_CK(cudaEventCreate(&a));
        if (!b) SFC_CK(cudaEventCreate(&b));
    }
};

struct CoarseSpace {
    bool built = false;                 // aggregates for (mesh, size)
    const sfc_mesh *mesh = nullptr;
    int size = 0;                       // nodes per aggregate along each axis (target)
    uint64_t op_serial = 0;             // operator the inverse below belongs to
    int dof = 3;                        // 3: six rigid-body modes per aggregate; 1: its constant
    int64_t nodes = 0;
    int64_t nagg = 0, nc = 0;           // aggregates, coarse dofs
    int nb[3] = {1, 1, 1};              // boxes per axis
    int dropped = 0;                    // dependent coarse dofs left out of the inverse
    DBuf<int32_t> node_agg;             // nodes
    DBuf<int32_t> agg_ptr, agg_nodes;   // aggregate -> its nodes
    DBuf<int32_t> agg_slot;             // colour class (box index mod 3 per axis)
    DBuf<int32_t> nbr;                  // [nagg][27]: neighbour aggregate per colour class
    DBuf<float4> offset;                // node offset from the centroid / box edge
    DBuf<float4> mode;                  // offset + constrained components (bits in w)
    DBuf<double> a64;                   // nc x nc: Galerkin matrix, inverted in place
    DBuf<float> a32;                    // FP32 copy of the inverse, symmetrised, lda x lda zero-padded
    int64_t lda = 0;                    // nc rounded up to 64: row stride of a32, rows of c32 / e32
    GjScratch gj;                       // inverse scratch
    DBuf<float> c32, e32;               // [lda][K] restriction and correction (block; rows past nc zero in c32)
    const float *c32_zeroed = nullptr;  // c32 allocation, K and lda whose padding rows are zero
    int c32_zeroed_K = 0;
    int64_t c32_zeroed_lda = 0;
    DBuf<double> c64, e64;              // single FP64 vector
};

// vectors of V consecutive columns of a K = 32*V column block (lane owns
// columns lane*V .. lane*V+V-1)
template <int V>
struct VecT;
template <> struct VecT<1> { using f = float; using d = double; };
template <> struct VecT<2> { using f = float2; using d = double2; };
template <> struct VecT<4> { using f = float4; using d = double4; };

template <int V>
__device__ __forceinline__ void ldv(const float *p, float (&v)[V])
{
    if constexpr (V == 1) v[0] = *p;
    if constexpr (V == 2) { const float2 t = *reinterpret_cast<const float2 *>(p); v[0] = t.x; v[1] = t.y; }
    if constexpr (V == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
}
template <int V>
__device__ __forceinline__ void stv(float *p, const float (&v)[V])
{
    if constexpr (V == 1) *p = v[0];
    if constexpr (V == 2) *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
    if constexpr (V == 4) *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// V consecutive doubles (16-byte loads where V >= 2; the rows are 16-byte aligned)
template <int V>
__device__ __forceinline__ void ldv64(const double *p, double (&v)[V])
{
    if constexpr (V == 1) {
        v[0] = *p;
    } else {
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            const double2 t = *reinterpret_cast<const double2 *>(p + k);
            v[k] = t.x;
            v[k + 1] = t.y;
        }
    }
}

// reduce per-lane column partials acc[V] (column lane*V+v) over the block's
// warps and add them to out[K]
template <int V>
__device__ __forceinline__ void block_cols_add(const double (&acc)[V], double *sh, double *out)
{
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    constexpr int K = 32 * V;
#pragma unroll
    for (int v = 0; v < V; ++v) sh[w * K + l * V + v] = acc[v];
    __syncthreads();
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        double s = 0;
        for (int j = 0; j < nw; ++j) s += sh[j * K + c];
        atomicAdd(out + c, s);
    }
}
}  // namespace sfc

// ---------------------------------------------------------------------------
// mesh + its symbolic (pattern) data
// ---------------------------------------------------------------------------
struct sfc_mesh {
    sfc_ctx *ctx = nullptr;
    int kind = 0, qps = 0, dim = 0, nn = 0, dof = 0, L = 0;
    int64_t num_nodes = 0, num_elems = 0, num_dofs = 0;
    sfc::QuadTable quad{};
    std::vector<double> h_coords;  // num_nodes x 3
    sfc::DBuf<double> coords;      // num_nodes x 3
    sfc::DBuf<uint32_t> conn;      // num_elems x nn
    sfc::DBuf<double> coeff;       // num_elems
    double nu = 0.3;
    // CSR pattern of the assembled matrix (sorted unique (row,col) pairs)
    int64_t nnz = 0;
    sfc::DBuf<int32_t> row_ptr;    // num_dofs + 1
    sfc::DBuf<int32_t> col;        // nnz
    sfc::DBuf<int32_t> diag;       // num_dofs: slot of (i,i)
    // sorted-key gather map: CSR slot s sums element entries
    // contrib[slot_ptr[s] .. slot_ptr[s+1]) in element order; an element entry
    // id is e*L*L + r*L + c
    sfc::DBuf<int32_t> slot_ptr;   // nnz + 1
    sfc::DBuf<int32_t> contrib;    // num_elems * L * L
    // node -> incident (element*nn + local node), ascending element order
    sfc::DBuf<int32_t> node_ptr;   // num_nodes + 1
    sfc::DBuf<int32_t> node_elem;  // num_elems * nn
    // element matrices of the last assembly (num_elems * L * L)
    sfc::DBuf<double> ke;
    // tensor-grid description of the node set (for the Kronecker covariance)
    bool is_grid = false;
    int gn[3] = {1, 1, 1};
    std::vector<double> gaxis[3];
};

// ---------------------------------------------------------------------------
// linear system
// ---------------------------------------------------------------------------
struct sfc_system {
    sfc_ctx *ctx = nullptr;
    int64_t N = 0;
    sfc_solver_options_t opt{};
    sfc_solve_stats_t stats{};
    // pattern (owned copy, from a mesh or from staged triplets)
    int64_t nnz = 0;
    bool has_pattern = false;
    const sfc_mesh *pattern_mesh = nullptr;  // mesh whose pattern is installed
    sfc::DBuf<int32_t> row_ptr, col, diag;
    // values
    sfc::DBuf<double> a_ref;   // reference semantics: K with constrained rows zeroed
    sfc::DBuf<double> a_op;    // symmetric elimination (SPD operator) FP64
    sfc::DBuf<float> a_op32;   // FP32 copy of a_op
    sfc::DBuf<double> dinv;    // 1 / diag(a_op)
    sfc::DBuf<float> dinv32;
    bool op_valid = false;
    // node-block (3 x 3) view of the operator for 3-dof meshes: block row of
    // node i is [bptr[i], bptr[i+1]); bval holds the row-major 3x3 blocks
    bool has_bsr = false;
    int64_t nodes = 0, nblocks = 0;
    sfc::DBuf<int32_t> bptr, bcol;
    sfc::DBuf<float> bval32;
    sfc::DBuf<double> bval64;
    sfc::DBuf<float> bdinv32;  // inverse of each node's 3x3 diagonal block
    // lattice view (3-dof meshes whose nodes form an nx x ny x nz lattice
    // numbered x fastest, blocks coupling lattice neighbours only): every
    // node's 27 neighbour blocks in canonical slots (dz, dy, dx), zero where
    // the neighbour is missing, rows padded to 4 floats (lattice.cu)
    bool has_lattice = false;
    int lat_mode = 0;         // product on the lattice view: 1 staged bricks, 2 streamed x-lines
    int lat[3] = {0, 0, 0};
    sfc::DBuf<float> bq;      // nodes x 27 x 12
    sfc::DBuf<double> bq64;   // the same in FP64 (true residuals)
    sfc::DBuf<int> lat_err;   // bounded-wait status of the staged SpMM
    CUtensorMap pmap{};       // TMA view of the block operand P as (K, 3, nx, ny, nz)
    const float *pmap_ptr = nullptr;
    int pmap_K = 0;
    // vectors
    sfc::DBuf<double> F, X;
    sfc::DBuf<unsigned char> mask;   // 1 for constrained dofs
    sfc::DBuf<double> bc_val;        // prescribed value on constrained dofs
    bool any_constraint = false;
    bool inhomogeneous = false;
    double bc_scalar = 1.0;
    // host staging for the compat insert path
    std::vector<uint32_t> st_rows, st_cols;
    std::vector<double> st_vals;
    std::vector<double> st_rhs;
    bool st_rhs_dirty = false;
    // solver workspaces
    sfc::DBuf<double> w64;
    sfc::DBuf<float> w32;
    sfc::DBuf<double> scal;  // per-iteration scalars
    sfc::DBuf<int> flags;
    sfc::DBuf<double> fix;   // transposed-constraint fixup scratch
    // persistent workspaces of the block solver and the forward solve
    sfc::DBuf<double> blk64;   // b, x, r : 3 x N x K
    sfc::DBuf<float> blk32;    // x, r, p, q : 4 x N x K
    sfc::DBuf<double> colsc;   // per-column scalars
    sfc::DBuf<int> restart;    // per-column restart flags
    sfc::DBuf<double> tmpN, tmpN2;
    sfc::DBuf<double> fwd_rhs;  // lifted forward right-hand side (the mixed solver uses tmpN itself)
    sfc::DBuf<uint32_t> cidx;  // constraint upload buffers
    sfc::DBuf<double> cval;
    struct sfc_mpnn *mpnn = nullptr;  // learned preconditioner for SFC_SOLVER_FCG_MPNN
    int spmv_lanes = 0;               // lanes per row of the FP64 SpMV (0: by row length; set by the tuner)
    uint64_t op_serial = 0;           // bumped by every operator (re)build
    sfc::CoarseSpace coarse;          // SFC_PRECOND_TWO_LEVEL
    // the mixed block solver's check interval of iterations, captured once
    // per launch configuration (block widths 32, 64, 128)
    sfc::GraphExec blk_graph[3];
    sfc::EventPair solve_ev;  // device time of the last solve call
};

// ---------------------------------------------------------------------------
// statX objects
// ---------------------------------------------------------------------------
struct sfc_covar_forcing {
    sfc_ctx *ctx = nullptr;
    const sfc_mesh *mesh = nullptr;
    int dim = 0, dof = 0;
    int64_t num_nodes = 0, num_dofs = 0;
    sfc::DBuf<double> phibar;  // num_dofs
    sfc::DBuf<double> kron[3]; // 1-D SE factors along the grid axes
    sfc::DBuf<double> atb_part; // split-K partial tiles of the projected covariance
};

struct sfc_forward_gauss {
    sfc_ctx *ctx = nullptr;
    sfc_system *sys = nullptr;
    sfc_covar_forcing *cf = nullptr;
    double reg = 1e-4;
    int64_t ns = 0;
    std::vector<int64_t> p_ptr;
    std::vector<int32_t> p_idx;
    std::vector<double> p_val;
    sfc::DBuf<int64_t> d_p_ptr;
    sfc::DBuf<int32_t> d_p_idx;
    sfc::DBuf<double> d_p_val;
    std::vector<double> ppt;          // P P^T (ns x ns), host
    sfc::DBuf<double> d_ppt;
    sfc::DBuf<double> R;              // num_dofs x ns (column a = r_a)
    sfc::DBuf<double> mean;           // ns
    sfc::DBuf<double> cov;            // ns x ns
    sfc::DBuf<double> work;           // covariance workspace
    sfc::DBuf<double> B;              // adjoint right-hand sides P^T (N x ns)
    bool valid = false;
};

struct sfc_koh {
    sfc_ctx *ctx = nullptr;
    sfc_forward_gauss *fg = nullptr;
    int dim = 0;
    int64_t ns = 0;
    int n_o = 0;
    sfc::DBuf<double> sensor_coords;  // ns x 3
    sfc::DBuf<double> Y;              // ns x n_o
    sfc::DBuf<double> work;
    sfc::DBuf<double> outv;           // posterior mean / covariance / log-likelihood
    sfc::DBuf<int> info;
    sfc::GjScratch gj;                // sensor-space inverses
    // batched log-likelihood scratch
    sfc::DBuf<double> bwork, bres;
    sfc::DBuf<int> binfo;
    sfc::DBuf<sfc_hparams_t> bhp;
};

namespace sfc {
// assembly.cu
void build_pattern(sfc_mesh *m);
void assemble_matrix(sfc_system *s, const sfc_mesh *m);
void assemble_load(sfc_ctx *ctx, const sfc_mesh *m, const double *f, double *F_dev, bool zero_first);
void apply_constraints_dev(sfc_system *s, const uint32_t *idx_dev, const double *val_dev, int64_t n,
                           double factor, double scalar);
// require_positive_diag: fail on a non-positive (or NaN) diagonal entry; the
// batch path passes false and lets the affected instance fail alone
void build_operator(sfc_system *s, bool require_positive_diag = true);
// lattice.cu
void build_lattice_blocks(sfc_system *s);
void lattice_spmm32(sfc_system *s, const float *P, float *Q, int K, double *pq, const int *stop);
void lattice_prepare(sfc_system *s, const float *P, int K);
void lattice_check(sfc_system *s);
void xline_spmm32(sfc_system *s, const float *P, float *Q, int K, double *pq, const int *stop);
void xline_prepare(int K);
void xline_resid64(sfc_system *s, const double *X, const double *B, double *R, int K, double *rr);
void xresid_prepare(int K);
void coarse_block_reserve(sfc_system *s, int K);
void flush_staged(sfc_system *s);
void ensure_pattern_from_mesh(sfc_system *s, const sfc_mesh *m);
void element_matrices_unit(const sfc_mesh *m, double *ke0);
void gather_weighted(const sfc_mesh *m, const double *ke0, const double *w_dev, int kc, double *out);
// solvers.cu
void solve_forward(sfc_system *s);
void solve_block(sfc_system *s, const double *B_dev, double *X_dev, int nrhs, int ld);
void transpose_fixup(sfc_system *s, const double *B_dev, double *X_dev, int nrhs, int ld);
void solve_multi(sfc_system *s, const double *B_dev, double *X_dev, int nrhs, int ld);
double device_dot(sfc_ctx *ctx, const double *a, const double *b, int64_t n);
void spmv_op64(sfc_system *s, const double *x, double *y);
// y = S x and *xy += x . y, skipped entirely when *done != 0 (done may be NULL)
void spmv_op64_dot(sfc_system *s, const double *x, double *y, double *xy, const int *done);
void lifted_rhs(sfc_system *s, double *b);
struct PcgStats {
    int iters;
    bool converged;
};
PcgStats pcg64_public(sfc_system *s, const double *b, double *x, double tol, int max_iter, int check);
// mpnn.cu
void solve_forward_fcg(sfc_system *s);
// solvers.cu: FP64 SpMV with a given number of lanes per row (4, 8, 16, 32)
void spmv_op64_lanes(sfc_system *s, int lanes, const double *x, double *y);
// In-place inverse of the n x n symmetric positive (semi)definite device
// matrix A by block Gauss-Jordan elimination (dense.cu).  A pivot not above
// rel x its original diagonal is dropped (row and column zeroed);
// *dropped = their number (rel = 0: the non-positive pivots, i.e. A is not
// positive definite).  pivots (device, n, nullable): the Schur pivots.
void spd_inverse_gj(sfc_ctx *ctx, double *A, int64_t n, double rel, GjScratch &w, double *pivots, int *dropped);
// two-level preconditioner (coarse.cu)
bool coarse_prepare(sfc_system *s);
template <int V>
void coarse_block_apply(sfc_system *s, const float *r, double *rz, const int *stop);
template <int V>
void coarse_block_gemm(sfc_system *s, double *rz, const int *stop);  // e = A_c^+ c of cs.c32
void coarse_vec_apply(sfc_system *s, const double *r, double *rz, const int *done);
// stats.cu
void forward_gauss_update(sfc_forward_gauss *fg, const sfc_hparams_t *hp);
void projected_covar(sfc_ctx *ctx, sfc_covar_forcing *cf, double sigma, double length, const double *X, int64_t ns,
                     double *C, DBuf<double> &work);
void kernel_times(sfc_ctx *ctx, sfc_covar_forcing *cf, double sigma, double length, const double *W, double *T,
                  int64_t ns, double *tmp);
void atb_accumulate(sfc_ctx *ctx, const double *A, const double *B, int64_t K, int64_t M, int64_t Nn, double *C);
// C = A^T B (M x M) for A, B: K x M when A^T B is symmetric (stats.cu)
void atb_symmetric(sfc_ctx *ctx, const double *A, const double *B, int64_t K, int64_t M, double *C,
                   sfc::DBuf<double> &part);
// autotune.cu: the process-wide table of tuned launch shapes
std::string tune_device_key(sfc_ctx *ctx);
bool tune_lookup(const std::string &key, std::string &val);
void tune_store(const std::string &key, const std::string &val);
}  // namespace sfc
