// C entry points of include/statfem_cuda.h.  Each one validates its
// arguments, runs the internal C++ code, and turns an internal error into a
// status code plus a message stored on the context (the reference aborts via
// FTL_VERIFY instead, corlib/verify.hpp:61-70).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <new>

#include "common.cuh"

namespace sfc {
void covar_projected_host(sfc_covar_forcing *cf, const sfc_hparams_t *hp, const double *M, int64_t rows, double *out);
void koh_loglik(sfc_koh *k, const sfc_hparams_t *hp, double *out);
void koh_proj(sfc_koh *k, const sfc_hparams_t *hp, double *mean, double *cov);
void koh_woodbury(sfc_koh *k, const sfc_hparams_t *hp, double *mean, double *cov);
void koh_woodbury_mean(sfc_koh *k, const sfc_hparams_t *hp, double *mean);
void koh_loglik_batch(sfc_koh *k, const sfc_hparams_t *hps, int n, double *out);

void *pinned(sfc_ctx *ctx, size_t bytes)
{
    if (bytes > ctx->pinned_bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        SFC_CK(cudaMallocHost(&ctx->pinned, bytes));
        ctx->pinned_bytes = bytes;
    }
    return ctx->pinned;
}
}  // namespace sfc

using namespace sfc;

namespace {

int guard(sfc_ctx *ctx, const std::function<void()> &fn)
{
    try {
        if (ctx) SFC_CK(cudaSetDevice(ctx->device));
        fn();
        return SFC_OK;
    } catch (const Error &e) {
        if (ctx) ctx->err = e.msg;
        if (e.code == SFC_ERR_CUDA) cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc &) {
        if (ctx) ctx->err = "host allocation failed";
        return SFC_ERR_NO_MEMORY;
    } catch (const std::exception &e) {
        if (ctx) ctx->err = e.what();
        return SFC_ERR_BAD_ARG;
    }
}

// out[c][r] = in[r][c] for an rows x cols row-major FP64 matrix: 32 x 32
// tiles through shared memory (padded against bank conflicts), so both the
// reads and the writes are coalesced
__global__ void k_transpose64(const double *__restrict__ in, double *__restrict__ out, int64_t rows, int64_t cols)
{
    __shared__ double tile[32][33];
    const int64_t ct = (cols + 31) / 32;  // tiles along the columns; the grid is one tile per CTA
    const int64_t r0 = ((int64_t)blockIdx.x / ct) * 32, c0 = ((int64_t)blockIdx.x % ct) * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = in[r * cols + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t c = c0 + j, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[c * rows + r] = tile[threadIdx.x][j];
    }
}

void transpose64(sfc_ctx *ctx, const double *in, double *out, int64_t rows, int64_t cols)
{
    const int64_t tiles = ((rows + 31) / 32) * ((cols + 31) / 32);
    SFC_REQUIRE(tiles <= 0x7fffffff, "transpose: too many tiles");
    k_transpose64<<<(unsigned)tiles, dim3(32, 8), 0, ctx->stream>>>(in, out, rows, cols);
    count_launch(ctx);
}

void ensure_vectors(sfc_system *s)
{
    if (!s->F.p) {
        s->F.alloc(s->N);
        SFC_CK(cudaMemsetAsync(s->F.p, 0, s->N * 8, s->ctx->stream));
    }
}

}  // namespace

extern "C" {

int32_t sfc_version(void) { return 1; }

int32_t sfc_ctx_create(int32_t device, sfc_ctx_t **out)
{
    if (!out) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_ctx *ctx = new (std::nothrow) sfc_ctx();
    if (!ctx) return SFC_ERR_NO_MEMORY;
    ctx->device = device;
    int rc = guard(ctx, [&] {
        int ndev = 0;
        SFC_CK(cudaGetDeviceCount(&ndev));
        SFC_REQUIRE(device >= 0 && device < ndev, "no such CUDA device");
        SFC_CK(cudaSetDevice(device));
        SFC_CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        SFC_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        for (auto &e : ctx->marks) SFC_CK(cudaEventCreate(&e));
        ctx->ierr.alloc(16);
        ctx->dsmall.alloc(16);
    });
    if (rc != SFC_OK) {
        delete ctx;
        return rc;
    }
    *out = ctx;
    return SFC_OK;
}

int32_t sfc_ctx_destroy(sfc_ctx_t *ctx)
{
    if (!ctx) return SFC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &e : ctx->marks)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->ev_pool) cudaEventDestroy(e);
    ctx->scratch.release();
    ctx->ierr.release();
    ctx->dsmall.release();
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SFC_OK;
}

const char *sfc_last_error(const sfc_ctx_t *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t sfc_ctx_synchronize(sfc_ctx_t *ctx)
{
    if (!ctx) return SFC_ERR_BAD_ARG;
    return guard(ctx, [&] { SFC_CK(cudaStreamSynchronize(ctx->stream)); });
}

int32_t sfc_ctx_kernel_launches(const sfc_ctx_t *ctx, int64_t *count)
{
    if (!ctx || !count) return SFC_ERR_BAD_ARG;
    *count = ctx->launches;
    return SFC_OK;
}

int32_t sfc_ctx_graph_launches(const sfc_ctx_t *ctx, int64_t *count)
{
    if (!ctx || !count) return SFC_ERR_BAD_ARG;
    *count = ctx->graph_replays;
    return SFC_OK;
}

int32_t sfc_ctx_mark(sfc_ctx_t *ctx, int32_t slot)
{
    if (!ctx || slot < 0 || slot >= 16) return SFC_ERR_BAD_ARG;
    return guard(ctx, [&] { SFC_CK(cudaEventRecord(ctx->marks[slot], ctx->stream)); });
}

int32_t sfc_ctx_marker_ms(sfc_ctx_t *ctx, int32_t a, int32_t b, double *ms)
{
    if (!ctx || !ms || a < 0 || a >= 16 || b < 0 || b >= 16) return SFC_ERR_BAD_ARG;
    return guard(ctx, [&] {
        SFC_CK(cudaEventSynchronize(ctx->marks[b]));
        float f = 0;
        SFC_CK(cudaEventElapsedTime(&f, ctx->marks[a], ctx->marks[b]));
        *ms = f;
    });
}

int32_t sfc_ctx_set_profiling(sfc_ctx_t *ctx, int32_t enable)
{
    if (!ctx) return SFC_ERR_BAD_ARG;
    ctx->prof = enable != 0;
    return SFC_OK;
}

int32_t sfc_ctx_profile_report(sfc_ctx_t *ctx, char *buf, int64_t buflen)
{
    if (!ctx || !buf || buflen <= 0) return SFC_ERR_BAD_ARG;
    return guard(ctx, [&] {
        SFC_CK(cudaStreamSynchronize(ctx->stream));
        std::vector<std::string> names;
        std::vector<double> ms, bytes;
        std::vector<long> cnt;
        for (auto &r : ctx->prof_recs) {
            float f = 0;
            SFC_CK(cudaEventElapsedTime(&f, r.a, r.b));
            size_t k = 0;
            while (k < names.size() && names[k] != r.name) ++k;
            if (k == names.size()) {
                names.emplace_back(r.name);
                ms.push_back(0);
                bytes.push_back(0);
                cnt.push_back(0);
            }
            ms[k] += f;
            bytes[k] += r.bytes;
            cnt[k] += 1;
        }
        std::string out;
        char line[256];
        for (size_t k = 0; k < names.size(); ++k) {
            snprintf(line, sizeof line, "%s %ld %.6f %.1f\n", names[k].c_str(), cnt[k], ms[k], bytes[k]);
            out += line;
        }
        ctx->prof_recs.clear();
        ctx->ev_used = 0;
        const size_t n = std::min<size_t>(out.size(), (size_t)buflen - 1);
        std::memcpy(buf, out.data(), n);
        buf[n] = 0;
    });
}

// ---- mesh -------------------------------------------------------------------
int32_t sfc_mesh_create(sfc_ctx_t *ctx, int32_t kind, int32_t qps, const double *coords, int64_t num_nodes,
                        const uint32_t *conn, int64_t num_elems, sfc_mesh_t **out)
{
    if (!ctx || !out || !coords || !conn || num_nodes <= 0 || num_elems <= 0) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_mesh *m = new (std::nothrow) sfc_mesh();
    if (!m) return SFC_ERR_NO_MEMORY;
    int rc = guard(ctx, [&] {
        SFC_REQUIRE(kind >= SFC_ELEM_LINE2_POISSON && kind <= SFC_ELEM_HEX8_ELASTIC, "unknown element kind");
        m->ctx = ctx;
        m->kind = kind;
        m->qps = qps;
        m->dim = elem_dim(kind);
        m->nn = elem_nodes(kind);
        m->dof = elem_dofs(kind);
        m->L = m->nn * m->dof;
        m->num_nodes = num_nodes;
        m->num_elems = num_elems;
        m->num_dofs = num_nodes * m->dof;
        SFC_REQUIRE_SIZE(m->num_dofs < (int64_t)INT32_MAX, "more than 2^31 - 1 dofs (32-bit column indices)");
        make_quadrature(kind, qps, m->quad);
        for (int64_t t = 0; t < num_elems * m->nn; ++t)
            SFC_REQUIRE(conn[t] < (uint64_t)num_nodes, "connectivity refers to a node that does not exist");
        m->h_coords.assign(coords, coords + 3 * num_nodes);
        upload(ctx, m->coords, coords, 3 * num_nodes);
        upload(ctx, m->conn, conn, num_elems * m->nn);
        build_pattern(m);
    });
    if (rc != SFC_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return SFC_OK;
}

int32_t sfc_mesh_destroy(sfc_mesh_t *m)
{
    if (!m) return SFC_OK;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    delete m;
    return SFC_OK;
}

int32_t sfc_mesh_set_coefficients(sfc_mesh_t *m, const double *values, double uniform, double nu)
{
    if (!m) return SFC_ERR_BAD_ARG;
    return guard(m->ctx, [&] {
        m->nu = nu;
        if (values) {
            upload(m->ctx, m->coeff, values, m->num_elems);
        } else {
            std::vector<double> v(m->num_elems, uniform);
            upload(m->ctx, m->coeff, v.data(), v.size());
        }
    });
}

int64_t sfc_mesh_num_dofs(const sfc_mesh_t *m) { return m ? m->num_dofs : -1; }
int64_t sfc_mesh_nnz(const sfc_mesh_t *m) { return m ? m->nnz : -1; }

// ---- system -------------------------------------------------------------------
int32_t sfc_system_create(sfc_ctx_t *ctx, int64_t num_dofs, sfc_system_t **out)
{
    if (!ctx || !out || num_dofs <= 0) return SFC_ERR_BAD_ARG;
    if (num_dofs >= (int64_t)INT32_MAX) return SFC_ERR_TOO_LARGE;  // 32-bit column indices
    *out = nullptr;
    sfc_system *s = new (std::nothrow) sfc_system();
    if (!s) return SFC_ERR_NO_MEMORY;
    int rc = guard(ctx, [&] {
        s->ctx = ctx;
        s->N = num_dofs;
        s->opt.method = SFC_SOLVER_PCG_FP64;
        s->opt.max_iter = 20000;
        s->opt.tol = 1e-8;
        s->opt.inner_tol = 1e-4;
        s->opt.block_width = 0;
        s->opt.check_every = 16;
        s->opt.precond = SFC_PRECOND_JACOBI;
        ensure_vectors(s);
        s->st_rhs.assign(num_dofs, 0.0);
    });
    if (rc != SFC_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return SFC_OK;
}

int32_t sfc_system_destroy(sfc_system_t *s)
{
    if (!s) return SFC_OK;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    delete s;
    return SFC_OK;
}

int32_t sfc_system_set_options(sfc_system_t *s, const sfc_solver_options_t *o)
{
    if (!s || !o) return SFC_ERR_BAD_ARG;
    if (o->precond != SFC_PRECOND_JACOBI && o->precond != SFC_PRECOND_BLOCK_JACOBI &&
        o->precond != SFC_PRECOND_TWO_LEVEL) {
        s->ctx->err = "unknown preconditioner";
        return SFC_ERR_BAD_ARG;
    }
    if (o->coarse_size < 0) {
        s->ctx->err = "coarse_size must be >= 0";
        return SFC_ERR_BAD_ARG;
    }
    if (o->method != SFC_SOLVER_PCG_FP64 && o->method != SFC_SOLVER_PCG_MIXED && o->method != SFC_SOLVER_FCG_MPNN) {
        s->ctx->err = "unknown solver method";
        return SFC_ERR_BAD_ARG;
    }
    if (!(o->tol > 0) || o->max_iter <= 0) {
        s->ctx->err = "tol and max_iter must be positive";
        return SFC_ERR_BAD_ARG;
    }
    s->opt = *o;
    return SFC_OK;
}

int32_t sfc_system_get_options(const sfc_system_t *s, sfc_solver_options_t *o)
{
    if (!s || !o) return SFC_ERR_BAD_ARG;
    *o = s->opt;
    return SFC_OK;
}

int32_t sfc_system_last_stats(const sfc_system_t *s, sfc_solve_stats_t *st)
{
    if (!s || !st) return SFC_ERR_BAD_ARG;
    *st = s->stats;
    return SFC_OK;
}

int32_t sfc_insert_matrix(sfc_system_t *s, const double *Ke, const uint32_t *rows, uint32_t n, const uint32_t *cols,
                          uint32_t m)
{
    if (!s || !Ke || !rows || !cols) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        for (uint32_t i = 0; i < n; ++i) SFC_REQUIRE(rows[i] < (uint64_t)s->N, "row index out of range");
        for (uint32_t j = 0; j < m; ++j) SFC_REQUIRE(cols[j] < (uint64_t)s->N, "column index out of range");
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = 0; j < m; ++j) {
                s->st_rows.push_back(rows[i]);
                s->st_cols.push_back(cols[j]);
                s->st_vals.push_back(Ke[(size_t)i * m + j]);
            }
    });
}

int32_t sfc_insert_rhs(sfc_system_t *s, const double *fe, const uint32_t *dofs, uint32_t n)
{
    if (!s || !fe || !dofs) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        for (uint32_t i = 0; i < n; ++i) SFC_REQUIRE(dofs[i] < (uint64_t)s->N, "dof index out of range");
        for (uint32_t i = 0; i < n; ++i) s->st_rhs[dofs[i]] += fe[i];
        s->st_rhs_dirty = true;
    });
}

int32_t sfc_finish_assembly(sfc_system_t *s)
{
    if (!s) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] { flush_staged(s); });
}

int32_t sfc_assemble_matrix(sfc_system_t *s, const sfc_mesh_t *m)
{
    if (!s || !m) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        SFC_REQUIRE(m->ctx == s->ctx, "mesh and system belong to different contexts");
        assemble_matrix(s, m);
    });
}

int32_t sfc_assemble_load(sfc_system_t *s, const sfc_mesh_t *m, const double *f)
{
    if (!s || !m || !f) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        SFC_REQUIRE(m->num_dofs == s->N, "mesh dof count differs from the system size");
        ensure_vectors(s);
        assemble_load(s->ctx, m, f, s->F.p, false);
    });
}

int32_t sfc_apply_constraints(sfc_system_t *s, const uint32_t *idx, const double *value, int64_t n, double factor,
                              double scalar)
{
    if (!s || (n > 0 && !idx) || n < 0) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        flush_staged(s);
        if (n == 0) return;
        upload(s->ctx, s->cidx, idx, n);
        if (value) {
            upload(s->ctx, s->cval, value, n);
            for (int64_t t = 0; t < n; ++t)
                if (value[t] != 0.0) s->inhomogeneous = true;
        }
        apply_constraints_dev(s, s->cidx.p, value ? s->cval.p : nullptr, n, factor, scalar);
        SFC_CK(cudaStreamSynchronize(s->ctx->stream));
    });
}

int32_t sfc_fix_dof(sfc_system_t *s, uint32_t idx, double scalar)
{
    double zero = 0.0;
    return sfc_apply_constraints(s, &idx, &zero, 1, 1.0, scalar);
}

int32_t sfc_solve(sfc_system_t *s, int32_t reuse)
{
    (void)reuse;
    if (!s) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        flush_staged(s);
        solve_forward(s);
    });
}

int32_t sfc_solve_transpose(sfc_system_t *s, const double *rhs, double *u, int32_t nrhs, int32_t reuse)
{
    (void)reuse;
    if (!s || !rhs || !u || nrhs <= 0) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        flush_staged(s);
        const int64_t N = s->N;
        std::vector<double> Bt((size_t)N * nrhs);
        for (int a = 0; a < nrhs; ++a)
            for (int64_t i = 0; i < N; ++i) Bt[(size_t)i * nrhs + a] = rhs[(size_t)a * N + i];
        DBuf<double> B, X;
        upload(s->ctx, B, Bt.data(), Bt.size());
        X.alloc((size_t)N * nrhs);
        solve_block(s, B.p, X.p, nrhs, nrhs);
        transpose_fixup(s, B.p, X.p, nrhs, nrhs);
        download(s->ctx, Bt.data(), X.p, Bt.size());
        for (int a = 0; a < nrhs; ++a)
            for (int64_t i = 0; i < N; ++i) u[(size_t)a * N + i] = Bt[(size_t)i * nrhs + a];
    });
}

int32_t sfc_solve_multi(sfc_system_t *s, const double *rhs, double *u, int32_t nrhs)
{
    if (!s || !rhs || !u || nrhs <= 0) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        flush_staged(s);
        const int64_t N = s->N;
        // the caller's [nrhs][N] columns go up as they are and are transposed
        // to the interleaved [N][nrhs] layout on the GPU (and back)
        DBuf<double> C, B, X;
        upload(s->ctx, C, rhs, (size_t)N * nrhs);
        B.alloc((size_t)N * nrhs);
        transpose64(s->ctx, C.p, B.p, nrhs, N);
        X.alloc((size_t)N * nrhs);
        solve_multi(s, B.p, X.p, nrhs, nrhs);
        transpose64(s->ctx, X.p, C.p, N, nrhs);
        download(s->ctx, u, C.p, (size_t)N * nrhs);
    });
}

int32_t sfc_solve_multi_device(sfc_system_t *s, const double *rhs_dev, double *u_dev, int32_t nrhs, int32_t ld)
{
    if (!s || !rhs_dev || !u_dev || nrhs <= 0 || ld < nrhs) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        flush_staged(s);
        solve_multi(s, rhs_dev, u_dev, nrhs, ld);
    });
}

static int give_vec(const sfc_system *s, const double *src, const uint32_t *dofs, int64_t n, double *out)
{
    if (!s || !out || (n > 0 && !dofs)) return SFC_ERR_BAD_ARG;
    sfc_system *sm = const_cast<sfc_system *>(s);
    return guard(sm->ctx, [&] {
        SFC_REQUIRE(src, "vector not available (solve first)");
        std::vector<double> h(s->N);
        download(sm->ctx, h.data(), src, s->N);
        for (int64_t t = 0; t < n; ++t) {
            SFC_REQUIRE(dofs[t] < (uint64_t)s->N, "dof index out of range");
            out[t] = h[dofs[t]];
        }
    });
}

int32_t sfc_give_solution(const sfc_system_t *s, const uint32_t *dofs, int64_t n, double *out)
{
    return give_vec(s, s ? s->X.p : nullptr, dofs, n, out);
}

int32_t sfc_give_force(const sfc_system_t *s, const uint32_t *dofs, int64_t n, double *out)
{
    if (s && s->st_rhs_dirty) {
        int rc = guard(s->ctx, [&] { flush_staged(const_cast<sfc_system *>(s)); });
        if (rc) return rc;
    }
    return give_vec(s, s ? s->F.p : nullptr, dofs, n, out);
}

int32_t sfc_clear_matrix(sfc_system_t *s)
{
    if (!s) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        // Triplet::erase keeps the entries and zeroes the values
        // (corlib/Triplet.hpp:356-366); staged entries are dropped
        flush_staged(s);
        if (s->has_pattern) SFC_CK(cudaMemsetAsync(s->a_ref.p, 0, s->nnz * 8, s->ctx->stream));
        if (s->mask.p) SFC_CK(cudaMemsetAsync(s->mask.p, 0, s->N, s->ctx->stream));
        s->any_constraint = false;
        s->inhomogeneous = false;
        s->op_valid = false;
        SFC_CK(cudaStreamSynchronize(s->ctx->stream));
    });
}

int32_t sfc_clear_rhs(sfc_system_t *s)
{
    if (!s) return SFC_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        std::fill(s->st_rhs.begin(), s->st_rhs.end(), 0.0);
        s->st_rhs_dirty = false;
        SFC_CK(cudaMemsetAsync(s->F.p, 0, s->N * 8, s->ctx->stream));
        SFC_CK(cudaStreamSynchronize(s->ctx->stream));
    });
}

int64_t sfc_num_nonzeros(const sfc_system_t *s)
{
    if (!s) return -1;
    return (s->has_pattern ? s->nnz : 0) + (int64_t)s->st_vals.size();
}

int32_t sfc_norms(const sfc_system_t *s, double *fro, double *n2rhs, double *n1rhs, double *n2sol)
{
    if (!s) return SFC_ERR_BAD_ARG;
    sfc_system *sm = const_cast<sfc_system *>(s);
    return guard(sm->ctx, [&] {
        flush_staged(sm);
        if (fro) {
            *fro = 0;
            if (s->has_pattern) *fro = std::sqrt(device_dot(sm->ctx, s->a_ref.p, s->a_ref.p, s->nnz));
        }
        if (n2rhs || n1rhs) {
            std::vector<double> h(s->N);
            download(sm->ctx, h.data(), s->F.p, s->N);
            double a = 0, b = 0;
            for (double v : h) {
                a += v * v;
                b += std::fabs(v);
            }
            if (n2rhs) *n2rhs = std::sqrt(a);
            if (n1rhs) *n1rhs = b;
        }
        if (n2sol) *n2sol = s->X.p ? std::sqrt(device_dot(sm->ctx, s->X.p, s->X.p, s->N)) : 0.0;
    });
}

int32_t sfc_get_csr(const sfc_system_t *s, int64_t *row_ptr, int32_t *col, double *val)
{
    if (!s) return SFC_ERR_BAD_ARG;
    sfc_system *sm = const_cast<sfc_system *>(s);
    return guard(sm->ctx, [&] {
        flush_staged(sm);
        SFC_REQUIRE(s->has_pattern, "no matrix assembled");
        if (row_ptr) {
            std::vector<int32_t> rp(s->N + 1);
            download(sm->ctx, rp.data(), s->row_ptr.p, s->N + 1);
            for (int64_t i = 0; i <= s->N; ++i) row_ptr[i] = rp[i];
        }
        if (col) download(sm->ctx, col, s->col.p, s->nnz);
        if (val) download(sm->ctx, val, s->a_ref.p, s->nnz);
    });
}

// ---- covariance forcing ---------------------------------------------------------
int32_t sfc_covar_forcing_create(sfc_ctx_t *ctx, const sfc_mesh_t *m, sfc_covar_forcing_t **out)
{
    if (!ctx || !m || !out) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_covar_forcing *cf = new (std::nothrow) sfc_covar_forcing();
    if (!cf) return SFC_ERR_NO_MEMORY;
    int rc = guard(ctx, [&] {
        cf->ctx = ctx;
        cf->mesh = m;
        cf->dim = m->dim;
        cf->dof = m->dof;
        cf->num_nodes = m->num_nodes;
        cf->num_dofs = m->num_dofs;
        cf->phibar.alloc(m->num_dofs);
        const double one[3] = {1.0, 1.0, 1.0};
        assemble_load(ctx, m, one, cf->phibar.p, true);
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    });
    if (rc != SFC_OK) {
        delete cf;
        return rc;
    }
    *out = cf;
    return SFC_OK;
}

int32_t sfc_covar_forcing_destroy(sfc_covar_forcing_t *cf)
{
    if (!cf) return SFC_OK;
    cudaSetDevice(cf->ctx->device);
    cudaStreamSynchronize(cf->ctx->stream);
    delete cf;
    return SFC_OK;
}

int32_t sfc_covar_forcing_apply_constraints(sfc_covar_forcing_t *cf, const uint32_t *idx, int64_t n)
{
    if (!cf || (n > 0 && !idx)) return SFC_ERR_BAD_ARG;
    return guard(cf->ctx, [&] {
        std::vector<double> h(cf->num_dofs);
        download(cf->ctx, h.data(), cf->phibar.p, cf->num_dofs);
        for (int64_t t = 0; t < n; ++t) {
            SFC_REQUIRE(idx[t] < (uint64_t)cf->num_dofs, "constraint index out of range");
            h[idx[t]] = 0.0;
        }
        upload(cf->ctx, cf->phibar, h.data(), h.size());
    });
}

int32_t sfc_covar_forcing_get_phibar(const sfc_covar_forcing_t *cf, double *out)
{
    if (!cf || !out) return SFC_ERR_BAD_ARG;
    return guard(cf->ctx, [&] { download(cf->ctx, out, cf->phibar.p, cf->num_dofs); });
}

int32_t sfc_covar_forcing_projected(sfc_covar_forcing_t *cf, const sfc_hparams_t *hp, const double *M, int64_t rows,
                                    double *out)
{
    if (!cf || !hp || !M || !out || rows <= 0) return SFC_ERR_BAD_ARG;
    return guard(cf->ctx, [&] { covar_projected_host(cf, hp, M, rows, out); });
}

// ---- forward gauss ------------------------------------------------------------------
int32_t sfc_forward_gauss_create(sfc_system_t *s, sfc_covar_forcing_t *cf, double reg, sfc_forward_gauss_t **out)
{
    if (!s || !cf || !out) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_forward_gauss *fg = new (std::nothrow) sfc_forward_gauss();
    if (!fg) return SFC_ERR_NO_MEMORY;
    fg->ctx = s->ctx;
    fg->sys = s;
    fg->cf = cf;
    fg->reg = reg;
    *out = fg;
    return SFC_OK;
}

int32_t sfc_forward_gauss_destroy(sfc_forward_gauss_t *fg)
{
    if (!fg) return SFC_OK;
    cudaSetDevice(fg->ctx->device);
    cudaStreamSynchronize(fg->ctx->stream);
    delete fg;
    return SFC_OK;
}

int32_t sfc_forward_gauss_set_projection(sfc_forward_gauss_t *fg, int64_t ns, const int64_t *indptr,
                                         const int32_t *indices, const double *data)
{
    if (!fg || ns <= 0 || !indptr || !indices || !data) return SFC_ERR_BAD_ARG;
    return guard(fg->ctx, [&] {
        const int64_t N = fg->sys->N;
        const int64_t nnz = indptr[ns];
        for (int64_t t = 0; t < nnz; ++t) SFC_REQUIRE(indices[t] >= 0 && indices[t] < N, "projection index out of range");
        fg->ns = ns;
        fg->p_ptr.assign(indptr, indptr + ns + 1);
        fg->p_idx.assign(indices, indices + nnz);
        fg->p_val.assign(data, data + nnz);
        upload(fg->ctx, fg->d_p_ptr, indptr, ns + 1);
        upload(fg->ctx, fg->d_p_idx, indices, nnz);
        upload(fg->ctx, fg->d_p_val, data, nnz);
        // P P^T on the host (sparse rows)
        fg->ppt.assign((size_t)ns * ns, 0.0);
        std::vector<double> row(N, 0.0);
        for (int64_t a = 0; a < ns; ++a) {
            for (int64_t t = indptr[a]; t < indptr[a + 1]; ++t) row[indices[t]] += data[t];
            for (int64_t b = 0; b < ns; ++b) {
                double v = 0;
                for (int64_t t = indptr[b]; t < indptr[b + 1]; ++t) v += row[indices[t]] * data[t];
                fg->ppt[(size_t)a * ns + b] = v;
            }
            for (int64_t t = indptr[a]; t < indptr[a + 1]; ++t) row[indices[t]] = 0.0;
        }
        upload(fg->ctx, fg->d_ppt, fg->ppt.data(), fg->ppt.size());
        fg->valid = false;
    });
}

int32_t sfc_forward_gauss_update(sfc_forward_gauss_t *fg, const sfc_hparams_t *hp)
{
    if (!fg || !hp) return SFC_ERR_BAD_ARG;
    return guard(fg->ctx, [&] { forward_gauss_update(fg, hp); });
}

int32_t sfc_forward_gauss_mean(const sfc_forward_gauss_t *fg, double *out)
{
    if (!fg || !out) return SFC_ERR_BAD_ARG;
    return guard(fg->ctx, [&] {
        SFC_REQUIRE(fg->valid, "updateSolution has not been called");
        download(fg->ctx, out, fg->mean.p, fg->ns);
    });
}

int32_t sfc_forward_gauss_covar(const sfc_forward_gauss_t *fg, double *out)
{
    if (!fg || !out) return SFC_ERR_BAD_ARG;
    return guard(fg->ctx, [&] {
        SFC_REQUIRE(fg->valid, "updateSolution has not been called");
        download(fg->ctx, out, fg->cov.p, fg->ns * fg->ns);
    });
}

// ---- KOH ----------------------------------------------------------------------------
int32_t sfc_koh_create(sfc_forward_gauss_t *fg, const double *sensor_coords, int32_t dim, sfc_koh_t **out)
{
    if (!fg || !sensor_coords || !out || dim < 1 || dim > 3) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_koh *k = new (std::nothrow) sfc_koh();
    if (!k) return SFC_ERR_NO_MEMORY;
    int rc = guard(fg->ctx, [&] {
        SFC_REQUIRE(fg->ns > 0, "set the projection matrix before creating the likelihood");
        k->ctx = fg->ctx;
        k->fg = fg;
        k->dim = dim;
        k->ns = fg->ns;
        std::vector<double> xs((size_t)3 * k->ns, 0.0);
        for (int64_t a = 0; a < k->ns; ++a)
            for (int d = 0; d < dim; ++d) xs[3 * a + d] = sensor_coords[a * dim + d];
        upload(k->ctx, k->sensor_coords, xs.data(), xs.size());
    });
    if (rc != SFC_OK) {
        delete k;
        return rc;
    }
    *out = k;
    return SFC_OK;
}

int32_t sfc_koh_destroy(sfc_koh_t *k)
{
    if (!k) return SFC_OK;
    cudaSetDevice(k->ctx->device);
    cudaStreamSynchronize(k->ctx->stream);
    delete k;
    return SFC_OK;
}

int32_t sfc_koh_set_sensor_values(sfc_koh_t *k, const double *Y, int32_t n_o)
{
    if (!k || !Y || n_o <= 0) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] {
        upload(k->ctx, k->Y, Y, (size_t)k->ns * n_o);
        k->n_o = n_o;
    });
}

int32_t sfc_koh_log_likelihood(sfc_koh_t *k, const sfc_hparams_t *hp, double *out)
{
    if (!k || !hp || !out) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] { koh_loglik(k, hp, out); });
}

int32_t sfc_koh_proj_conditioned(sfc_koh_t *k, const sfc_hparams_t *hp, double *mean, double *cov)
{
    if (!k || !hp) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] { koh_proj(k, hp, mean, cov); });
}

int32_t sfc_koh_woodbury(sfc_koh_t *k, const sfc_hparams_t *hp, double *mean, double *cov)
{
    if (!k || !hp) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] { koh_woodbury(k, hp, mean, cov); });
}

int32_t sfc_koh_log_likelihood_batch(sfc_koh_t *k, const sfc_hparams_t *hps, int32_t n, double *loglik)
{
    if (!k || !hps || n <= 0 || !loglik) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] { koh_loglik_batch(k, hps, n, loglik); });
}

int32_t sfc_koh_woodbury_mean(sfc_koh_t *k, const sfc_hparams_t *hp, double *mean)
{
    if (!k || !hp || !mean) return SFC_ERR_BAD_ARG;
    return guard(k->ctx, [&] { koh_woodbury_mean(k, hp, mean); });
}

}  // extern "C"
