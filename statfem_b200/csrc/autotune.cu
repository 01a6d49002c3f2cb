// Autotuner: launch shapes chosen by measurement on the caller's own problem,
// kept per (device, problem shape class) in a process-wide table that can be
// saved to and loaded from a text file.  (No reference counterpart: the
// reference has no tunable kernels.)
//
// Tuned knobs:
//   spmv   lanes per row of the FP64 SpMV (4, 8, 16, 32): each variant timed
//          over a few launches on the system's operator
//   block  block width of the mixed block solver (32, 64, 128 right-hand
//          sides per block) x preconditioner (point Jacobi, nodal 3x3 block
//          Jacobi on 3-dof meshes): each candidate solves the same sample of
//          the caller's right-hand sides to the system's tolerance, and the
//          fastest time to solution per right-hand side wins (so a stronger
//          preconditioner is credited with its fewer iterations)
//   batch  CTAs per instance of the batch kernel (tuned in batch.cu)
// Shape class: device name and SM count, log2 of the dof count, dofs per
// node, mean row length, log2 of the right-hand-side count.

#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "common.cuh"

namespace sfc {

namespace {
std::mutex g_tune_mu;
std::map<std::string, std::string> g_tune;  // shape-class key -> "v1 v2 ..."

int ilog2(int64_t v)
{
    int k = 0;
    while (v > 1) {
        v >>= 1;
        ++k;
    }
    return k;
}
}  // namespace

std::string tune_device_key(sfc_ctx *ctx)
{
    cudaDeviceProp p;
    SFC_CK(cudaGetDeviceProperties(&p, ctx->device));
    std::string name = p.name;
    for (char &c : name)
        if (c == ' ') c = '_';
    return name + "/sm" + std::to_string(p.multiProcessorCount);
}

bool tune_lookup(const std::string &key, std::string &val)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    val = it->second;
    return true;
}

void tune_store(const std::string &key, const std::string &val)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = val;
}

namespace {

std::string system_class(sfc_system *s, const char *what, int nrhs, int dof)
{
    const int row = (int)std::lround((double)s->nnz / (double)std::max<int64_t>(1, s->N));
    return std::string(what) + ":" + tune_device_key(s->ctx) + ":n" + std::to_string(ilog2(s->N)) + ":d" +
           std::to_string(dof) + ":r" + std::to_string(row) + ":k" + std::to_string(ilog2(std::max(1, nrhs)));
}

// device time of fn() on the context stream
double timed_ms(sfc_ctx *ctx, const std::function<void()> &fn)
{
    cudaEvent_t a, b;
    SFC_CK(cudaEventCreate(&a));
    SFC_CK(cudaEventCreate(&b));
    SFC_CK(cudaEventRecord(a, ctx->stream));
    fn();
    SFC_CK(cudaEventRecord(b, ctx->stream));
    SFC_CK(cudaEventSynchronize(b));
    float ms = 0;
    SFC_CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

int tune_spmv(sfc_system *s, bool measure)
{
    build_operator(s);
    const std::string key = system_class(s, "spmv", 1, s->has_bsr ? 3 : 1);
    std::string v;
    if (!measure && tune_lookup(key, v)) return std::atoi(v.c_str());
    const int64_t N = s->N;
    DBuf<double> x, y;
    x.alloc(N);
    y.alloc(N);
    std::vector<double> hx(N);
    std::mt19937_64 gen(7);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (auto &t : hx) t = u(gen);
    upload(s->ctx, x, hx.data(), N);
    int best = 32;
    double best_ms = 1e300;
    for (int lanes : {4, 8, 16, 32}) {
        spmv_op64_lanes(s, lanes, x.p, y.p);  // warm
        const double ms = timed_ms(s->ctx, [&] {
            for (int r = 0; r < 10; ++r) spmv_op64_lanes(s, lanes, x.p, y.p);
        });
        if (ms < best_ms) {
            best_ms = ms;
            best = lanes;
        }
    }
    tune_store(key, std::to_string(best));
    return best;
}

}  // namespace
}  // namespace sfc

using namespace sfc;

namespace {
int tguard(sfc_ctx *ctx, const std::function<void()> &fn)
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

int32_t sfc_autotune_spmv(sfc_system_t *s, int32_t remeasure, int32_t *lanes)
{
    if (!s) return SFC_ERR_BAD_ARG;
    return tguard(s->ctx, [&] {
        flush_staged(s);
        s->spmv_lanes = tune_spmv(s, remeasure != 0);
        if (lanes) *lanes = s->spmv_lanes;
    });
}

int32_t sfc_autotune_block_solver(sfc_system_t *s, const double *rhs, int32_t nrhs, int32_t remeasure,
                                  sfc_solver_options_t *best)
{
    if (!s || !rhs || nrhs <= 0) return SFC_ERR_BAD_ARG;
    return tguard(s->ctx, [&] {
        flush_staged(s);
        build_operator(s);
        const int dof = s->has_bsr ? 3 : 1;
        const std::string key = system_class(s, "block", nrhs, dof);
        sfc_solver_options_t o = s->opt;
        o.method = SFC_SOLVER_PCG_MIXED;
        std::string v;
        if (!remeasure && tune_lookup(key, v)) {
            int bw = 0, pc = 0, cs = 0;
            if (std::sscanf(v.c_str(), "%d %d %d", &bw, &pc, &cs) >= 2) {
                o.block_width = bw;
                o.precond = pc;
                o.coarse_size = cs;
                s->opt = o;
                if (best) *best = o;
                return;
            }
        }
        // sample: the first min(nrhs, 128) right-hand sides, interleaved
        const int64_t N = s->N;
        const int k = std::min(nrhs, 128);
        std::vector<double> Bt((size_t)N * k);
        for (int a = 0; a < k; ++a)
            for (int64_t i = 0; i < N; ++i) Bt[(size_t)i * k + a] = rhs[(size_t)a * N + i];
        DBuf<double> B, X;
        upload(s->ctx, B, Bt.data(), Bt.size());
        X.alloc((size_t)N * k);
        const sfc_solver_options_t keep = s->opt;
        double best_ms = 1e300;
        int best_bw = 32, best_pc = SFC_PRECOND_JACOBI, best_cs = 0;
        // (preconditioner, coarse size) candidates; the two-level ones only
        // where the system has a coarse space
        std::vector<std::pair<int, int>> pcs{{SFC_PRECOND_JACOBI, 0}};
        if (dof == 3) pcs.push_back({SFC_PRECOND_BLOCK_JACOBI, 0});
        if (s->pattern_mesh)
            for (int cs : {6, 8, 12}) pcs.push_back({SFC_PRECOND_TWO_LEVEL, cs});
        for (int bw : {32, 64, 128}) {
            if (bw > 32 && bw / 2 >= k) continue;  // wider blocks would be mostly padding
            for (auto [pc, csz] : pcs) {
                sfc_solver_options_t c = o;
                c.block_width = bw;
                c.precond = pc;
                c.coarse_size = csz;
                s->opt = c;
                double ms = 0;
                try {
                    solve_block(s, B.p, X.p, k, k);  // warm (first use of the width allocates)
                    ms = timed_ms(s->ctx, [&] { solve_block(s, B.p, X.p, k, k); });
                } catch (const Error &e) {
                    if (e.code != SFC_ERR_NOT_CONVERGED) {
                        s->opt = keep;
                        throw;
                    }
                    continue;  // this candidate does not reach tol within max_iter
                }
                if (pc == SFC_PRECOND_TWO_LEVEL && s->stats.coarse_dofs == 0) continue;  // no coarse space
                if (ms < best_ms) {
                    best_ms = ms;
                    best_bw = bw;
                    best_pc = pc;
                    best_cs = csz;
                }
            }
        }
        s->opt = keep;
        SFC_REQUIRE(best_ms < 1e300, "no block-solver candidate converged on the sample");
        o.block_width = best_bw;
        o.precond = best_pc;
        o.coarse_size = best_cs;
        s->opt = o;
        tune_store(key, std::to_string(best_bw) + " " + std::to_string(best_pc) + " " + std::to_string(best_cs));
        if (best) *best = o;
    });
}

int32_t sfc_autotune_save(const char *path)
{
    if (!path) return SFC_ERR_BAD_ARG;
    FILE *f = std::fopen(path, "w");
    if (!f) return SFC_ERR_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        std::fprintf(f, "# statfem_b200 autotune cache: shape-class key, tuned values\n");
        for (const auto &kv : g_tune) std::fprintf(f, "%s %s\n", kv.first.c_str(), kv.second.c_str());
    }
    return std::fclose(f) == 0 ? SFC_OK : SFC_ERR_BAD_ARG;
}

int32_t sfc_autotune_load(const char *path)
{
    if (!path) return SFC_ERR_BAD_ARG;
    FILE *f = std::fopen(path, "r");
    if (!f) return SFC_ERR_BAD_ARG;
    char line[1024];
    int rc = SFC_OK;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        char *sp = std::strchr(line, ' ');
        if (!sp) {
            rc = SFC_ERR_BAD_ARG;
            break;
        }
        *sp = 0;
        std::string val(sp + 1);
        while (!val.empty() && (val.back() == '\n' || val.back() == '\r')) val.pop_back();
        tune_store(line, val);
    }
    std::fclose(f);
    return rc;
}

int32_t sfc_autotune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    return SFC_OK;
}

}  // extern "C"
