// First-order material uncertainty: statX::infer::ForwardPerturbation
// (statX/infer/ForwardPerturbation.hpp:109-195) with CovarianceMaterial
// (statX/infer/CovarianceMaterial.hpp) and the stiffness derivative
// ElementPotential::stiffnessDerivIntegrand (del2/fem/ElementPotential.ipp:
// 225-237).
//
// The reference forms, with R = P A^-1 (adjoint solves), u = A^-1 F,
// M = A^-1 C_f A^-T + u u^T and the material covariance C_m over element
// centroids,
//   C_s = R C_f R^T + sum_e sum_d C_m(e,d) R A'_e M A'_d^T R^T
//         + (reg sigma_m)^2 P P^T,   mean = P u,
// a double sum over element pairs of dense N x N products.  Here C_m = L L^T
// (pivoted Cholesky on the host, to a relative tolerance), which turns the
// double sum into sum_k B_k M B_k^T with B_k = R A'(L[:,k]), A'(w) =
// sum_e w_e dA/dkappa_e the stiffness assembled with element weights w.
// Then
//   B_k M B_k^T = Y_k^T C_f Y_k + (B_k u)(B_k u)^T,  Y_k = A^-T B_k^T,
// i.e. r * ns adjoint solves (one block solve per chunk of k) and the
// forcing-covariance kernels already used for C_s.  dA/dkappa_e is the unit-
// conductivity element matrix with the constrained rows zeroed (the
// reference's row-zeroed A does not depend on kappa there), so
// B_k^T = K'(L[:,k]) (free .* R^T) with the symmetric unconstrained K'.
//
// The reference fills only the first ns rows of its A^-1 (its loop runs over
// the sensors, ForwardPerturbation.hpp:128-138); the two agree when P is the
// identity, the setting of the shipped laplaceRHSinfer inputs.  This code and
// the oracle use the whole A^-1.

#include <algorithm>
#include <cmath>
#include <functional>
#include <new>
#include <vector>

#include "common.cuh"

struct sfc_perturbation {
    sfc_ctx *ctx = nullptr;
    sfc_forward_gauss *fg = nullptr;
    double reg = 1e-4;
    int rank = 0;
    sfc::DBuf<double> ke0;  // unit-conductivity element matrices
    std::vector<double> cent;  // element centroids, E x dim
    sfc::DBuf<double> cov, mean;
};

namespace sfc {
namespace {

// out[i][k ns + a] = sum_j K'_k[i][j] free(j) R[j][a]  (CSR values of K'_k in vals[k])
__global__ void k_spmm_multi(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                             const double *__restrict__ vals, int64_t nnz, const double *__restrict__ R,
                             const unsigned char *__restrict__ mask, int64_t N, int ns, int kc,
                             double *__restrict__ out)
{
    const int64_t total = N * kc * ns;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ((int64_t)kc * ns);
        const int rem = (int)(t - i * kc * ns), k = rem / ns, a = rem - k * ns;
        const double *v = vals + (int64_t)k * nnz;
        double acc = 0.0;
        for (int32_t s = rp[i]; s < rp[i + 1]; ++s) {
            const int32_t j = col[s];
            if (!mask[j]) acc += v[s] * R[(int64_t)j * ns + a];
        }
        out[t] = acc;
    }
}

__global__ void k_scale_rows_w(const double *__restrict__ X, const double *__restrict__ phibar, int64_t N, int64_t w,
                               double *__restrict__ out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * w; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = phibar[t / w] * X[t];
}

// V[c] = sum_i X[i][c] u[i]
__global__ void k_coldot(const double *__restrict__ X, const double *__restrict__ u, int64_t N, int64_t w,
                         double *__restrict__ V)
{
    for (int64_t c = blockIdx.x; c < w; c += gridDim.x) {
        double acc = 0.0;
        for (int64_t i = threadIdx.x; i < N; i += blockDim.x) acc += X[i * w + c] * u[i];
        __shared__ double sh[32];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            acc = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (threadIdx.x == 0) V[c] = acc;
        }
        __syncthreads();
    }
}

__global__ void k_add_scaled2(double *__restrict__ y, const double *__restrict__ x, double a, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        y[t] += a * x[t];
}

// pivoted Cholesky of sigma^2 exp(-|c_e - c_d|^2 / (2 l^2)) over the
// centroids (E x dim), greedy on the largest remaining diagonal, until it
// drops below rel * sigma^2 or max_rank columns; returns L (E x r, column k
// contiguous)
std::vector<double> material_factor(const std::vector<double> &cent, int dim, double sigma, double length,
                                    double rel, int max_rank, int &rank)
{
    const int64_t E = (int64_t)cent.size() / dim;
    const double s2 = sigma * sigma, inv = 1.0 / (2.0 * length * length);
    std::vector<double> d(E, s2);
    std::vector<std::vector<double>> cols;
    const double stop = rel * s2;
    while ((int)cols.size() < max_rank) {
        const int64_t j = std::max_element(d.begin(), d.end()) - d.begin();
        if (!(d[j] > stop)) break;
        std::vector<double> c(E);
        const double piv = std::sqrt(d[j]);
        for (int64_t e = 0; e < E; ++e) {
            double dd = 0.0;
            for (int q = 0; q < dim; ++q) {
                const double t = cent[e * dim + q] - cent[j * dim + q];
                dd += t * t;
            }
            double v = s2 * std::exp(-dd * inv);
            for (const auto &pc : cols) v -= pc[e] * pc[j];
            c[e] = v / piv;
        }
        for (int64_t e = 0; e < E; ++e) d[e] = std::max(d[e] - c[e] * c[e], 0.0);
        d[j] = 0.0;
        cols.push_back(std::move(c));
    }
    rank = (int)cols.size();
    std::vector<double> L((size_t)E * rank);
    for (int k = 0; k < rank; ++k)
        for (int64_t e = 0; e < E; ++e) L[(size_t)k * E + e] = cols[k][e];  // column-major: column k contiguous
    return L;
}

}  // namespace

void perturbation_update(sfc_perturbation *pt, const sfc_hparams_t *hp, double msigma, double mlength, double rel,
                         int max_rank)
{
    sfc_ctx *ctx = pt->ctx;
    sfc_forward_gauss *fg = pt->fg;
    sfc_system *s = fg->sys;
    const sfc_mesh *m = fg->cf->mesh;
    SFC_REQUIRE(m, "the covariance object has no mesh");
    SFC_REQUIRE(m->dof == 1, "material perturbation is defined for the Poisson element kinds");
    const int64_t N = s->N, ns = fg->ns, E = m->num_elems;
    // R^T = A^-T P^T, mean = R F (ForwardGaussRHS update) and u = A^-1 F
    forward_gauss_update(fg, hp);
    solve_forward(s);
    build_operator(s);
    if (!pt->ke0.p) {
        pt->ke0.alloc(E * m->L * m->L);
        element_matrices_unit(m, pt->ke0.p);
        std::vector<uint32_t> conn(E * m->nn);
        download(ctx, conn.data(), m->conn.p, conn.size());
        pt->cent.assign(E * m->dim, 0.0);
        for (int64_t e = 0; e < E; ++e)
            for (int a = 0; a < m->nn; ++a)
                for (int q = 0; q < m->dim; ++q)
                    pt->cent[e * m->dim + q] += m->h_coords[(size_t)conn[e * m->nn + a] * 3 + q] / m->nn;
    }
    int r = 0;
    const std::vector<double> L = material_factor(pt->cent, m->dim, msigma, mlength, rel, max_rank, r);
    pt->rank = r;
    DBuf<double> Ld;
    upload(ctx, Ld, L.data(), L.size());
    // C_s = R C_f R^T + (reg sigma_m)^2 P P^T + material term
    pt->cov.alloc(ns * ns);
    DBuf<double> work;
    projected_covar(ctx, fg->cf, hp->forcing_sigma, hp->forcing_length, fg->R.p, ns, pt->cov.p, work);
    const double add = pt->reg * msigma;
    k_add_scaled2<<<grid_for(ns * ns, 256), 256, 0, ctx->stream>>>(pt->cov.p, fg->d_ppt.p, add * add, ns * ns);
    count_launch(ctx);
    // chunks of kc factor columns: kc * ns right-hand sides per block solve
    int64_t kcap = std::min<int64_t>(4096 / std::max<int64_t>(ns, 1), (int64_t)(64e6 / std::max<int64_t>(N * ns, 1)));
    if (!m->is_grid) kcap = std::min<int64_t>(kcap, 256 / std::max<int64_t>(ns, 1));  // dense kernel: <= 256 columns
    const int kc_max = (int)std::max<int64_t>(1, kcap);
    DBuf<double> vals, Bt, Y, W, T, V;
    for (int k0 = 0; k0 < r; k0 += kc_max) {
        const int kc = std::min(kc_max, r - k0);
        const int64_t w = (int64_t)kc * ns;
        vals.reserve((size_t)m->nnz * kc);
        gather_weighted(m, pt->ke0.p, Ld.p + (size_t)k0 * E, kc, vals.p);
        Bt.reserve(N * w);
        k_spmm_multi<<<grid_for(N * w, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, vals.p, m->nnz, fg->R.p,
                                                                    s->mask.p, N, (int)ns, kc, Bt.p);
        count_launch(ctx);
        // (B_k u)(B_k u)^T
        V.reserve(w);
        k_coldot<<<(unsigned)std::min<int64_t>(w, 4096), 256, 0, ctx->stream>>>(Bt.p, s->X.p, N, w, V.p);
        count_launch(ctx);
        atb_accumulate(ctx, V.p, V.p, kc, ns, ns, pt->cov.p);
        // Y = A^-T B^T (one block adjoint solve), then Y^T C_f Y per k
        Y.reserve(N * w);
        solve_block(s, Bt.p, Y.p, (int)w, (int)w);
        transpose_fixup(s, Bt.p, Y.p, (int)w, (int)w);
        W.reserve(N * w);
        T.reserve(2 * N * w);
        k_scale_rows_w<<<grid_for(N * w, 256), 256, 0, ctx->stream>>>(Y.p, fg->cf->phibar.p, N, w, W.p);
        count_launch(ctx);
        kernel_times(ctx, fg->cf, hp->forcing_sigma, hp->forcing_length, W.p, T.p, w, T.p + N * w);
        // rows (i, k) of the N x (kc ns) arrays are the rows of an (N kc) x ns matrix
        atb_accumulate(ctx, W.p, T.p, N * kc, ns, ns, pt->cov.p);
    }
    pt->mean.alloc(ns);
    SFC_CK(cudaMemcpyAsync(pt->mean.p, fg->mean.p, ns * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    SFC_CK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace sfc

using namespace sfc;

namespace sfc {
namespace {
int pguard(sfc_ctx *ctx, const std::function<void()> &fn)
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

int32_t sfc_perturbation_create(sfc_forward_gauss_t *fg, double reg, sfc_perturbation_t **out)
{
    if (!fg || !out || !(reg >= 0)) return SFC_ERR_BAD_ARG;
    *out = nullptr;
    sfc_perturbation *pt = new (std::nothrow) sfc_perturbation();
    if (!pt) return SFC_ERR_NO_MEMORY;
    pt->ctx = fg->ctx;
    pt->fg = fg;
    pt->reg = reg;
    *out = pt;
    return SFC_OK;
}

int32_t sfc_perturbation_destroy(sfc_perturbation_t *pt)
{
    if (!pt) return SFC_OK;
    cudaSetDevice(pt->ctx->device);
    cudaStreamSynchronize(pt->ctx->stream);
    delete pt;
    return SFC_OK;
}

int32_t sfc_perturbation_update(sfc_perturbation_t *pt, const sfc_hparams_t *hp, double material_sigma,
                                double material_length, double factor_tol, int32_t max_rank, int32_t *rank)
{
    if (!pt || !hp || !(material_sigma >= 0) || !(material_length > 0) || !(factor_tol > 0) || max_rank <= 0)
        return SFC_ERR_BAD_ARG;
    return pguard(pt->ctx, [&] {
        perturbation_update(pt, hp, material_sigma, material_length, factor_tol, max_rank);
        if (rank) *rank = pt->rank;
    });
}

int32_t sfc_perturbation_mean(const sfc_perturbation_t *pt, double *mean)
{
    if (!pt || !mean || !pt->mean.p) return SFC_ERR_BAD_ARG;
    return pguard(pt->ctx, [&] { download(pt->ctx, mean, pt->mean.p, pt->fg->ns); });
}

int32_t sfc_perturbation_covar(const sfc_perturbation_t *pt, double *cov)
{
    if (!pt || !cov || !pt->cov.p) return SFC_ERR_BAD_ARG;
    return pguard(pt->ctx, [&] { download(pt->ctx, cov, pt->cov.p, (size_t)pt->fg->ns * pt->fg->ns); });
}

}  // extern "C"
