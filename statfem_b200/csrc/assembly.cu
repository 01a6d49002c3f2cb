// Element matrices, loads, sparse assembly and Dirichlet constraints on the GPU.
//
// The floating-point expressions follow the reference line for line (cited at
// each kernel) with every multiply / add / divide issued as an explicitly
// rounded intrinsic (__dmul_rn, __dadd_rn, ...) so that the compiler cannot
// contract them into FMAs: the element matrices and the assembled CSR values
// are therefore bit-identical to a plain C evaluation of the same expressions
// in the same order.  Inner products that the reference hands to Eigen's
// fixed-size evaluator use Eigen's unrolled pairwise reduction order.
//
// Assembly is "sorted-key" (gather) assembly: a one-time symbolic phase sorts
// every element-entry key (row, col) with a stable radix sort, which gives the
// CSR pattern of the merged triplets (corlib/Triplet.hpp:126-170) and, per CSR
// slot, the list of element entries that sum into it in element order.  The
// numeric phase writes element matrices to a buffer and one thread per CSR
// slot sums its list in that order: deterministic, no atomics.

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace sfc {

// ---------------------------------------------------------------------------
// element traits and quadrature tables
// ---------------------------------------------------------------------------
int elem_dim(int kind) { return kind == SFC_ELEM_LINE2_POISSON ? 1 : kind == SFC_ELEM_TRI3_POISSON ? 2 : 3; }
int elem_nodes(int kind) { return kind == SFC_ELEM_LINE2_POISSON ? 2 : kind == SFC_ELEM_TRI3_POISSON ? 3 : 8; }
int elem_dofs(int kind) { return kind == SFC_ELEM_HEX8_ELASTIC ? 3 : 1; }

// Gauss-Legendre rules on (0,1), descending points, the reference's 15-digit
// literals (corlib/GaussLegendre.hpp:65-100).
static int gauss_legendre(int n, double *w, double *x)
{
    static const double W[5][5] = {
        {1, 0, 0, 0, 0},
        {0.5, 0.5, 0, 0, 0},
        {0.277777777777777, 0.444444444444444, 0.277777777777777, 0, 0},
        {0.173927422568727, 0.326072577431273, 0.326072577431273, 0.173927422568727, 0},
        {0.118463442528095, 0.239314335249683, 0.284444444444444, 0.239314335249683, 0.118463442528095}};
    static const double X[5][5] = {
        {0.5, 0, 0, 0, 0},
        {0.788675134594813, 0.211324865405187, 0, 0, 0},
        {0.887298334620741, 0.5, 0.112701665379259, 0, 0},
        {0.930568155797026, 0.669990521792428, 0.330009478207572, 0.069431844202974, 0},
        {0.953089922969332, 0.769234655052841, 0.5, 0.230765344947159, 0.046910077030668}};
    if (n < 1 || n > 5) return 0;
    for (int i = 0; i < n; ++i) {
        w[i] = W[n - 1][i];
        x[i] = X[n - 1][i];
    }
    return n;
}

// Shape functions and their reference gradients at xi
// (corlib/Shapefun.ipp: line :36-49, triangle :180-196, hexahedron :926-975).
static void shape_host(int kind, const double *xi, double *phi, double d[3][8])
{
    std::memset(d, 0, sizeof(double) * 24);
    if (kind == SFC_ELEM_LINE2_POISSON) {
        phi[0] = 1. - xi[0];
        phi[1] = xi[0];
        d[0][0] = -1.;
        d[0][1] = 1.;
    } else if (kind == SFC_ELEM_TRI3_POISSON) {
        phi[0] = 1. - (xi[0] + xi[1]);
        phi[1] = xi[0];
        phi[2] = xi[1];
        d[0][0] = -1.; d[0][1] = 1.; d[0][2] = 0.;
        d[1][0] = -1.; d[1][1] = 0.; d[1][2] = 1.;
    } else {
        const double x = xi[0], y = xi[1], z = xi[2];
        phi[0] = (1. - x) * (1. - y) * (1. - z);
        phi[1] = x * (1. - y) * (1. - z);
        phi[2] = x * y * (1. - z);
        phi[3] = (1. - x) * y * (1. - z);
        phi[4] = (1. - x) * (1. - y) * z;
        phi[5] = x * (1. - y) * z;
        phi[6] = x * y * z;
        phi[7] = (1. - x) * y * z;
        d[0][0] = -(1. - y) * (1. - z);
        d[0][1] = (1. - y) * (1. - z);
        d[0][2] = y * (1. - z);
        d[0][3] = -y * (1. - z);
        d[0][4] = -(1. - y) * z;
        d[0][5] = (1. - y) * z;
        d[0][6] = y * z;
        d[0][7] = -y * z;
        d[1][0] = -(1. - x) * (1. - z);
        d[1][1] = -x * (1. - z);
        d[1][2] = x * (1. - z);
        d[1][3] = (1. - x) * (1. - z);
        d[1][4] = -(1. - x) * z;
        d[1][5] = -x * z;
        d[1][6] = x * z;
        d[1][7] = (1. - x) * z;
        d[2][0] = -(1. - x) * (1. - y);
        d[2][1] = -x * (1. - y);
        d[2][2] = -x * y;
        d[2][3] = -(1. - x) * y;
        d[2][4] = (1. - x) * (1. - y);
        d[2][5] = x * (1. - y);
        d[2][6] = x * y;
        d[2][7] = (1. - x) * y;
    }
}

// Quadrature<SHAPE,QPS> point / weight tables:
//   line:       SimplexQuadratureConstructor<1,QPS> = GL<QPS> (corlib/SimplexQuadrature.hpp:97-106)
//   triangle:   SimplexQuadratureConstructor<2,1|3> (corlib/SimplexQuadrature.hpp:160-191)
//   hexahedron: TensorQuadratureConstructor<GL<n>,3>, weight (w_i*w_j)*w_k,
//               first coordinate fastest (corlib/TensorQuadrature.hpp:101-139)
void make_quadrature(int kind, int qps, QuadTable &t)
{
    std::memset(&t, 0, sizeof t);
    double gw[5], gx[5];
    if (kind == SFC_ELEM_LINE2_POISSON) {
        int n = gauss_legendre(qps, gw, gx);
        SFC_REQUIRE(n > 0, "line quadrature supports 1..5 points");
        t.nq = n;
        for (int i = 0; i < n; ++i) {
            t.w[i] = gw[i];
            t.xi[i][0] = gx[i];
        }
    } else if (kind == SFC_ELEM_TRI3_POISSON) {
        if (qps == 1) {
            t.nq = 1;
            t.w[0] = 0.5;
            t.xi[0][0] = 0.333333333333333;
            t.xi[0][1] = 0.333333333333333;
        } else if (qps == 3) {
            t.nq = 3;
            const double a = 0.666666666666667, b = 0.166666666666667;
            t.w[0] = t.w[1] = t.w[2] = 0.166666666666666;
            t.xi[0][0] = a; t.xi[0][1] = b;
            t.xi[1][0] = b; t.xi[1][1] = a;
            t.xi[2][0] = b; t.xi[2][1] = b;
        } else {
            fail(SFC_ERR_BAD_ARG, "triangle quadrature supports 1 or 3 points");
        }
    } else if (kind == SFC_ELEM_HEX8_POISSON || kind == SFC_ELEM_HEX8_ELASTIC) {
        int n = 0;
        for (int c = 1; c <= 3; ++c)
            if (c * c * c == qps) n = c;
        SFC_REQUIRE(n > 0, "hexahedron quadrature supports 1, 8 or 27 points");
        gauss_legendre(n, gw, gx);
        t.nq = n * n * n;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    int q = (k * n + j) * n + i;
                    t.w[q] = (gw[i] * gw[j]) * gw[k];
                    t.xi[q][0] = gx[i];
                    t.xi[q][1] = gx[j];
                    t.xi[q][2] = gx[k];
                }
    } else {
        fail(SFC_ERR_BAD_ARG, "unknown element kind");
    }
    for (int q = 0; q < t.nq; ++q) shape_host(kind, t.xi[q], t.phi[q], t.dphi[q]);
}

// ---------------------------------------------------------------------------
// device arithmetic helpers: explicitly rounded, never contracted
// ---------------------------------------------------------------------------
__device__ __forceinline__ double MUL(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ADD(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double SUB(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double DIV(double a, double b) { return __ddiv_rn(a, b); }

// Eigen's unrolled pairwise reduction for the lengths that occur here
template <int N>
__device__ __forceinline__ double redux(const double *t);
template <> __device__ __forceinline__ double redux<1>(const double *t) { return t[0]; }
template <> __device__ __forceinline__ double redux<2>(const double *t) { return ADD(t[0], t[1]); }
template <> __device__ __forceinline__ double redux<3>(const double *t) { return ADD(t[0], ADD(t[1], t[2])); }
template <> __device__ __forceinline__ double redux<8>(const double *t)
{
    return ADD(ADD(ADD(t[0], t[1]), ADD(t[2], t[3])), ADD(ADD(t[4], t[5]), ADD(t[6], t[7])));
}

// determinant (corlib/linalg.hpp:47-74), row-major D x D
template <int D>
__device__ __forceinline__ double det_rm(const double *m)
{
    if (D == 1) return m[0];
    if (D == 2) return SUB(MUL(m[0], m[3]), MUL(m[1], m[2]));
    double r = ADD(MUL(MUL(m[0], m[4]), m[8]), MUL(MUL(m[1], m[5]), m[6]));
    r = ADD(r, MUL(MUL(m[2], m[3]), m[7]));
    r = SUB(r, MUL(MUL(m[0], m[5]), m[7]));
    r = SUB(r, MUL(MUL(m[1], m[3]), m[8]));
    r = SUB(r, MUL(MUL(m[2], m[4]), m[6]));
    return r;
}

// in-place inverse returning the determinant (corlib/linalg.hpp:100-152)
template <int D>
__device__ __forceinline__ double inverse_rm(double *m)
{
    const double det = det_rm<D>(m);
    if (D == 1) {
        m[0] = DIV(1., det);
    } else if (D == 2) {
        const double aux = m[0];
        m[0] = DIV(m[3], det);
        m[1] = DIV(m[1], -det);
        m[2] = DIV(m[2], -det);
        m[3] = DIV(aux, det);
    } else {
        double t[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) t[i] = m[i];
        m[0] = DIV(SUB(MUL(t[4], t[8]), MUL(t[5], t[7])), det);
        m[4] = DIV(SUB(MUL(t[0], t[8]), MUL(t[2], t[6])), det);
        m[8] = DIV(SUB(MUL(t[0], t[4]), MUL(t[1], t[3])), det);
        m[1] = DIV(SUB(MUL(t[2], t[7]), MUL(t[1], t[8])), det);
        m[2] = DIV(SUB(MUL(t[1], t[5]), MUL(t[2], t[4])), det);
        m[3] = DIV(SUB(MUL(t[5], t[6]), MUL(t[3], t[8])), det);
        m[5] = DIV(SUB(MUL(t[2], t[3]), MUL(t[0], t[5])), det);
        m[6] = DIV(SUB(MUL(t[3], t[7]), MUL(t[4], t[6])), det);
        m[7] = DIV(SUB(MUL(t[1], t[6]), MUL(t[0], t[7])), det);
    }
    return det;
}

// covariant basis G[i][a] = sum_K X[K][i] dphi[a][K]  (X * dphiDxi^T)
template <int D, int NN>
__device__ __forceinline__ void covariant(const double (*X)[3], const double (*dphi)[8], double *G)
{
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int a = 0; a < D; ++a) {
            double t[NN];
#pragma unroll
            for (int K = 0; K < NN; ++K) t[K] = MUL(X[K][i], dphi[a][K]);
            G[i * D + a] = redux<NN>(t);
        }
}

// ElementBasic::globalDerivatives (corlib/ElementBasic.ipp:178-204) with
// ContraVariantBasis<D,D> (corlib/linalg.hpp:200-217): contra = (G^T)^-1,
// dx[i][K] = sum_a contra[i][a] dphi[a][K]; returns det(G^T).
template <int D, int NN>
__device__ __forceinline__ double global_derivatives(const double (*X)[3], const double (*dphi)[8],
                                                     double (*dx)[8])
{
    double G[D * D], C[D * D];
    covariant<D, NN>(X, dphi, G);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int a = 0; a < D; ++a) C[i * D + a] = G[a * D + i];
    const double det = inverse_rm<D>(C);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int K = 0; K < NN; ++K) {
            double t[D];
#pragma unroll
            for (int a = 0; a < D; ++a) t[a] = MUL(C[i * D + a], dphi[a][K]);
            dx[i][K] = redux<D>(t);
        }
    return det;
}

// ElementBasic::jacobian (corlib/ElementBasic.ipp:132-153): determinant of G
template <int D, int NN>
__device__ __forceinline__ double jacobian(const double (*X)[3], const double (*dphi)[8])
{
    double G[D * D];
    covariant<D, NN>(X, dphi, G);
    return det_rm<D>(G);
}

// ---------------------------------------------------------------------------
// element matrices
// ---------------------------------------------------------------------------

// Poisson element matrix, one thread per element (L = NN <= 8):
// Ke = 0; per quadrature point Ke += ((kappa*detJ)*w) * (dphiDx^T dphiDx)
// (del2/fem/ElementPotential.ipp:58-74, corlib/ComputeElementMatrix.hpp:62-77,
// corlib/MatrixAssembler.hpp:213-220).  Ke is exactly symmetric (products
// commute), so the upper triangle is computed and mirrored.
template <int D, int NN>
__global__ void __launch_bounds__(128) k_elem_poisson(const double *__restrict__ coords,
                                                      const uint32_t *__restrict__ conn,
                                                      const double *__restrict__ coeff, const QuadTable qt,
                                                      int64_t E, double *__restrict__ ke, int *err)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        double X[NN][3];
#pragma unroll
        for (int K = 0; K < NN; ++K) {
            const double *p = coords + 3 * (int64_t)conn[e * NN + K];
            X[K][0] = p[0];
            X[K][1] = p[1];
            X[K][2] = p[2];
        }
        const double kappa = coeff[e];
        double Ke[NN * (NN + 1) / 2];
#pragma unroll
        for (int i = 0; i < NN * (NN + 1) / 2; ++i) Ke[i] = 0.0;
        for (int q = 0; q < qt.nq; ++q) {
            double dx[D][8];
            const double det = global_derivatives<D, NN>(X, qt.dphi[q], dx);
            if (!(det > 0.)) atomicExch(err, 1);
            const double s = MUL(MUL(kappa, det), qt.w[q]);
            int u = 0;
#pragma unroll
            for (int m = 0; m < NN; ++m)
#pragma unroll
                for (int n = m; n < NN; ++n) {
                    double t[D];
#pragma unroll
                    for (int a = 0; a < D; ++a) t[a] = MUL(dx[a][m], dx[a][n]);
                    Ke[u] = ADD(Ke[u], MUL(s, redux<D>(t)));
                    ++u;
                }
        }
        double *out = ke + e * (NN * NN);
        int u = 0;
#pragma unroll
        for (int m = 0; m < NN; ++m)
#pragma unroll
            for (int n = m; n < NN; ++n) {
                out[m * NN + n] = Ke[u];
                out[n * NN + m] = Ke[u];
                ++u;
            }
    }
}

// Elasticity element matrix (24 x 24), one warp per element.  Reference:
// solid/fem/ElementStatic.ipp:286-320 with SVenant::elasticityTensor at F = I
// (solid/material/svenant/SVenant.ipp:107-140):
//   K[m*3+i][n*3+k] += (kentry*detJ)*w,  kentry = sum_J sum_L (C_iJkL*a_J)*b_L
// with C_iJkL = lambda d_iJ d_kL + mu d_iL d_kJ + mu d_JL d_ik.  Terms with
// C = 0 add signed zeros, which never change the running sum, so only the
// nonzero terms are evaluated, in the same (J, L) order.
// Lanes 0..nq-1 evaluate the geometry of one quadrature point each into shared
// memory; every lane then owns two (m, n) node pairs (9 entries each).
constexpr int kElasticWarps = 4;

__global__ void __launch_bounds__(32 * kElasticWarps) k_elem_elastic(const double *__restrict__ coords,
                                                                     const uint32_t *__restrict__ conn,
                                                                     const double *__restrict__ coeff, double nu,
                                                                     const QuadTable qt, int64_t E,
                                                                     double *__restrict__ ke, int *err)
{
    __shared__ double sX[kElasticWarps][8][3];
    __shared__ double sdx[kElasticWarps][8][3][8];
    __shared__ double sdet[kElasticWarps][8];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kElasticWarps;
    for (int64_t e = blockIdx.x * (int64_t)kElasticWarps + wid; e < E; e += nwarps) {
        if (lane < 8) {
            const double *p = coords + 3 * (int64_t)conn[e * 8 + lane];
            sX[wid][lane][0] = p[0];
            sX[wid][lane][1] = p[1];
            sX[wid][lane][2] = p[2];
        }
        __syncwarp();
        if (lane < qt.nq) {
            double dx[3][8];
            const double det = global_derivatives<3, 8>(sX[wid], qt.dphi[lane], dx);
            if (!(det > 0.)) atomicExch(err, 1);
            sdet[wid][lane] = det;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int K = 0; K < 8; ++K) sdx[wid][lane][i][K] = dx[i][K];
        }
        __syncwarp();
        // Lame constants, SVenant.ipp:32-37
        const double Ey = coeff[e];
        const double lambda = DIV(DIV(MUL(Ey, nu), ADD(1.0, nu)), SUB(1.0, MUL(2.0, nu)));
        const double mu = DIV(DIV(Ey, 2.0), ADD(1.0, nu));
        const double cdd = ADD(ADD(lambda, mu), mu);  // C_iiii
        double acc[2][3][3];
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) acc[j][i][k] = 0.0;
        for (int q = 0; q < qt.nq; ++q) {
            const double det = sdet[wid][q], w = qt.w[q];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int p = lane + 32 * j, m = p >> 3, n = p & 7;
                double a[3], b[3];
#pragma unroll
                for (int J = 0; J < 3; ++J) {
                    a[J] = sdx[wid][q][J][m];
                    b[J] = sdx[wid][q][J][n];
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        double kentry;
                        if (i == k) {
                            double t0 = MUL(MUL(i == 0 ? cdd : mu, a[0]), b[0]);
                            double t1 = MUL(MUL(i == 1 ? cdd : mu, a[1]), b[1]);
                            double t2 = MUL(MUL(i == 2 ? cdd : mu, a[2]), b[2]);
                            kentry = ADD(ADD(t0, t1), t2);
                        } else {
                            const double tl = MUL(MUL(lambda, a[i]), b[k]);  // J = i, L = k
                            const double tm = MUL(MUL(mu, a[k]), b[i]);      // J = k, L = i
                            kentry = i < k ? ADD(tl, tm) : ADD(tm, tl);
                        }
                        acc[j][i][k] = ADD(acc[j][i][k], MUL(MUL(kentry, det), w));
                    }
            }
        }
        double *out = ke + e * 576;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int p = lane + 32 * j, m = p >> 3, n = p & 7;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) out[(m * 3 + i) * 24 + n * 3 + k] = acc[j][i][k];
        }
        __syncwarp();
    }
}

// CSR slot s = sum of its element entries in element order, starting at 0.0
// (Triplet::combineTriplets_, corlib/Triplet.hpp:565-580).
__global__ void k_gather(const int32_t *__restrict__ slot_ptr, const int32_t *__restrict__ contrib,
                         const double *__restrict__ ke, int64_t nnz, double *__restrict__ a)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nnz; s += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        const int32_t b = slot_ptr[s], t1 = slot_ptr[s + 1];
        for (int32_t t = b; t < t1; ++t) v = ADD(v, ke[contrib[t]]);
        a[s] = v;
    }
}

// ---------------------------------------------------------------------------
// body-force load: one thread per node, sums its elements' quadrature-point
// contributions in element order, then quadrature order -- the order in which
// Node::addToForce receives them (corlib/Integrator.hpp:61-73).  Per point:
// ((w*detJ)*factor) * (f_c*phi_n)  (del2/fem/ElementPotential.ipp:149-176;
// solid/fem/ElementStatic.ipp:441-466), factor = 1.
// ---------------------------------------------------------------------------
template <int D, int NN>
__global__ void k_load(const double *__restrict__ coords, const uint32_t *__restrict__ conn,
                       const int32_t *__restrict__ node_ptr, const int32_t *__restrict__ node_elem,
                       const QuadTable qt, int64_t num_nodes, int dof, double f0, double f1, double f2,
                       double *__restrict__ F)
{
    const double f[3] = {f0, f1, f2};
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < num_nodes;
         nd += (int64_t)gridDim.x * blockDim.x) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int32_t t = node_ptr[nd]; t < node_ptr[nd + 1]; ++t) {
            const int32_t ek = node_elem[t];
            const int64_t e = ek / NN;
            const int k = ek - (int)(e * NN);
            double X[NN][3];
#pragma unroll
            for (int K = 0; K < NN; ++K) {
                const double *p = coords + 3 * (int64_t)conn[e * NN + K];
                X[K][0] = p[0];
                X[K][1] = p[1];
                X[K][2] = p[2];
            }
            for (int q = 0; q < qt.nq; ++q) {
                const double det = jacobian<D, NN>(X, qt.dphi[q]);
                const double s = MUL(MUL(qt.w[q], det), 1.0);
                for (int c = 0; c < dof; ++c) acc[c] = ADD(acc[c], MUL(s, MUL(f[c], qt.phi[q][k])));
            }
        }
        for (int c = 0; c < dof; ++c) F[nd * dof + c] = ADD(F[nd * dof + c], acc[c]);
    }
}

// ---------------------------------------------------------------------------
// constraints and the SPD operator
// ---------------------------------------------------------------------------

// Triplet::zeroRow (corlib/Triplet.hpp:219-260) + F[c] = (factor*value)*scalar
// (corlib/SystemSolveEigenSparse.hpp:197-215)
__global__ void k_constraints(const uint32_t *__restrict__ idx, const double *__restrict__ val, int64_t n,
                              const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
                              double *__restrict__ a_ref, double *__restrict__ F, unsigned char *mask,
                              double *bc_val, double factor, double scalar, int64_t N, int *err)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = idx[t];
        if (c >= N) {
            atomicExch(err, 2);
            continue;
        }
        bool found = false;
        for (int32_t s = row_ptr[c]; s < row_ptr[c + 1]; ++s) {
            if (col[s] == c) {
                a_ref[s] = scalar;
                found = true;
            } else {
                a_ref[s] = 0.0;
            }
        }
        if (!found) atomicExch(err, 3);
        const double v = val ? MUL(factor, val[t]) : 0.0;
        F[c] = MUL(v, scalar);
        mask[c] = 1;
        bc_val[c] = v;
    }
}

// symmetric elimination: free rows drop constrained columns, constrained rows
// keep only their diagonal; Jacobi inverse diagonal; FP32 copies.
__global__ void k_build_op(const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
                           const int32_t *__restrict__ diag, const double *__restrict__ a_ref,
                           const unsigned char *__restrict__ mask, int64_t N, double *__restrict__ a_op,
                           float *__restrict__ a_op32, double *__restrict__ dinv, float *__restrict__ dinv32,
                           int *err)
{
    // warp per row, lanes over the row's entries (coalesced)
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        const bool mi = mask[i];
        for (int32_t s = row_ptr[i] + lane; s < row_ptr[i + 1]; s += 32) {
            const int32_t j = col[s];
            double v = a_ref[s];
            if ((mi || mask[j]) && j != i) v = 0.0;
            a_op[s] = v;
            a_op32[s] = (float)v;
        }
        if (lane) continue;
        const int32_t d = diag[i];
        if (d < 0) {
            atomicExch(err, 4);
            continue;
        }
        const double dv = a_ref[d];
        if (!(dv > 0.0)) atomicExch(err, 5);
        dinv[i] = 1.0 / dv;
        dinv32[i] = (float)(1.0 / dv);
    }
}

// ---------------------------------------------------------------------------
// symbolic phase helpers
// ---------------------------------------------------------------------------
__global__ void k_entry_keys(const uint32_t *__restrict__ conn, int64_t E, int nn, int dof, int L, int64_t N,
                             uint64_t *__restrict__ keys, int32_t *__restrict__ ids)
{
    const int64_t LL = (int64_t)L * L, M = E * LL;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / LL;
        const int rc = (int)(t - e * LL), r = rc / L, c = rc - r * L;
        const uint64_t row = (uint64_t)conn[e * nn + r / dof] * dof + (r % dof);
        const uint64_t cl = (uint64_t)conn[e * nn + c / dof] * dof + (c % dof);
        keys[t] = row * (uint64_t)N + cl;
        ids[t] = (int32_t)t;
    }
}

__global__ void k_flag_unique(const uint64_t *__restrict__ keys, int64_t M, int32_t *__restrict__ flag)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M; t += (int64_t)gridDim.x * blockDim.x)
        flag[t] = (t == 0 || keys[t] != keys[t - 1]) ? 1 : 0;
}

// slot = inclusive-scan(flag) - 1; write col / slot_ptr / row boundaries
__global__ void k_emit_pattern(const uint64_t *__restrict__ keys, const int32_t *__restrict__ flag,
                               const int32_t *__restrict__ slot, int64_t M, int64_t N, int32_t *__restrict__ col,
                               int32_t *__restrict__ slot_ptr, int32_t *__restrict__ slot_row)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M; t += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[t]) continue;
        const int32_t s = slot[t] - 1;
        col[s] = (int32_t)(keys[t] % (uint64_t)N);
        slot_row[s] = (int32_t)(keys[t] / (uint64_t)N);
        slot_ptr[s] = (int32_t)t;
    }
}

// row_ptr from the (sorted) row of every slot; diagonal slots
__global__ void k_row_ptr(const int32_t *__restrict__ slot_row, const int32_t *__restrict__ col, int64_t nnz,
                          int64_t N, int32_t *__restrict__ row_ptr, int32_t *__restrict__ diag)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nnz; s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = slot_row[s];
        const int32_t rp = s == 0 ? -1 : slot_row[s - 1];
        for (int32_t rr = rp + 1; rr <= r; ++rr) row_ptr[rr] = (int32_t)s;
        if (s == nnz - 1)
            for (int64_t rr = r + 1; rr <= N; ++rr) row_ptr[rr] = (int32_t)nnz;
        if (col[s] == r) diag[r] = (int32_t)s;
    }
}

__global__ void k_fill_i32(int32_t *p, int64_t n, int32_t v)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) p[t] = v;
}

__global__ void k_node_keys(const uint32_t *__restrict__ conn, int64_t n, uint32_t *__restrict__ keys,
                            int32_t *__restrict__ ids)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        keys[t] = conn[t];
        ids[t] = (int32_t)t;
    }
}

__global__ void k_node_ptr(const uint32_t *__restrict__ keys, int64_t n, int64_t num_nodes,
                           int32_t *__restrict__ node_ptr)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = keys[t];
        const int64_t rp = t == 0 ? -1 : (int64_t)keys[t - 1];
        for (int64_t rr = rp + 1; rr <= r; ++rr) node_ptr[rr] = (int32_t)t;
        if (t == n - 1)
            for (int64_t rr = r + 1; rr <= num_nodes; ++rr) node_ptr[rr] = (int32_t)n;
    }
}

static int bits_for(uint64_t v)
{
    int b = 0;
    while (b < 64 && (v >> b)) ++b;
    return std::max(b, 1);
}

// Sort (key, id) pairs stably by key; merge equal keys into CSR slots.
// keys/ids are consumed.  Produces col, row_ptr, diag (num rows N), the slot
// pointer into the sorted id list and the sorted ids themselves.
static int64_t sort_and_merge(sfc_ctx *ctx, DBuf<uint64_t> &keys, DBuf<int32_t> &ids, int64_t M, int64_t N,
                              DBuf<int32_t> &row_ptr, DBuf<int32_t> &col, DBuf<int32_t> &diag,
                              DBuf<int32_t> &slot_ptr, DBuf<int32_t> &sorted_ids)
{
    DBuf<uint64_t> keys2;
    keys2.alloc(M);
    sorted_ids.alloc(M);
    const int end_bit = bits_for((uint64_t)N * (uint64_t)N - 1);
    size_t tmp = 0;
    SFC_CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, keys2.p, ids.p, sorted_ids.p, M, 0, end_bit,
                                           ctx->stream));
    ctx->scratch.reserve(tmp);
    SFC_CK(cub::DeviceRadixSort::SortPairs(ctx->scratch.p, tmp, keys.p, keys2.p, ids.p, sorted_ids.p, M, 0,
                                           end_bit, ctx->stream));
    count_launch(ctx, 4);
    ids.release();
    DBuf<int32_t> flag, slot;
    flag.alloc(M);
    slot.alloc(M);
    k_flag_unique<<<grid_for(M, 256), 256, 0, ctx->stream>>>(keys2.p, M, flag.p);
    count_launch(ctx);
    tmp = 0;
    SFC_CK(cub::DeviceScan::InclusiveSum(nullptr, tmp, flag.p, slot.p, M, ctx->stream));
    ctx->scratch.reserve(tmp);
    SFC_CK(cub::DeviceScan::InclusiveSum(ctx->scratch.p, tmp, flag.p, slot.p, M, ctx->stream));
    count_launch(ctx, 2);
    int32_t nnz32 = 0;
    download(ctx, &nnz32, slot.p + (M - 1), 1);
    const int64_t nnz = nnz32;
    col.alloc(nnz);
    slot_ptr.alloc(nnz + 1);
    DBuf<int32_t> slot_row;
    slot_row.alloc(nnz);
    k_emit_pattern<<<grid_for(M, 256), 256, 0, ctx->stream>>>(keys2.p, flag.p, slot.p, M, N, col.p, slot_ptr.p,
                                                             slot_row.p);
    count_launch(ctx);
    const int32_t Mi = (int32_t)M;
    SFC_CK(cudaMemcpyAsync(slot_ptr.p + nnz, &Mi, sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    row_ptr.alloc(N + 1);
    diag.alloc(N);
    k_fill_i32<<<grid_for(N, 256), 256, 0, ctx->stream>>>(diag.p, N, -1);
    count_launch(ctx);
    k_row_ptr<<<grid_for(nnz, 256), 256, 0, ctx->stream>>>(slot_row.p, col.p, nnz, N, row_ptr.p, diag.p);
    count_launch(ctx);
    SFC_CK(cudaStreamSynchronize(ctx->stream));
    return nnz;
}

// Tensor-grid test of the node set: node i sits at (ax0[i%n0], ax1[(i/n0)%n1],
// ax2[i/(n0 n1)]) exactly.  Used for the Kronecker form of the SE covariance.
static void detect_grid(sfc_mesh *m)
{
    m->is_grid = false;
    const int64_t n = m->num_nodes;
    std::vector<double> ax[3];
    for (int a = 0; a < m->dim; ++a) {
        std::vector<double> v(n);
        for (int64_t i = 0; i < n; ++i) v[i] = m->h_coords[3 * i + a];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        ax[a] = v;
    }
    int64_t prod = 1;
    for (int a = 0; a < m->dim; ++a) prod *= (int64_t)ax[a].size();
    if (prod != n) return;
    int gn[3] = {1, 1, 1};
    for (int a = 0; a < m->dim; ++a) gn[a] = (int)ax[a].size();
    for (int64_t i = 0; i < n; ++i) {
        int64_t r = i;
        for (int a = 0; a < m->dim; ++a) {
            const int64_t ia = r % gn[a];
            r /= gn[a];
            if (m->h_coords[3 * i + a] != ax[a][ia]) return;
        }
    }
    m->is_grid = true;
    for (int a = 0; a < 3; ++a) {
        m->gn[a] = gn[a];
        m->gaxis[a] = a < m->dim ? ax[a] : std::vector<double>{0.0};
    }
}

void build_pattern(sfc_mesh *m)
{
    sfc_ctx *ctx = m->ctx;
    const int64_t M = m->num_elems * m->L * m->L;
    // element entries, slots and CSR offsets are 32-bit: E * L^2 < 2^31 (about
    // 3.7 M elasticity hexahedra, a 155^3 mesh; 33 M P1 triangles)
    SFC_REQUIRE_SIZE(M < (int64_t)INT32_MAX, "more than 2^31 - 1 element-matrix entries (32-bit indices)");
    SFC_REQUIRE_SIZE(m->num_dofs < (int64_t)INT32_MAX, "more than 2^31 - 1 dofs (32-bit column indices)");
    {
        DBuf<uint64_t> keys;
        DBuf<int32_t> ids;
        keys.alloc(M);
        ids.alloc(M);
        k_entry_keys<<<grid_for(M, 256), 256, 0, ctx->stream>>>(m->conn.p, m->num_elems, m->nn, m->dof, m->L,
                                                                m->num_dofs, keys.p, ids.p);
        count_launch(ctx);
        m->nnz = sort_and_merge(ctx, keys, ids, M, m->num_dofs, m->row_ptr, m->col, m->diag, m->slot_ptr,
                                m->contrib);
        SFC_REQUIRE(m->nnz < (int64_t)INT32_MAX, "too many nonzeros for 32-bit indices");
    }
    {
        const int64_t n = m->num_elems * m->nn;
        DBuf<uint32_t> k1, k2;
        DBuf<int32_t> id1;
        k1.alloc(n);
        k2.alloc(n);
        id1.alloc(n);
        m->node_elem.alloc(n);
        k_node_keys<<<grid_for(n, 256), 256, 0, ctx->stream>>>(m->conn.p, n, k1.p, id1.p);
        count_launch(ctx);
        size_t tmp = 0;
        const int end_bit = bits_for((uint64_t)m->num_nodes);
        SFC_CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k1.p, k2.p, id1.p, m->node_elem.p, n, 0, end_bit,
                                               ctx->stream));
        ctx->scratch.reserve(tmp);
        SFC_CK(cub::DeviceRadixSort::SortPairs(ctx->scratch.p, tmp, k1.p, k2.p, id1.p, m->node_elem.p, n, 0,
                                               end_bit, ctx->stream));
        count_launch(ctx, 4);
        m->node_ptr.alloc(m->num_nodes + 1);
        k_node_ptr<<<grid_for(n, 256), 256, 0, ctx->stream>>>(k2.p, n, m->num_nodes, m->node_ptr.p);
        count_launch(ctx);
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    }
    detect_grid(m);
}

// ---------------------------------------------------------------------------
// numeric phase
// ---------------------------------------------------------------------------
void ensure_pattern_from_mesh(sfc_system *s, const sfc_mesh *m)
{
    SFC_REQUIRE(m->num_dofs == s->N, "mesh dof count differs from the system size");
    if (s->has_pattern && s->pattern_mesh == m) return;
    sfc_ctx *ctx = s->ctx;
    s->nnz = m->nnz;
    s->row_ptr.alloc(s->N + 1);
    s->col.alloc(s->nnz);
    s->diag.alloc(s->N);
    SFC_CK(cudaMemcpyAsync(s->row_ptr.p, m->row_ptr.p, (s->N + 1) * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    SFC_CK(cudaMemcpyAsync(s->col.p, m->col.p, s->nnz * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    SFC_CK(cudaMemcpyAsync(s->diag.p, m->diag.p, s->N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    s->a_ref.alloc(s->nnz);
    s->a_op.alloc(s->nnz);
    s->a_op32.alloc(s->nnz);
    SFC_CK(cudaMemsetAsync(s->a_ref.p, 0, s->nnz * 8, ctx->stream));
    s->has_pattern = true;
    s->pattern_mesh = m;
    s->coarse.built = false;  // aggregates belong to the installed mesh
    s->op_valid = false;
}

void assemble_matrix(sfc_system *s, const sfc_mesh *mc)
{
    sfc_mesh *m = const_cast<sfc_mesh *>(mc);
    sfc_ctx *ctx = s->ctx;
    SFC_REQUIRE(s->st_vals.empty(), "staged insertToMatrix entries pending; finish or clear them first");
    SFC_REQUIRE(m->coeff.p, "element coefficients not set");
    ensure_pattern_from_mesh(s, m);
    const int64_t E = m->num_elems;
    m->ke.alloc(E * m->L * m->L);
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    ProfScope ps_elem(ctx, "element_matrices",
                      (double)E * (m->nn * 4 + m->nn * 24 + 8) + (double)E * m->L * m->L * 8);
    switch (m->kind) {
    case SFC_ELEM_LINE2_POISSON:
        k_elem_poisson<1, 2><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->coeff.p, m->quad,
                                                                         E, m->ke.p, err.p);
        break;
    case SFC_ELEM_TRI3_POISSON:
        k_elem_poisson<2, 3><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->coeff.p, m->quad,
                                                                         E, m->ke.p, err.p);
        break;
    case SFC_ELEM_HEX8_POISSON:
        k_elem_poisson<3, 8><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->coeff.p, m->quad,
                                                                         E, m->ke.p, err.p);
        break;
    case SFC_ELEM_HEX8_ELASTIC:
        SFC_REQUIRE(m->quad.nq <= 8, "elastic kernel supports up to 8 quadrature points");
        k_elem_elastic<<<grid_for(E, kElasticWarps, 148 * 64), 32 * kElasticWarps, 0, ctx->stream>>>(
            m->coords.p, m->conn.p, m->coeff.p, m->nu, m->quad, E, m->ke.p, err.p);
        break;
    default:
        fail(SFC_ERR_BAD_ARG, "unknown element kind");
    }
    count_launch(ctx);
    {
        const double M = (double)E * m->L * m->L;
        ProfScope ps(ctx, "csr_gather", (double)s->nnz * 12 + M * 12);
        k_gather<<<grid_for(s->nnz, 256), 256, 0, ctx->stream>>>(m->slot_ptr.p, m->contrib.p, m->ke.p, s->nnz,
                                                                 s->a_ref.p);
    }
    count_launch(ctx);
    int h_err = 0;
    download(ctx, &h_err, err.p, 1);
    if (h_err) fail(SFC_ERR_NEG_JACOBIAN, "Negative Jacobian in an element");
    // a full assembly replaces the matrix: constraints must be applied again
    s->op_valid = false;
    if (s->mask.p) SFC_CK(cudaMemsetAsync(s->mask.p, 0, s->N, ctx->stream));
    s->any_constraint = false;
    s->inhomogeneous = false;
}

// Element matrices of the Poisson kinds with conductivity 1: the stiffness
// derivative d K_e / d kappa_e (ElementPotential::stiffnessDerivIntegrand,
// del2/fem/ElementPotential.ipp:225-237, 1.0 * detG * w * dphiDx^T dphiDx)
void element_matrices_unit(const sfc_mesh *m, double *ke0)
{
    sfc_ctx *ctx = m->ctx;
    const int64_t E = m->num_elems;
    DBuf<double> ones;
    std::vector<double> h(E, 1.0);
    upload(ctx, ones, h.data(), E);
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    switch (m->kind) {
    case SFC_ELEM_LINE2_POISSON:
        k_elem_poisson<1, 2><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, ones.p, m->quad, E,
                                                                         ke0, err.p);
        break;
    case SFC_ELEM_TRI3_POISSON:
        k_elem_poisson<2, 3><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, ones.p, m->quad, E,
                                                                         ke0, err.p);
        break;
    case SFC_ELEM_HEX8_POISSON:
        k_elem_poisson<3, 8><<<grid_for(E, 128), 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, ones.p, m->quad, E,
                                                                         ke0, err.p);
        break;
    default:
        fail(SFC_ERR_BAD_ARG, "stiffness derivatives are defined for the Poisson element kinds");
    }
    count_launch(ctx);
    int h_err = 0;
    download(ctx, &h_err, err.p, 1);
    if (h_err) fail(SFC_ERR_NEG_JACOBIAN, "Negative Jacobian in an element");
}

// CSR values of sum_e w_e K_e for kc weight vectors at once:
// out[k * nnz + s] = sum over the slot's element entries of w[k * E + e] ke[entry]
__global__ void k_gather_weighted(const int32_t *__restrict__ slot_ptr, const int32_t *__restrict__ contrib,
                                  const double *__restrict__ ke, int LL, const double *__restrict__ w, int64_t E,
                                  int kc, int64_t nnz, double *__restrict__ out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz * kc; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / nnz, sl = t - k * nnz;
        double v = 0.0;
        for (int32_t q = slot_ptr[sl]; q < slot_ptr[sl + 1]; ++q) {
            const int32_t id = contrib[q];
            v += w[k * E + id / LL] * ke[id];
        }
        out[t] = v;
    }
}

void gather_weighted(const sfc_mesh *m, const double *ke0, const double *w_dev, int kc, double *out)
{
    sfc_ctx *ctx = m->ctx;
    k_gather_weighted<<<grid_for(m->nnz * kc, 256), 256, 0, ctx->stream>>>(m->slot_ptr.p, m->contrib.p, ke0,
                                                                          m->L * m->L, w_dev, m->num_elems, kc,
                                                                          m->nnz, out);
    count_launch(ctx);
}

void assemble_load(sfc_ctx *ctx, const sfc_mesh *m, const double *f, double *F_dev, bool zero_first)
{
    if (zero_first) SFC_CK(cudaMemsetAsync(F_dev, 0, m->num_dofs * 8, ctx->stream));
    const double f0 = f[0], f1 = m->dof > 1 ? f[1] : 0.0, f2 = m->dof > 2 ? f[2] : 0.0;
    const unsigned g = grid_for(m->num_nodes, 128);
    switch (m->kind) {
    case SFC_ELEM_LINE2_POISSON:
        k_load<1, 2><<<g, 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->node_ptr.p, m->node_elem.p, m->quad,
                                                  m->num_nodes, m->dof, f0, f1, f2, F_dev);
        break;
    case SFC_ELEM_TRI3_POISSON:
        k_load<2, 3><<<g, 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->node_ptr.p, m->node_elem.p, m->quad,
                                                  m->num_nodes, m->dof, f0, f1, f2, F_dev);
        break;
    default:
        k_load<3, 8><<<g, 128, 0, ctx->stream>>>(m->coords.p, m->conn.p, m->node_ptr.p, m->node_elem.p, m->quad,
                                                  m->num_nodes, m->dof, f0, f1, f2, F_dev);
        break;
    }
    count_launch(ctx);
}

void apply_constraints_dev(sfc_system *s, const uint32_t *idx_dev, const double *val_dev, int64_t n, double factor,
                           double scalar)
{
    sfc_ctx *ctx = s->ctx;
    SFC_REQUIRE(s->has_pattern, "no matrix assembled before applyConstraints");
    if (!s->mask.p) {
        s->mask.alloc(s->N);
        s->bc_val.alloc(s->N);
        SFC_CK(cudaMemsetAsync(s->mask.p, 0, s->N, ctx->stream));
        SFC_CK(cudaMemsetAsync(s->bc_val.p, 0, s->N * 8, ctx->stream));
    }
    if (n == 0) return;
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    k_constraints<<<grid_for(n, 128), 128, 0, ctx->stream>>>(idx_dev, val_dev, n, s->row_ptr.p, s->col.p, s->a_ref.p,
                                                             s->F.p, s->mask.p, s->bc_val.p, factor, scalar, s->N,
                                                             err.p);
    count_launch(ctx);
    int h = 0;
    download(ctx, &h, err.p, 1);
    if (h == 2) fail(SFC_ERR_BAD_ARG, "constraint dof index out of range");
    if (h == 3) fail(SFC_ERR_BAD_ARG, "constrained row has no diagonal entry");
    s->any_constraint = true;
    s->bc_scalar = scalar;
    s->op_valid = false;
}

static void build_bsr(sfc_system *s);

void build_operator(sfc_system *s, bool require_positive_diag)
{
    if (s->op_valid) return;
    sfc_ctx *ctx = s->ctx;
    flush_staged(s);
    SFC_REQUIRE(s->has_pattern, "no matrix assembled");
    if (!s->mask.p) {
        s->mask.alloc(s->N);
        s->bc_val.alloc(s->N);
        SFC_CK(cudaMemsetAsync(s->mask.p, 0, s->N, ctx->stream));
        SFC_CK(cudaMemsetAsync(s->bc_val.p, 0, s->N * 8, ctx->stream));
    }
    s->a_op.alloc(s->nnz);
    s->a_op32.alloc(s->nnz);
    s->dinv.alloc(s->N);
    s->dinv32.alloc(s->N);
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    k_build_op<<<grid_for(s->N * 32, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->diag.p, s->a_ref.p,
                                                             s->mask.p, s->N, s->a_op.p, s->a_op32.p, s->dinv.p,
                                                             s->dinv32.p, err.p);
    count_launch(ctx);
    int h = 0;
    download(ctx, &h, err.p, 1);
    if (h == 4) fail(SFC_ERR_BAD_ARG, "a row has no diagonal entry");
    if (h == 5 && require_positive_diag) fail(SFC_ERR_NOT_SPD, "non-positive diagonal entry: the operator is not SPD");
    build_bsr(s);
    s->op_valid = true;
    ++s->op_serial;
}

// ---------------------------------------------------------------------------
// node-block (3 x 3) view of the operator for 3-dof meshes.  The three rows of
// node i have the same columns, grouped node by node (every component couples
// to every component of each neighbour, and the triplet pattern keeps explicit
// zeros), so block t of node i is read off rows 3i..3i+2 at offset 3t.
// ---------------------------------------------------------------------------
__global__ void k_bsr_ptr(const int32_t *__restrict__ row_ptr, int64_t nodes, int32_t *__restrict__ bptr, int *err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r0 = row_ptr[3 * i];
        if (r0 % 9) atomicExch(err, 1);
        bptr[i] = r0 / 9;
        if (i < nodes) {
            const int32_t len = row_ptr[3 * i + 1] - r0;
            if (row_ptr[3 * i + 2] - row_ptr[3 * i + 1] != len || row_ptr[3 * i + 3] - row_ptr[3 * i + 2] != len ||
                len % 3)
                atomicExch(err, 1);
        }
    }
}

__global__ void k_bsr_fill(const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
                           const double *__restrict__ a_op, const int32_t *__restrict__ bptr, int64_t nodes,
                           int32_t *__restrict__ bcol, float *__restrict__ b32, double *__restrict__ b64, int *err)
{
    // warp per node, lanes over the node's 9 nb block values (coalesced writes)
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nodes; i += warps) {
        const int32_t r0 = row_ptr[3 * i];
        const int32_t nb = bptr[i + 1] - bptr[i];
        for (int32_t e = lane; e < 9 * nb; e += 32) {
            const int32_t t = e / 9, r = (e % 9) / 3, c = e % 3;
            const int64_t b = bptr[i] + t;
            const int32_t j = col[r0 + 3 * t] / 3;
            if (r == 0 && c == 0) bcol[b] = j;
            const int32_t s = r0 + r * 3 * nb + 3 * t + c;
            if (col[s] != 3 * j + c) atomicExch(err, 1);
            b64[b * 9 + r * 3 + c] = a_op[s];
            b32[b * 9 + r * 3 + c] = (float)a_op[s];
        }
    }
}

// inverse of node i's diagonal 3x3 block (FP64 cofactors, stored FP32)
__global__ void k_bsr_dinv(const int32_t *__restrict__ bptr, const int32_t *__restrict__ bcol,
                           const double *__restrict__ b64, int64_t nodes, float *__restrict__ dinv, int *err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t d = -1;
        for (int32_t b = bptr[i]; b < bptr[i + 1]; ++b)
            if (bcol[b] == i) d = b;
        if (d < 0) {
            atomicExch(err, 1);
            continue;
        }
        const double *m = b64 + 9 * d;
        const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
        const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
        if (!(det > 0.0)) {
            atomicExch(err, 1);
            continue;
        }
        const double inv[9] = {c00, m[2] * m[7] - m[1] * m[8], m[1] * m[5] - m[2] * m[4],
                               c01, m[0] * m[8] - m[2] * m[6], m[2] * m[3] - m[0] * m[5],
                               c02, m[1] * m[6] - m[0] * m[7], m[0] * m[4] - m[1] * m[3]};
        for (int k = 0; k < 9; ++k) dinv[9 * i + k] = (float)(inv[k] / det);
    }
}

static void build_bsr(sfc_system *s)
{
    sfc_ctx *ctx = s->ctx;
    s->has_bsr = false;
    if (!s->pattern_mesh || s->pattern_mesh->dof != 3 || s->N % 3) return;
    const int64_t nodes = s->N / 3, nb = s->nnz / 9;
    s->nodes = nodes;
    s->nblocks = nb;
    s->bptr.alloc(nodes + 1);
    s->bcol.alloc(nb);
    s->bval32.alloc(nb * 9);
    s->bval64.alloc(nb * 9);
    DevInt err = status_word(ctx);
    SFC_CK(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
    k_bsr_ptr<<<grid_for(nodes + 1, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, nodes, s->bptr.p, err.p);
    k_bsr_fill<<<grid_for(nodes * 32, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->a_op.p, s->bptr.p, nodes,
                                                              s->bcol.p, s->bval32.p, s->bval64.p, err.p);
    count_launch(ctx, 2);
    int h = 0;
    download(ctx, &h, err.p, 1);
    s->has_bsr = (h == 0);
    if (!s->has_bsr) s->bdinv32.release();
    if (s->has_bsr) {
        s->bdinv32.alloc(nodes * 9);  // kept across rebuilds: a free + malloc here synchronises the device
        k_bsr_dinv<<<grid_for(nodes, 128), 128, 0, ctx->stream>>>(s->bptr.p, s->bcol.p, s->bval64.p, nodes,
                                                                  s->bdinv32.p, err.p);
        count_launch(ctx);
        download(ctx, &h, err.p, 1);
        if (h) s->bdinv32.release();  // block Jacobi unavailable: point Jacobi is used
    }
    if (s->has_bsr) build_lattice_blocks(s);
    else s->has_lattice = false;
}

// ---------------------------------------------------------------------------
// compat path: host-staged triplets merged on the GPU
// ---------------------------------------------------------------------------
__global__ void k_csr_to_keys(const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col, int64_t N,
                              uint64_t *__restrict__ keys, int32_t *__restrict__ ids)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        for (int32_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s) {
            keys[s] = (uint64_t)i * (uint64_t)N + (uint64_t)col[s];
            ids[s] = s;
        }
}

__global__ void k_staged_keys(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols, int64_t n,
                              int64_t off, int64_t N, uint64_t *__restrict__ keys, int32_t *__restrict__ ids)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        keys[off + t] = (uint64_t)rows[t] * (uint64_t)N + cols[t];
        ids[off + t] = (int32_t)(off + t);
    }
}

__global__ void k_add_vec(double *__restrict__ y, const double *__restrict__ x, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        y[t] = ADD(y[t], x[t]);
}

void flush_staged(sfc_system *s)
{
    sfc_ctx *ctx = s->ctx;
    if (s->st_rhs_dirty) {
        DBuf<double> tmp;
        upload(ctx, tmp, s->st_rhs.data(), s->N);
        k_add_vec<<<grid_for(s->N, 256), 256, 0, ctx->stream>>>(s->F.p, tmp.p, s->N);
        count_launch(ctx);
        SFC_CK(cudaStreamSynchronize(ctx->stream));
        std::fill(s->st_rhs.begin(), s->st_rhs.end(), 0.0);
        s->st_rhs_dirty = false;
    }
    if (s->st_vals.empty()) return;
    SFC_REQUIRE(!s->any_constraint, "insertToMatrix after applyConstraints is not supported");
    const int64_t n_new = (int64_t)s->st_vals.size();
    const int64_t n_old = s->has_pattern ? s->nnz : 0;
    const int64_t M = n_old + n_new;
    SFC_REQUIRE_SIZE(M < (int64_t)INT32_MAX, "more than 2^31 - 1 staged matrix entries (32-bit indices)");
    DBuf<uint64_t> keys;
    DBuf<int32_t> ids;
    keys.alloc(M);
    ids.alloc(M);
    DBuf<double> vals;  // old CSR values first, then staged ones: insertion order
    vals.alloc(M);
    if (n_old) {
        k_csr_to_keys<<<grid_for(s->N, 256), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col.p, s->N, keys.p, ids.p);
        count_launch(ctx);
        SFC_CK(cudaMemcpyAsync(vals.p, s->a_ref.p, n_old * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    {
        DBuf<uint32_t> r, c;
        upload(ctx, r, s->st_rows.data(), n_new);
        upload(ctx, c, s->st_cols.data(), n_new);
        SFC_CK(cudaMemcpyAsync(vals.p + n_old, s->st_vals.data(), n_new * 8, cudaMemcpyHostToDevice, ctx->stream));
        k_staged_keys<<<grid_for(n_new, 256), 256, 0, ctx->stream>>>(r.p, c.p, n_new, n_old, s->N, keys.p, ids.p);
        count_launch(ctx);
        SFC_CK(cudaStreamSynchronize(ctx->stream));
    }
    DBuf<int32_t> slot_ptr, sorted;
    s->nnz = sort_and_merge(ctx, keys, ids, M, s->N, s->row_ptr, s->col, s->diag, slot_ptr, sorted);
    s->a_ref.alloc(s->nnz);
    k_gather<<<grid_for(s->nnz, 256), 256, 0, ctx->stream>>>(slot_ptr.p, sorted.p, vals.p, s->nnz, s->a_ref.p);
    count_launch(ctx);
    SFC_CK(cudaStreamSynchronize(ctx->stream));
    s->st_rows.clear();
    s->st_cols.clear();
    s->st_vals.clear();
    s->has_pattern = true;
    s->pattern_mesh = nullptr;
    s->op_valid = false;
}

}  // namespace sfc
