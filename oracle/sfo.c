/*
 * sfo.c -- CPU oracle for the statFEM forward-and-conditioning path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the arithmetic
 * of the reference's element, quadrature and assembly code so that the CUDA
 * product can be checked against it.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load it; the product never does.
 *
 * Every floating-point expression below keeps the operation order of the
 * reference line it cites (compiled with -ffp-contract=off so that no FMA is
 * formed).  Where the reference delegates an inner product to Eigen's
 * fixed-size evaluator, this file uses Eigen's unrolled pairwise reduction
 * order (sum(a[0..n)) = sum(first n/2) + sum(rest)); the reference itself
 * could not be compiled here, so that convention is unpinned and is
 * documented as such.
 *
 * Reference files cited (paths inside fcirak/statFEM):
 *   corlib/GaussLegendre.hpp, corlib/SimplexQuadrature.hpp,
 *   corlib/TensorQuadrature.hpp, corlib/Shapefun.ipp, corlib/linalg.hpp,
 *   corlib/ElementBasic.ipp, del2/fem/ElementPotential.ipp,
 *   solid/fem/ElementStatic.ipp, solid/material/svenant/SVenant.ipp,
 *   corlib/ComputeElementMatrix.hpp, corlib/MatrixAssembler.hpp,
 *   corlib/Triplet.hpp, corlib/Integrator.hpp, corlib/BodyForce.hpp,
 *   corlib/VectorAssembler.hpp, statX/infer/ExpKernel.hpp,
 *   statX/infer/CovarianceForcing.ipp.
 */
#include <math.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdlib.h>
#include <string.h>

/* element kinds; the numeric values match SFC_ELEM_* of the public header */
enum {
    SFO_LINE2_POISSON = 1,
    SFO_TRI3_POISSON = 2,
    SFO_HEX8_POISSON = 3,
    SFO_HEX8_ELASTIC = 4
};

#define SFO_MAXQ 125

/* ------------------------------------------------------------------------ */
/* quadrature rules                                                          */
/* ------------------------------------------------------------------------ */

/* Gauss-Legendre on (0,1), points in descending order, 15-digit literals:
 * corlib/GaussLegendre.hpp:65-100 */
static int gauss_legendre(int n, double *w, double *x)
{
    switch (n) {
    case 1: w[0] = 1; x[0] = 0.5; return 1;
    case 2:
        w[0] = 0.5; x[0] = 0.788675134594813;
        w[1] = 0.5; x[1] = 0.211324865405187;
        return 2;
    case 3:
        w[0] = 0.277777777777777; x[0] = 0.887298334620741;
        w[1] = 0.444444444444444; x[1] = 0.5;
        w[2] = 0.277777777777777; x[2] = 0.112701665379259;
        return 3;
    case 4:
        w[0] = 0.173927422568727; x[0] = 0.930568155797026;
        w[1] = 0.326072577431273; x[1] = 0.669990521792428;
        w[2] = 0.326072577431273; x[2] = 0.330009478207572;
        w[3] = 0.173927422568727; x[3] = 0.069431844202974;
        return 4;
    case 5:
        w[0] = 0.118463442528095; x[0] = 0.953089922969332;
        w[1] = 0.239314335249683; x[1] = 0.769234655052841;
        w[2] = 0.284444444444444; x[2] = 0.5;
        w[3] = 0.239314335249683; x[3] = 0.230765344947159;
        w[4] = 0.118463442528095; x[4] = 0.046910077030668;
        return 5;
    }
    return 0;
}

static int int_cbrt(int q)
{
    for (int n = 1; n <= 5; ++n)
        if (n * n * n == q) return n;
    return 0;
}

/* Fill weights w[q] and points pts[q*3+a]; returns the number of points or 0.
 * LINE:  Quadrature<LINE,QPS> -> SimplexQuadratureConstructor<1,QPS> -> GL<QPS>
 *        (corlib/SimplexQuadrature.hpp:97-106).
 * TRI:   SimplexQuadratureConstructor<2,1> and <2,3>
 *        (corlib/SimplexQuadrature.hpp:160-191; truncated 15-digit literals).
 * HEX:   TensorQuadratureConstructor<GL<n>,3>: index = outer*n*n + lower,
 *        weight = (w_i*w_j)*w_k, point = (x_i,x_j,x_k), first coordinate fastest
 *        (corlib/TensorQuadrature.hpp:101-139). */
int sfo_quadrature(int kind, int qps, double *w, double *pts)
{
    double gw[5], gx[5];
    memset(pts, 0, sizeof(double) * 3 * (qps > 0 ? qps : 1));
    if (kind == SFO_LINE2_POISSON) {
        int n = gauss_legendre(qps, gw, gx);
        for (int i = 0; i < n; ++i) { w[i] = gw[i]; pts[3 * i] = gx[i]; }
        return n;
    }
    if (kind == SFO_TRI3_POISSON) {
        if (qps == 1) {
            w[0] = 0.5; pts[0] = 0.333333333333333; pts[1] = 0.333333333333333;
            return 1;
        }
        if (qps == 3) {
            w[0] = 0.166666666666666; pts[0] = 0.666666666666667; pts[1] = 0.166666666666667;
            w[1] = 0.166666666666666; pts[3] = 0.166666666666667; pts[4] = 0.666666666666667;
            w[2] = 0.166666666666666; pts[6] = 0.166666666666667; pts[7] = 0.166666666666667;
            return 3;
        }
        return 0;
    }
    if (kind == SFO_HEX8_POISSON || kind == SFO_HEX8_ELASTIC) {
        int n = int_cbrt(qps);
        if (!n || !gauss_legendre(n, gw, gx)) return 0;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    int q = k * n * n + j * n + i;
                    w[q] = (gw[i] * gw[j]) * gw[k];
                    pts[3 * q + 0] = gx[i];
                    pts[3 * q + 1] = gx[j];
                    pts[3 * q + 2] = gx[k];
                }
        return n * n * n;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* element traits                                                            */
/* ------------------------------------------------------------------------ */

int sfo_dim(int kind) { return kind == SFO_LINE2_POISSON ? 1 : kind == SFO_TRI3_POISSON ? 2 : 3; }
int sfo_nodes_per_elem(int kind) { return kind == SFO_LINE2_POISSON ? 2 : kind == SFO_TRI3_POISSON ? 3 : 8; }
int sfo_dofs_per_node(int kind) { return kind == SFO_HEX8_ELASTIC ? 3 : 1; }

/* Eigen's fixed-size unrolled reduction: split in halves, recurse. */
static double redux(const double *t, int n)
{
    switch (n) {
    case 1: return t[0];
    case 2: return t[0] + t[1];
    case 3: return t[0] + (t[1] + t[2]);
    case 8: return ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
    }
    return NAN; /* no other length occurs for the supported elements */
}

/* shape functions phi[K] at xi: corlib/Shapefun.ipp (LINE,2) :36-41,
 * (TRIANGLE,3) :180-187, (HEXAHEDRON,8) :926-937 */
static void shape(int kind, const double *xi, double *phi)
{
    if (kind == SFO_LINE2_POISSON) {
        phi[0] = 1. - xi[0];
        phi[1] = xi[0];
    } else if (kind == SFO_TRI3_POISSON) {
        phi[0] = 1. - (xi[0] + xi[1]);
        phi[1] = xi[0];
        phi[2] = xi[1];
    } else {
        phi[0] = (1. - xi[0]) * (1. - xi[1]) * (1. - xi[2]);
        phi[1] = xi[0] * (1. - xi[1]) * (1. - xi[2]);
        phi[2] = xi[0] * xi[1] * (1. - xi[2]);
        phi[3] = (1. - xi[0]) * xi[1] * (1. - xi[2]);
        phi[4] = (1. - xi[0]) * (1. - xi[1]) * xi[2];
        phi[5] = xi[0] * (1. - xi[1]) * xi[2];
        phi[6] = xi[0] * xi[1] * xi[2];
        phi[7] = (1. - xi[0]) * xi[1] * xi[2];
    }
}

/* gradients dphi[a*8+K] = d phi^K / d xi_a: corlib/Shapefun.ipp (LINE,2) :44-49,
 * (TRIANGLE,3) :190-196, (HEXAHEDRON,8) :940-975 */
static void shape_grad(int kind, const double *xi, double *d)
{
    if (kind == SFO_LINE2_POISSON) {
        d[0] = -1.; d[1] = 1.;
    } else if (kind == SFO_TRI3_POISSON) {
        d[0] = -1.; d[1] = 1.; d[2] = 0.;
        d[8] = -1.; d[9] = 0.; d[10] = 1.;
    } else {
        d[0] = -(1. - xi[1]) * (1. - xi[2]);
        d[1] = (1. - xi[1]) * (1. - xi[2]);
        d[2] = xi[1] * (1. - xi[2]);
        d[3] = -xi[1] * (1. - xi[2]);
        d[4] = -(1. - xi[1]) * xi[2];
        d[5] = (1. - xi[1]) * xi[2];
        d[6] = xi[1] * xi[2];
        d[7] = -xi[1] * xi[2];
        d[8 + 0] = -(1. - xi[0]) * (1. - xi[2]);
        d[8 + 1] = -xi[0] * (1. - xi[2]);
        d[8 + 2] = xi[0] * (1. - xi[2]);
        d[8 + 3] = (1. - xi[0]) * (1. - xi[2]);
        d[8 + 4] = -(1. - xi[0]) * xi[2];
        d[8 + 5] = -xi[0] * xi[2];
        d[8 + 6] = xi[0] * xi[2];
        d[8 + 7] = (1. - xi[0]) * xi[2];
        d[16 + 0] = -(1. - xi[0]) * (1. - xi[1]);
        d[16 + 1] = -xi[0] * (1. - xi[1]);
        d[16 + 2] = -xi[0] * xi[1];
        d[16 + 3] = -(1. - xi[0]) * xi[1];
        d[16 + 4] = (1. - xi[0]) * (1. - xi[1]);
        d[16 + 5] = xi[0] * (1. - xi[1]);
        d[16 + 6] = xi[0] * xi[1];
        d[16 + 7] = (1. - xi[0]) * xi[1];
    }
}

/* determinant: corlib/linalg.hpp:47-74 (m is row-major dim x dim) */
static double determinant(int dim, const double *m)
{
    if (dim == 1) return m[0];
    if (dim == 2) return m[0] * m[3] - m[1] * m[2];
    return m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7]
         - m[0] * m[5] * m[7] - m[1] * m[3] * m[8] - m[2] * m[4] * m[6];
}

/* in-place inverse returning the determinant: corlib/linalg.hpp:100-152 */
static double inverse(int dim, double *m)
{
    double det = determinant(dim, m);
    if (dim == 1) {
        m[0] = 1. / det;
    } else if (dim == 2) {
        double aux = m[0];
        m[0] = m[3] / det;
        m[1] /= -det;
        m[2] /= -det;
        m[3] = aux / det;
    } else {
        double t[9];
        memcpy(t, m, sizeof t);
        m[0] = (t[4] * t[8] - t[5] * t[7]) / det;
        m[4] = (t[0] * t[8] - t[2] * t[6]) / det;
        m[8] = (t[0] * t[4] - t[1] * t[3]) / det;
        m[1] = (t[2] * t[7] - t[1] * t[8]) / det;
        m[2] = (t[1] * t[5] - t[2] * t[4]) / det;
        m[3] = (t[5] * t[6] - t[3] * t[8]) / det;
        m[5] = (t[2] * t[3] - t[0] * t[5]) / det;
        m[6] = (t[3] * t[7] - t[4] * t[6]) / det;
        m[7] = (t[1] * t[6] - t[0] * t[7]) / det;
    }
    return det;
}

/* covariant basis G[i][a] = sum_K X[K][i] dphi[a][K] (X * dphiDxi^T) */
static void covariant(int dim, int nn, const double *X, const double *dphi, double *G)
{
    double t[8];
    for (int i = 0; i < dim; ++i)
        for (int a = 0; a < dim; ++a) {
            for (int K = 0; K < nn; ++K) t[K] = X[K * 3 + i] * dphi[a * 8 + K];
            G[i * dim + a] = redux(t, nn);
        }
}

/* ElementBasic::globalDerivatives, corlib/ElementBasic.ipp:178-204 with
 * ContraVariantBasis<DIM,DIM>::compute, corlib/linalg.hpp:200-217:
 * contra = inverse(G^T); dphiDx = contra * dphiDxi.  Returns detJ (the
 * determinant of G^T).  dx[i*8+K] = d phi^K / d x_i. */
static double global_derivatives(int kind, const double *X, const double *xi, double *dx)
{
    int dim = sfo_dim(kind), nn = sfo_nodes_per_elem(kind);
    double dphi[24], G[9], C[9], t[3];
    shape_grad(kind, xi, dphi);
    covariant(dim, nn, X, dphi, G);
    for (int i = 0; i < dim; ++i)
        for (int a = 0; a < dim; ++a) C[i * dim + a] = G[a * dim + i];
    double det = inverse(dim, C);
    for (int i = 0; i < dim; ++i)
        for (int K = 0; K < nn; ++K) {
            for (int a = 0; a < dim; ++a) t[a] = C[i * dim + a] * dphi[a * 8 + K];
            dx[i * 8 + K] = redux(t, dim);
        }
    return det;
}

/* ElementBasic::jacobian, corlib/ElementBasic.ipp:132-153: metric(G) =
 * determinant(G) for square G (corlib/linalg.hpp:404-417). */
static double jacobian(int kind, const double *X, const double *xi)
{
    int dim = sfo_dim(kind), nn = sfo_nodes_per_elem(kind);
    double dphi[24], G[9];
    shape_grad(kind, xi, dphi);
    covariant(dim, nn, X, dphi, G);
    return determinant(dim, G);
}

/* Lame constants: solid/material/svenant/SVenant.ipp:32-37 */
static void lame(double E, double nu, double *lambda, double *mu)
{
    *lambda = E * nu / (1.0 + nu) / (1.0 - 2.0 * nu);
    *mu = E / 2.0 / (1.0 + nu);
}

/* SVenant::elasticityTensor at F = I (zero displacement), SVenant.ipp:107-140.
 * With F = I: E = 0, S = 0, FFt = I. */
static double ctensor(double lambda, double mu, int i, int J, int k, int L)
{
    double F_iJ = (i == J), F_kL = (k == L), F_iL = (i == L), F_kJ = (k == J);
    double c = lambda * F_iJ * F_kL;
    c += mu * F_iL * F_kJ;
    if (J == L) c += mu * (double)(i == k);
    if (i == k) c += 0.0;
    return c;
}

/*
 * Element matrix Ke (L x L row-major, L = nn*dof), zero-initialised as in
 * corlib/MatrixAssembler.hpp:213-214 and accumulated over the quadrature in
 * rule order (corlib/ComputeElementMatrix.hpp:62-77); the assembler's factor
 * is 1.0 (MatrixAssembler.hpp:220).
 *   Poisson:    Ke += ((kappa*detJ)*w) * (dphiDx^T dphiDx)
 *               del2/fem/ElementPotential.ipp:58-74
 *   elasticity: Ke[m*3+i][n*3+k] += (kentry*detJ)*w,
 *               kentry = sum_J sum_L (C_iJkL*dX_Jm)*dX_Ln
 *               solid/fem/ElementStatic.ipp:286-320
 * X is the element's nodal coordinates (nn x 3, SMF layout).
 */
int sfo_element_matrix(int kind, int qps, const double *X, double coeff, double nu, double *Ke)
{
    double w[SFO_MAXQ], pts[3 * SFO_MAXQ], dx[24], t[3];
    int nq = sfo_quadrature(kind, qps, w, pts);
    if (!nq) return -1;
    int dim = sfo_dim(kind), nn = sfo_nodes_per_elem(kind), d = sfo_dofs_per_node(kind);
    int L = nn * d;
    memset(Ke, 0, sizeof(double) * L * L);
    for (int q = 0; q < nq; ++q) {
        double det = global_derivatives(kind, X, pts + 3 * q, dx);
        if (!(det > 0.)) return -2;
        if (kind != SFO_HEX8_ELASTIC) {
            double s = coeff * det * w[q];
            for (int m = 0; m < nn; ++m)
                for (int n = 0; n < nn; ++n) {
                    for (int a = 0; a < dim; ++a) t[a] = dx[a * 8 + m] * dx[a * 8 + n];
                    Ke[m * L + n] += s * redux(t, dim);
                }
        } else {
            double lambda, mu;
            lame(coeff, nu, &lambda, &mu);
            for (int m = 0; m < nn; ++m)
                for (int i = 0; i < 3; ++i)
                    for (int n = 0; n < nn; ++n)
                        for (int k = 0; k < 3; ++k) {
                            double kentry = 0;
                            for (int J = 0; J < 3; ++J)
                                for (int Lx = 0; Lx < 3; ++Lx)
                                    kentry += ctensor(lambda, mu, i, J, k, Lx) * dx[J * 8 + m] * dx[Lx * 8 + n];
                            Ke[(m * 3 + i) * L + n * 3 + k] += kentry * det * w[q];
                        }
        }
    }
    return nq;
}

/*
 * Body-force contributions of one element at one quadrature point:
 * out[n*dof + c] = ((w*detJ)*factor) * (f_c * phi_n)  for a constant force f.
 *   Poisson:    del2/fem/ElementPotential.ipp:149-176
 *   elasticity: solid/fem/ElementStatic.ipp:441-466 ((detG*w)*factor: equal
 *               bit for bit because IEEE multiplication commutes)
 * detJ here is ElementBasic::jacobian (determinant of G, not of G^T).
 */
static void element_load_q(int kind, const double *X, const double *xi, double wq,
                           const double *f, double factor, double *out)
{
    int nn = sfo_nodes_per_elem(kind), d = sfo_dofs_per_node(kind);
    double phi[8];
    shape(kind, xi, phi);
    double det = jacobian(kind, X, xi);
    double s = wq * det * factor;
    for (int n = 0; n < nn; ++n)
        for (int c = 0; c < d; ++c) out[n * d + c] = s * (f[c] * phi[n]);
}

static void gather_X(const double *coords, const uint32_t *conn, int nn, int64_t e, double *X)
{
    for (int K = 0; K < nn; ++K) {
        const double *p = coords + 3 * (int64_t)conn[e * nn + K];
        X[K * 3 + 0] = p[0];
        X[K * 3 + 1] = p[1];
        X[K * 3 + 2] = p[2];
    }
}

/*
 * Nodal load vector F[node*dof + c] for a constant force f (dof components):
 * nodes' force arrays cleared, Integrator over elements in mesh order and
 * quadrature points in rule order (corlib/Integrator.hpp:61-73), each point
 * adding F.col(n) to node n (Node::addToForce), then VectorAssembler copying
 * node forces into a zeroed global vector (corlib/VectorAssembler.hpp:101-114,
 * factor 1).  With f = 1 this is the shape-function integral phibar used by
 * CovarianceForcing (del2/apps/reference/laplaceRHSinfer/inference.hpp:108-119).
 */
int sfo_assemble_load(int kind, int qps, const double *coords, int64_t num_nodes,
                      const uint32_t *conn, int64_t num_elems, const double *f,
                      double *F)
{
    double w[SFO_MAXQ], pts[3 * SFO_MAXQ], X[24], out[24];
    int nq = sfo_quadrature(kind, qps, w, pts);
    if (!nq) return -1;
    int nn = sfo_nodes_per_elem(kind), d = sfo_dofs_per_node(kind);
    memset(F, 0, sizeof(double) * num_nodes * d);
    for (int64_t e = 0; e < num_elems; ++e) {
        gather_X(coords, conn, nn, e, X);
        for (int q = 0; q < nq; ++q) {
            element_load_q(kind, X, pts + 3 * q, w[q], f, 1.0, out);
            for (int n = 0; n < nn; ++n)
                for (int c = 0; c < d; ++c)
                    F[(int64_t)conn[e * nn + n] * d + c] += out[n * d + c];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* triplet assembly -> CSR                                                   */
/* ------------------------------------------------------------------------ */

typedef struct { uint64_t key; int64_t seq; double val; } trip_t;

static int trip_cmp(const void *a, const void *b)
{
    const trip_t *x = a, *y = b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->seq < y->seq ? -1 : x->seq > y->seq;
}

/*
 * Global matrix in the reference's triplet semantics: every element entry is
 * inserted (corlib/SystemSolveEigenSparse.hpp insertToMatrix, row-major over
 * the element's (row,col) dof pairs), triplets are sorted by (row,col) and
 * merged by summation starting from 0.0 (corlib/Triplet.hpp:126-170,565-580).
 * std::sort is unstable, so the reference leaves the order of equal keys
 * unspecified; this oracle fixes it to insertion order (element order), the
 * documented "sorted-segment" convention the GPU assembler also follows.
 * Explicit zeros stay in the pattern.
 *
 * Two-call protocol: with row_ptr == NULL the function returns nnz only.
 * row_ptr has num_dofs+1 entries.  Returns nnz, or a negative error.
 */
int64_t sfo_assemble_csr(int kind, int qps, const double *coords, int64_t num_nodes,
                         const uint32_t *conn, int64_t num_elems, const double *coeff,
                         double nu, int64_t *row_ptr, int32_t *col, double *val)
{
    int nn = sfo_nodes_per_elem(kind), d = sfo_dofs_per_node(kind);
    int L = nn * d;
    int64_t N = num_nodes * d;
    int64_t M = num_elems * L * L;
    trip_t *tr = malloc(sizeof(trip_t) * (M > 0 ? M : 1));
    if (!tr) return -3;
    double X[24], Ke[576];
    uint32_t dofs[24];
    for (int64_t e = 0; e < num_elems; ++e) {
        gather_X(coords, conn, nn, e, X);
        int rc = sfo_element_matrix(kind, qps, X, coeff ? coeff[e] : 1.0, nu, Ke);
        if (rc < 0) { free(tr); return rc; }
        for (int K = 0; K < nn; ++K)
            for (int c = 0; c < d; ++c) dofs[K * d + c] = conn[e * nn + K] * d + c;
        for (int r = 0; r < L; ++r)
            for (int c = 0; c < L; ++c) {
                int64_t s = e * L * L + r * L + c;
                tr[s].key = (uint64_t)dofs[r] * (uint64_t)N + dofs[c];
                tr[s].seq = s;
                tr[s].val = Ke[r * L + c];
            }
    }
    qsort(tr, M, sizeof(trip_t), trip_cmp);
    int64_t nnz = 0;
    for (int64_t s = 0; s < M; ++s)
        if (s == 0 || tr[s].key != tr[s - 1].key) ++nnz;
    if (row_ptr) {
        int64_t k = -1;
        for (int64_t i = 0; i <= N; ++i) row_ptr[i] = 0;
        for (int64_t s = 0; s < M; ++s) {
            if (s == 0 || tr[s].key != tr[s - 1].key) {
                ++k;
                int64_t row = tr[s].key / N;
                col[k] = (int32_t)(tr[s].key % N);
                val[k] = 0.0;
                row_ptr[row + 1]++;
            }
            val[k] += tr[s].val;
        }
        for (int64_t i = 0; i < N; ++i) row_ptr[i + 1] += row_ptr[i];
    }
    free(tr);
    return nnz;
}

/*
 * Dirichlet constraints in the reference's row-zeroing form:
 * Triplet::zeroRow (corlib/Triplet.hpp:219-260) zeroes every entry of row c
 * and puts `scalar` on the diagonal; SystemSolveEigenSparse::applyConstraints
 * (corlib/SystemSolveEigenSparse.hpp:197-215) sets F[c] = (factor*value)*scalar.
 * A missing diagonal is an error here (it cannot occur for FE patterns).
 */
int sfo_apply_constraints(int64_t num_dofs, const int64_t *row_ptr, const int32_t *col,
                          double *val, double *F, const uint32_t *idx, const double *value,
                          int64_t n, double factor, double scalar)
{
    for (int64_t t = 0; t < n; ++t) {
        int64_t c = idx[t];
        if (c >= num_dofs) return -1;
        int found = 0;
        for (int64_t s = row_ptr[c]; s < row_ptr[c + 1]; ++s) {
            if (col[s] == c) { val[s] = scalar; found = 1; }
            else val[s] = 0.0;
        }
        if (!found) return -2;
        if (F) F[c] = (factor * value[t]) * scalar;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* squared-exponential kernel and the nodal forcing covariance              */
/* ------------------------------------------------------------------------ */

/* ExpKernel::giveValue, statX/infer/ExpKernel.hpp:74-92:
 * sigma^2 * exp(-|x-y|^2 / (2 l^2)), squaredNorm reduced pairwise. */
double sfo_se_kernel(int dim, const double *x, const double *y, double sigma, double length)
{
    double t[3];
    for (int a = 0; a < dim; ++a) { double dd = x[a] - y[a]; t[a] = dd * dd; }
    return sigma * sigma * exp(-redux(t, dim) / (2. * length * length));
}

/*
 * Dense C_f (N x N, row-major, N = num_nodes*dof) as built by
 * CovarianceForcing::giveProjectedCovar (statX/infer/CovarianceForcing.ipp:38-109):
 * (C_f)[dof*i+k][dof*j+k] = (phibar_i * k(x_i,x_j)) * phibar_j for each
 * component k, zero between different components.  cutEps = 0 keeps every
 * value >= 0 (a negative value, impossible for phibar >= 0, would be dropped).
 * coords are per node (num_nodes x 3); only the first dim are used.
 */
int sfo_forcing_covariance_dense(int dim, int dof, int64_t num_nodes, const double *coords,
                                 const double *phibar, double sigma, double length, double *Cf)
{
    int64_t N = num_nodes * dof;
    memset(Cf, 0, sizeof(double) * N * N);
    for (int64_t i = 0; i < num_nodes; ++i)
        for (int64_t j = i; j < num_nodes; ++j) {
            double kv = sfo_se_kernel(dim, coords + 3 * i, coords + 3 * j, sigma, length);
            for (int k = 0; k < dof; ++k) {
                int64_t r = dof * i + k, c = dof * j + k;
                double v = phibar[r] * kv * phibar[c];
                if (v < 0.0) continue;
                Cf[r * N + c] = v;
                Cf[c * N + r] = v;
            }
        }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* plain FP64 Jacobi-PCG on a CSR matrix (CPU baseline for large meshes)    */
/* ------------------------------------------------------------------------ */

/*
 * Solves S x = b with S the symmetric elimination of the row-zeroed matrix
 * (free rows keep only free columns; constrained rows keep their diagonal).
 * mask[i] != 0 marks constrained dofs.  Stops at ||r|| <= tol*||b||.
 * Returns the iteration count, or -1 when max_iter is reached.
 */
int sfo_pcg(int64_t N, const int64_t *row_ptr, const int32_t *col, const double *val,
            const unsigned char *mask, const double *b, double *x, double tol, int max_iter,
            double *work /* 4N */)
{
    double *r = work, *z = work + N, *p = work + 2 * N, *q = work + 3 * N;
    double bb = 0, rz = 0;
    for (int64_t i = 0; i < N; ++i) {
        x[i] = 0;
        r[i] = b[i];
        bb += b[i] * b[i];
    }
    if (bb == 0) return 0;
    double *dinv = malloc(sizeof(double) * N);
    for (int64_t i = 0; i < N; ++i) {
        double dg = 1.0;
        for (int64_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s)
            if (col[s] == i) dg = val[s];
        dinv[i] = 1.0 / dg;
        z[i] = dinv[i] * r[i];
        p[i] = z[i];
        rz += r[i] * z[i];
    }
    int it;
    for (it = 1; it <= max_iter; ++it) {
        double pq = 0, rr = 0, rz2 = 0;
#pragma omp parallel for reduction(+ : pq) schedule(static) if (N >= 20000)
        for (int64_t i = 0; i < N; ++i) {
            double acc = 0;
            if (mask[i]) {
                acc = p[i] / dinv[i];
            } else {
                for (int64_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s)
                    if (!mask[col[s]]) acc += val[s] * p[col[s]];
            }
            q[i] = acc;
            pq += p[i] * acc;
        }
        double alpha = rz / pq;
#pragma omp parallel for reduction(+ : rr, rz2) schedule(static) if (N >= 20000)
        for (int64_t i = 0; i < N; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = dinv[i] * r[i];
            rr += r[i] * r[i];
            rz2 += r[i] * z[i];
        }
        if (rr <= tol * tol * bb) break;
        double beta = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule(static) if (N >= 20000)
        for (int64_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
    }
    free(dinv);
    return it > max_iter ? -1 : it;
}

/*
 * Block FP64 Jacobi-PCG: k independent right-hand sides solved together so
 * that one pass over the matrix serves all of them (each column keeps its own
 * alpha, beta and stopping test; no block-Krylov coupling).  Same operator as
 * sfo_pcg.  B and X are interleaved [N][k].  When use_x0 != 0 the iteration
 * starts from the X passed in (r = b - S x), else from zero.  Column c stops
 * once ||r_c|| <= tol*||b_c||; its_out[c] receives its iteration count (or -1
 * when max_iter is reached).  Returns the largest count, or -1.
 * Parallel over rows (OpenMP); the result does not depend on the thread count
 * except through the order of the dot-product reductions.
 */
static int max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int thread_id(void)
{
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

int sfo_block_pcg(int64_t N, const int64_t *row_ptr, const int32_t *col, const double *val,
                  const unsigned char *mask, int k, const double *B, double *X, double tol,
                  int max_iter, int use_x0, int *its_out)
{
    const int64_t NK = N * (int64_t)k;
    double *r = malloc(sizeof(double) * NK), *p = malloc(sizeof(double) * NK);
    double *q = malloc(sizeof(double) * NK), *dinv = malloc(sizeof(double) * N);
    double *bb = calloc(k, sizeof(double)), *rz = calloc(k, sizeof(double));
    double *pq = calloc(k, sizeof(double)), *rr = calloc(k, sizeof(double));
    double *rz2 = calloc(k, sizeof(double)), *alpha = calloc(k, sizeof(double));
    double *beta = calloc(k, sizeof(double));
    char *active = calloc(k, 1);
    /* Small systems run serially.  Each thread's row scratch and partial sums
     * are its own allocations (a pointer into a shared array would keep the
     * compiler from proving that the scratch row aliases no operand, and the
     * column loops would not vectorise); the partial sums are merged in
     * thread order after the loop, so the reductions do not depend on which
     * thread finishes first. */
    const int par = N * (int64_t)k >= (1 << 20);
    const int nthr = max_threads();
    double **part = calloc(2 * (size_t)nthr, sizeof(double *));
    if (!r || !p || !q || !dinv || !bb || !rz || !pq || !rr || !rz2 || !alpha || !beta || !active || !part)
        return -2;
    int fail = 0;
#pragma omp parallel for schedule(static) if (par)
    for (int64_t i = 0; i < N; ++i) {
        double dg = 1.0;
        for (int64_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s)
            if (col[s] == i) dg = val[s];
        dinv[i] = 1.0 / dg;
    }
    /* r = b - S x (x = 0 unless use_x0) */
#pragma omp parallel for schedule(static) if (par)
    for (int64_t i = 0; i < N; ++i) {
        double *ri = r + i * k;
        for (int c = 0; c < k; ++c) ri[c] = B[i * k + c];
        if (!use_x0) {
            for (int c = 0; c < k; ++c) X[i * k + c] = 0.0;
        } else if (mask[i]) {
            for (int c = 0; c < k; ++c) ri[c] -= X[i * k + c] / dinv[i];
        } else {
            for (int64_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s) {
                if (mask[col[s]]) continue;
                const double v = val[s];
                const double *xj = X + (int64_t)col[s] * k;
                for (int c = 0; c < k; ++c) ri[c] -= v * xj[c];
            }
        }
    }
    for (int64_t i = 0; i < N; ++i)
        for (int c = 0; c < k; ++c) {
            const double b = B[i * k + c], rv = r[i * k + c];
            bb[c] += b * b;
            p[i * k + c] = dinv[i] * rv;
            rz[c] += rv * (dinv[i] * rv);
            rr[c] += rv * rv;
        }
    int nact = 0;
    for (int c = 0; c < k; ++c) {
        its_out[c] = 0;
        active[c] = bb[c] > 0 && rr[c] > tol * tol * bb[c];
        nact += active[c];
    }
    int it = 0;
    while (nact > 0 && it < max_iter) {
        ++it;
        for (int c = 0; c < k; ++c) pq[c] = 0;
#pragma omp parallel if (par)
        {
            double *acc = malloc(sizeof(double) * k), *lpq = calloc(k, sizeof(double));
            part[thread_id()] = lpq;
            if (!acc || !lpq) {
#pragma omp atomic write
                fail = 1;
            }
#pragma omp for schedule(static)
            for (int64_t i = 0; i < N; ++i) {
                if (!acc || !lpq) continue;
                const double *pi = p + i * k;
                if (mask[i]) {
                    for (int c = 0; c < k; ++c) acc[c] = pi[c] / dinv[i];
                } else {
                    for (int c = 0; c < k; ++c) acc[c] = 0.0;
                    for (int64_t s = row_ptr[i]; s < row_ptr[i + 1]; ++s) {
                        if (mask[col[s]]) continue;
                        const double v = val[s];
                        const double *pj = p + (int64_t)col[s] * k;
                        for (int c = 0; c < k; ++c) acc[c] += v * pj[c];
                    }
                }
                double *qi = q + i * k;
                for (int c = 0; c < k; ++c) {
                    qi[c] = acc[c];
                    lpq[c] += pi[c] * acc[c];
                }
            }
            free(acc);
        }
        for (int t = 0; t < nthr; ++t) {
            if (part[t])
                for (int c = 0; c < k; ++c) pq[c] += part[t][c];
            free(part[t]);
            part[t] = NULL;
        }
        if (fail) break;
        for (int c = 0; c < k; ++c) {
            alpha[c] = active[c] ? rz[c] / pq[c] : 0.0;
            rr[c] = rz2[c] = 0;
        }
#pragma omp parallel if (par)
        {
            double *lrr = calloc(k, sizeof(double)), *lrz = calloc(k, sizeof(double));
            part[2 * thread_id()] = lrr;
            part[2 * thread_id() + 1] = lrz;
            if (!lrr || !lrz) {
#pragma omp atomic write
                fail = 1;
            }
#pragma omp for schedule(static)
            for (int64_t i = 0; i < N; ++i) {
                if (!lrr || !lrz) continue;
                double *xi = X + i * k, *ri = r + i * k;
                const double *pi = p + i * k, *qi = q + i * k;
                for (int c = 0; c < k; ++c) {
                    xi[c] += alpha[c] * pi[c];
                    ri[c] -= alpha[c] * qi[c];
                    lrr[c] += ri[c] * ri[c];
                    lrz[c] += ri[c] * (dinv[i] * ri[c]);
                }
            }
        }
        for (int t = 0; t < nthr; ++t) {
            if (part[2 * t] && part[2 * t + 1])
                for (int c = 0; c < k; ++c) {
                    rr[c] += part[2 * t][c];
                    rz2[c] += part[2 * t + 1][c];
                }
            free(part[2 * t]);
            free(part[2 * t + 1]);
            part[2 * t] = part[2 * t + 1] = NULL;
        }
        if (fail) break;
        for (int c = 0; c < k; ++c) {
            beta[c] = 0.0;
            if (!active[c]) continue;
            if (rr[c] <= tol * tol * bb[c]) {
                active[c] = 0;
                its_out[c] = it;
                --nact;
                continue;
            }
            beta[c] = rz2[c] / rz[c];
            rz[c] = rz2[c];
        }
#pragma omp parallel for schedule(static) if (par)
        for (int64_t i = 0; i < N; ++i) {
            double *pi = p + i * k;
            const double *ri = r + i * k;
            for (int c = 0; c < k; ++c)
                if (active[c]) pi[c] = dinv[i] * ri[c] + beta[c] * pi[c];
        }
    }
    int worst = 0;
    for (int c = 0; c < k; ++c) {
        if (active[c]) its_out[c] = -1;
        if (its_out[c] < 0) worst = -1;
        else if (worst >= 0 && its_out[c] > worst) worst = its_out[c];
    }
    free(r); free(p); free(q); free(dinv); free(bb); free(rz); free(pq); free(rr); free(rz2);
    free(alpha); free(beta); free(active);
    free(part);
    if (fail) return -2;
    return worst;
}
