// C++ integration driver: the laplaceRHSinfer flow
// (del2/apps/reference/laplaceRHSinfer/{laplaceRHSinfer.cpp,fem.hpp,inference.hpp})
// written against the drop-in classes corlib::SystemSolveCuda and
// corlib::GpuMatrixAssembler plus the statX part of the C ABI.  The mesh /
// node / element types are minimal stand-ins with the corlib method names the
// assembler uses (corlib needs Eigen and Boost, which this build does not
// have).  Reads a plain-text problem file and prints the Woodbury posterior
// mean, one value per line.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "corlib/GpuMatrixAssembler.hpp"
#include "corlib/SystemSolveCuda.hpp"

struct Vec1 {
    double v[3];
    int n;
    double operator()(int i) const { return v[i]; }
    int size() const { return n; }
};

struct Node {
    double x;
    unsigned dof;
    Vec1 giveCoordinates() const { return Vec1{{x, 0, 0}, 1}; }
};

struct Element {
    Node *nodes[2];
    double conductivity;
    void getDofIndices(std::vector<unsigned> &d) const { d = {nodes[0]->dof, nodes[1]->dof}; }
    Node *const *nodesBegin() const { return nodes; }
    Node *const *nodesEnd() const { return nodes + 2; }
    double getConductivity() const { return conductivity; }
};

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    std::ifstream in(argv[1]);
    int nn, ne, ns, no;
    double force, fsig, flen, rho, msig, mlen, eps, reg, cond;
    in >> nn >> ne >> ns >> no >> force >> fsig >> flen >> rho >> msig >> mlen >> eps >> reg >> cond;
    std::vector<Node> nodes(nn);
    for (int i = 0; i < nn; ++i) in >> nodes[i].x;
    std::vector<Element> elems(ne);
    for (int e = 0; e < ne; ++e) {
        unsigned a, b;
        in >> a >> b;
        elems[e].nodes[0] = &nodes[a];
        elems[e].nodes[1] = &nodes[b];
        elems[e].conductivity = cond;
    }
    std::vector<double> Y((size_t)ns * no), sc(ns);
    for (auto &v : Y) in >> v;
    for (auto &v : sc) in >> v;
    // Node::numberDOFs over nodes in order
    unsigned numDofs = 0;
    for (auto &n : nodes) n.dof = numDofs++;

    corlib::SystemSolveCuda sysmat(numDofs);
    sfc_solver_options_t opt{SFC_SOLVER_PCG_FP64, 20000, 1e-13, 1e-4, 0, 16, SFC_PRECOND_JACOBI};
    sysmat.setOptions(opt);

    // fem(): constraints from x == 0 or x == 1 (fem.hpp:35-40), element matrices, body force
    std::vector<std::pair<unsigned, double> > constraints;
    for (auto &n : nodes)
        if (std::fabs(n.x - 0.) < 1e-8 || std::fabs(n.x - 1.) < 1e-8) constraints.push_back({n.dof, 0.0});
    corlib::GpuMatrixAssembler<Element> maf(&sysmat, SFC_ELEM_LINE2_POISSON, 3);
    for (auto &e : elems) maf(&e);
    maf.assemble();
    maf.assembleLoad(&force);
    sysmat.finishAssembly();
    sysmat.applyConstraints(constraints, 1., 1.);
    sysmat.solveSystem();

    // inference(): CovarianceForcing, ForwardGaussRHS with P = I, KOH Woodbury
    sfc_ctx_t *ctx = sysmat.context();
    sfc_covar_forcing_t *cf = nullptr;
    corlib::sfc_detail::check(sfc_covar_forcing_create(ctx, maf.mesh(), &cf), ctx, "CovarianceForcing");
    std::vector<uint32_t> bc;
    for (auto &c : constraints) bc.push_back(c.first);
    corlib::sfc_detail::check(sfc_covar_forcing_apply_constraints(cf, bc.data(), (int64_t)bc.size()), ctx, "bc");
    sfc_forward_gauss_t *fg = nullptr;
    corlib::sfc_detail::check(sfc_forward_gauss_create(sysmat.handle(), cf, reg, &fg), ctx, "ForwardGaussRHS");
    std::vector<int64_t> ip(ns + 1);
    std::vector<int32_t> ix(ns);
    std::vector<double> dv(ns, 1.0);
    for (int a = 0; a <= ns; ++a) ip[a] = a;
    for (int a = 0; a < ns; ++a) ix[a] = a;
    corlib::sfc_detail::check(sfc_forward_gauss_set_projection(fg, ns, ip.data(), ix.data(), dv.data()), ctx, "P");
    sfc_hparams_t hp{fsig, flen, rho, msig, mlen, eps};
    corlib::sfc_detail::check(sfc_forward_gauss_update(fg, &hp), ctx, "updateSolution");
    sfc_koh_t *koh = nullptr;
    corlib::sfc_detail::check(sfc_koh_create(fg, sc.data(), 1, &koh), ctx, "LikelihoodKOH");
    corlib::sfc_detail::check(sfc_koh_set_sensor_values(koh, Y.data(), no), ctx, "setSensorValues");
    std::vector<double> mean(numDofs);
    corlib::sfc_detail::check(sfc_koh_woodbury(koh, &hp, mean.data(), nullptr), ctx, "Woodbury");
    for (double v : mean) std::printf("%.12e\n", v);
    sfc_koh_destroy(koh);
    sfc_forward_gauss_destroy(fg);
    sfc_covar_forcing_destroy(cf);
    return 0;
}
