// GpuMatrixAssembler.hpp -- GPU replacement for the element loop
//     corlib::MatrixComputeAndAssembleFun<Element,Quad,Solver> maf(...);
//     mesh.iterateOverElements(maf);
// (corlib/MatrixAssembler.hpp:43-100, del2/apps/reference/laplaceRHSinfer/fem.hpp:69-74)
// and for the body-force Integrator + VectorAssembler pair (fem.hpp:77-90).
//
// Applied to every element through mesh.iterateOverElements(gpuAssembler), it
// records the element's node coordinates, dof indices and coefficient (the
// element's conductivity, or any functor the caller passes); assemble() then
// uploads the mesh once (the GPU builds the CSR pattern and the sorted-key
// gather map) and computes every element matrix and the global matrix on the
// device, with the reference's quadrature and integrand arithmetic.  Later
// calls re-use the mesh and only upload new coefficients, which is what a
// material-proposal loop needs (laplaceInverse's giveFEsolution).
//
// Requirements on ELEMENT (duck-typed like the reference's own functors):
// getDofIndices(std::vector<unsigned>&), nodesBegin()/nodesEnd() over node
// pointers with giveCoordinates() returning a vector with operator()(i) and
// size() or rows(); dofs numbered node-interleaved (Node::numberDOFs in node
// order, del2/fem/NodePotential.hpp:65).
#ifndef corlib_gpumatrixassembler_h
#define corlib_gpumatrixassembler_h

#include <cstdint>
#include <vector>

#include "SystemSolveCuda.hpp"

namespace corlib {

template <typename ELEMENT>
struct ConductivityOf {
    double operator()(const ELEMENT *ep) const { return ep->getConductivity(); }
};

template <typename ELEMENT, typename COEFF = ConductivityOf<ELEMENT> >
class GpuMatrixAssembler
{
public:
    GpuMatrixAssembler(SystemSolveCuda *solver, int elementKind, int quadPoints, double poissonRatio = 0.3,
                       COEFF coeff = COEFF())
        : solver_(solver), kind_(elementKind), qps_(quadPoints), nu_(poissonRatio), coeff_(coeff)
    {
        dofsPerNode_ = elementKind == SFC_ELEM_HEX8_ELASTIC ? 3 : 1;
    }

    ~GpuMatrixAssembler()
    {
        if (mesh_) sfc_mesh_destroy(mesh_);
    }

    GpuMatrixAssembler(const GpuMatrixAssembler &) = delete;
    GpuMatrixAssembler &operator=(const GpuMatrixAssembler &) = delete;

    //! functor applied to each element by Mesh::iterateOverElements
    void operator()(ELEMENT *ep)
    {
        std::vector<unsigned> dofs;
        ep->getDofIndices(dofs);
        unsigned k = 0;
        for (auto it = ep->nodesBegin(); it != ep->nodesEnd(); ++it, ++k) {
            const unsigned node = dofs[k * dofsPerNode_] / dofsPerNode_;
            if (!mesh_) {
                conn_.push_back(node);
                if (coords_.size() < 3 * (size_t)(node + 1)) coords_.resize(3 * (size_t)(node + 1), 0.0);
                const auto x = (*it)->giveCoordinates();
                for (int a = 0; a < (int)dimOf_(x) && a < 3; ++a) coords_[3 * (size_t)node + a] = x(a);
            }
        }
        coefficients_.push_back(coeff_(ep));
    }

    //! upload (first call: mesh + pattern), compute, and assemble the matrix
    void assemble()
    {
        sfc_ctx_t *ctx = solver_->context();
        if (!mesh_) {
            const int64_t nn = kind_ == SFC_ELEM_LINE2_POISSON ? 2 : kind_ == SFC_ELEM_TRI3_POISSON ? 3 : 8;
            sfc_detail::check(sfc_mesh_create(ctx, kind_, qps_, coords_.data(), (int64_t)coords_.size() / 3,
                                              conn_.data(), (int64_t)conn_.size() / nn, &mesh_),
                              ctx, "GpuMatrixAssembler mesh");
        }
        sfc_detail::check(sfc_mesh_set_coefficients(mesh_, coefficients_.data(), 0.0, nu_), ctx,
                          "GpuMatrixAssembler coefficients");
        sfc_detail::check(sfc_assemble_matrix(solver_->handle(), mesh_), ctx, "GpuMatrixAssembler");
        coefficients_.clear();
    }

    //! body force f (one value per dof component) on the GPU, added to F
    void assembleLoad(const double *f)
    {
        sfc_detail::check(sfc_assemble_load(solver_->handle(), mesh_, f), solver_->context(), "assembleLoad");
    }

    sfc_mesh_t *mesh() const { return mesh_; }

private:
    template <typename V>
    static auto dimOf_(const V &x) -> decltype(x.size())
    {
        return x.size();
    }

    SystemSolveCuda *solver_;
    int kind_, qps_;
    double nu_;
    COEFF coeff_;
    unsigned dofsPerNode_ = 1;
    sfc_mesh_t *mesh_ = nullptr;
    std::vector<double> coords_;
    std::vector<uint32_t> conn_;
    std::vector<double> coefficients_;
};

}  // namespace corlib

#endif
