// SystemSolveCuda.hpp -- drop-in replacement for corlib::SystemSolveEigenSparse
// (corlib/SystemSolveEigenSparse.hpp:40-158) backed by the B200 C ABI in
// statfem_cuda.h.  An application switches by changing its solver typedef
// (del2/apps/reference/laplaceRHSinfer/laplaceRHSinfer.cpp:99):
//
//     typedef corlib::SystemSolveCuda SysSolve;
//
// The method set and argument meaning are those of SystemSolveEigenSparse.
// Local matrices / vectors are templates, so Eigen::MatrixXd, Eigen
// expressions (e.g. the transposed element matrix MatrixAssembler passes when
// TRANS is set, corlib/MatrixAssembler.hpp:224-229) or any type with
// operator()(i, j) / operator()(i) and rows() / size() work; the header does not
// include Eigen itself.
//
// Errors: the reference aborts through FTL_VERIFY (corlib/verify.hpp:61-70);
// this class does the same (message to stderr, abort()) unless
// SFC_THROW_ON_ERROR is defined, in which case it throws std::runtime_error.
#ifndef corlib_systemsolvecuda_h
#define corlib_systemsolvecuda_h

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../statfem_cuda.h"

namespace corlib {

namespace sfc_detail {

inline void check(int rc, sfc_ctx_t *ctx, const char *what)
{
    if (rc == SFC_OK) return;
    std::string msg = std::string(what) + " failed (" + std::to_string(rc) + "): " + sfc_last_error(ctx);
#ifdef SFC_THROW_ON_ERROR
    throw std::runtime_error(msg);
#else
    std::fprintf(stderr, "FTL_VERIFY failed: %s\n", msg.c_str());
    std::abort();
#endif
}

// one context per host thread and device, created on first use
inline sfc_ctx_t *context(int device)
{
    thread_local std::vector<sfc_ctx_t *> ctxs;
    if ((int)ctxs.size() <= device) ctxs.resize(device + 1, nullptr);
    if (!ctxs[device]) {
        sfc_ctx_t *c = nullptr;
        int rc = sfc_ctx_create(device, &c);
        if (rc != SFC_OK) {
            std::fprintf(stderr, "FTL_VERIFY failed: no CUDA device %d (%d)\n", device, rc);
            std::abort();
        }
        ctxs[device] = c;
    }
    return ctxs[device];
}

}  // namespace sfc_detail

class SystemSolveCuda
{
public:
    typedef std::vector<unsigned> VectorUInt_;
    typedef std::vector<std::pair<unsigned, double> > VectorConstraint_;

    //! Construct with number of dofs (matrix size), as SystemSolveEigenSparse
    explicit SystemSolveCuda(const unsigned &numDofs, int device = 0)
        : numDofs_(numDofs), ctx_(sfc_detail::context(device))
    {
        sfc_detail::check(sfc_system_create(ctx_, numDofs, &sys_), ctx_, "SystemSolveCuda");
    }

    ~SystemSolveCuda() { sfc_system_destroy(sys_); }

    SystemSolveCuda(const SystemSolveCuda &) = delete;
    SystemSolveCuda &operator=(const SystemSolveCuda &) = delete;

    //! @name Insertion routines (SystemSolveEigenSparse.hpp:160-184)
    //@{
    template <typename MAT>
    void insertToMatrix(const MAT &eStiff, const VectorUInt_ &rowIndices, const VectorUInt_ &colIndices)
    {
        const unsigned n = rowIndices.size(), m = colIndices.size();
        buf_.resize((size_t)n * m);
        for (unsigned i = 0; i < n; ++i)
            for (unsigned j = 0; j < m; ++j) buf_[(size_t)i * m + j] = eStiff(i, j);
        sfc_detail::check(sfc_insert_matrix(sys_, buf_.data(), rowIndices.data(), n, colIndices.data(), m), ctx_,
                          "insertToMatrix");
    }

    template <typename VEC>
    void insertToRhs(const VEC &eForce, const VectorUInt_ &dofIndices)
    {
        const unsigned n = dofIndices.size();
        buf_.resize(n);
        for (unsigned i = 0; i < n; ++i) buf_[i] = eForce(i);
        sfc_detail::check(sfc_insert_rhs(sys_, buf_.data(), dofIndices.data(), n), ctx_, "insertToRhs");
    }
    //@}

    //! @name Constraint routines (SystemSolveEigenSparse.hpp:197-226)
    //@{
    void applyConstraints(const VectorConstraint_ &constraints, const double factor, const double scalar)
    {
        std::vector<uint32_t> idx;
        std::vector<double> val;
        idx.reserve(constraints.size());
        val.reserve(constraints.size());
        for (const auto &c : constraints) {
            idx.push_back(c.first);
            val.push_back(c.second);
        }
        sfc_detail::check(sfc_apply_constraints(sys_, idx.data(), val.data(), (int64_t)idx.size(), factor, scalar),
                          ctx_, "applyConstraints");
    }

    void fixDOF(const unsigned index, const double scalar = 1.)
    {
        sfc_detail::check(sfc_fix_dof(sys_, index, scalar), ctx_, "fixDOF");
    }
    //@}

    //! Debug writing of matrix: "row  col  value" lines (Triplet::write)
    void writeMatrix(std::ostream &out)
    {
        std::vector<int64_t> rp(numDofs_ + 1);
        std::vector<int32_t> col(numNonZeros());
        std::vector<double> val(col.size());
        sfc_detail::check(sfc_get_csr(sys_, rp.data(), col.data(), val.data()), ctx_, "writeMatrix");
        for (unsigned i = 0; i < numDofs_; ++i)
            for (int64_t s = rp[i]; s < rp[i + 1]; ++s)
                out << i << "  " << col[s] << "  " << std::setprecision(12) << val[s] << std::endl;
    }

    //! Debug writing of right hand side
    void writeRhs(std::ostream &out)
    {
        std::vector<double> F = vec_(&sfc_give_force);
        out << std::setprecision(6);
        for (double v : F) out << v << "\n";
    }

    //! @name Norms (SystemSolveEigenSparse.hpp:78-83)
    //@{
    double normMatrix() { return norms_()[0]; }
    double normRhs() const { return norms_()[1]; }
    double norm1Rhs() const { return norms_()[2]; }
    double normSol() const { return norms_()[3]; }
    //@}

    //! flush host-staged insertions to the device (no-ops in the reference)
    void finishRhsAssembly() { finishAssembly(); }
    void finishMatAssembly() { finishAssembly(); }
    void finishAssembly() { sfc_detail::check(sfc_finish_assembly(sys_), ctx_, "finishAssembly"); }

    //! @name Solve (SystemSolveEigenSparse.hpp:273-404)
    //@{
    void solveSystem() { sfc_detail::check(sfc_solve(sys_, 0), ctx_, "solveSystem"); }
    void solveSystem(const bool reuseFactoredMatrix)
    {
        sfc_detail::check(sfc_solve(sys_, reuseFactoredMatrix ? 1 : 0), ctx_, "solveSystem");
    }
    template <typename VIN, typename VOUT>
    void solveSystemTranspose(const VIN &rhsVec, VOUT &uVec, const bool reuseFactoredMatrix)
    {
        std::vector<double> r(numDofs_), u(numDofs_);
        for (unsigned i = 0; i < numDofs_; ++i) r[i] = rhsVec(i);
        sfc_detail::check(sfc_solve_transpose(sys_, r.data(), u.data(), 1, reuseFactoredMatrix ? 1 : 0), ctx_,
                          "solveSystemTranspose");
        uVec.resize(numDofs_);
        for (unsigned i = 0; i < numDofs_; ++i) uVec(i) = u[i];
    }
    //@}

    //! Clear matrix (values zeroed, pattern kept) / RHS storage
    void clearMatrix() { sfc_detail::check(sfc_clear_matrix(sys_), ctx_, "clearMatrix"); }
    void clearRhs() { sfc_detail::check(sfc_clear_rhs(sys_), ctx_, "clearRhs"); }

    //! Solution accessor (result must already have dofIndices.size() entries)
    template <typename VEC>
    void giveSolution(const VectorUInt_ &dofIndices, VEC &result) const
    {
        give_(&sfc_give_solution, dofIndices, result);
    }
    //! Force accessor
    template <typename VEC>
    void giveForce(const VectorUInt_ &dofIndices, VEC &result) const
    {
        give_(&sfc_give_force, dofIndices, result);
    }

    unsigned numNonZeros() const { return (unsigned)sfc_num_nonzeros(sys_); }

    //! @name GPU extensions (no reference counterpart)
    //@{
    void setOptions(const sfc_solver_options_t &opt)
    {
        sfc_detail::check(sfc_system_set_options(sys_, &opt), ctx_, "setOptions");
    }
    sfc_solver_options_t options() const
    {
        sfc_solver_options_t opt;
        sfc_detail::check(sfc_system_get_options(sys_, &opt), ctx_, "options");
        return opt;
    }
    sfc_solve_stats_t lastStats() const
    {
        sfc_solve_stats_t st;
        sfc_detail::check(sfc_system_last_stats(sys_, &st), ctx_, "lastStats");
        return st;
    }
    sfc_system_t *handle() const { return sys_; }
    sfc_ctx_t *context() const { return ctx_; }
    unsigned numDofs() const { return numDofs_; }
    //@}

private:
    typedef int32_t (*GiveFn)(const sfc_system_t *, const uint32_t *, int64_t, double *);

    std::vector<double> vec_(GiveFn fn) const
    {
        std::vector<uint32_t> d(numDofs_);
        for (unsigned i = 0; i < numDofs_; ++i) d[i] = i;
        std::vector<double> v(numDofs_);
        sfc_detail::check(fn(sys_, d.data(), numDofs_, v.data()), ctx_, "give");
        return v;
    }

    template <typename VEC>
    void give_(GiveFn fn, const VectorUInt_ &dofIndices, VEC &result) const
    {
        std::vector<double> v(dofIndices.size());
        sfc_detail::check(fn(sys_, dofIndices.data(), (int64_t)dofIndices.size(), v.data()), ctx_, "give");
        for (size_t i = 0; i < v.size(); ++i) result[i] = v[i];
    }

    std::vector<double> norms_() const
    {
        std::vector<double> n(4, 0.0);
        sfc_detail::check(sfc_norms(sys_, &n[0], &n[1], &n[2], &n[3]), ctx_, "norms");
        return n;
    }

    const unsigned numDofs_;
    sfc_ctx_t *ctx_ = nullptr;
    sfc_system_t *sys_ = nullptr;
    std::vector<double> buf_;
};

}  // namespace corlib

#endif
