// mfs_b200_factorizer.hpp -- header-only C++ host interface over the C ABI of
// mfs_b200.h, shaped like the reference's CholeskyFactorizerBase
// (Solvers/CholeskyFactorizerBase.hh:50-443) so C++ callers keep their calls:
// factorizeSymbolic / factorizeNumeric / factorizeNumericWithShift / factorize,
// solve / solveMultiRHS / solveRawReduced[InPlace], stash / swap / clear,
// getFactorNNZ / getFlopEstimate / getInversePermutation, m / n / m_reduced /
// n_reduced. Failures throw like the reference: a failed pivot or a missing
// factorization throws std::runtime_error (the factorizer drops back to its
// symbolic state, CatamariFactorizer.cc:701-705); bad sizes or arguments throw
// std::invalid_argument. Matrices are borrowed views of the caller's
// upper block-CSC Hessian (BlockCSCHessian<..., ContiguousBlocks=true>:
// Ap/Ai block pattern, Ax bs*bs scalars per block, column-major).
#ifndef MFS_B200_FACTORIZER_HPP
#define MFS_B200_FACTORIZER_HPP

#include "mfs_b200.h"

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mfs {

enum class CholeskySys { A, L, Lt, P, Pt };
enum class FactorizationType { None = 0, Symbolic = 1, Numeric = 2 };

// Borrowed view of an upper block-CSC Hessian.
struct BlockCSCView {
    int64_t numBlocks = 0;
    int32_t blockSize = 3;
    const int64_t *Ap = nullptr;    // numBlocks + 1
    const int64_t *Ai = nullptr;    // Ap[numBlocks]
    const double *Ax = nullptr;     // blockSize^2 * Ap[numBlocks], or null for a pattern only
};

class B200Factorizer {
public:
    // device -1: analysis only (ordering, supernodes, plan on the host, no GPU state)
    explicit B200Factorizer(bool singlePrecision = false, int device = 0, bool refine = true) {
        mfs_options o;
        check(mfs_default_options(&o));
        o.precision = singlePrecision ? MFS_PREC_FP32 : MFS_PREC_FP64;
        o.refine = (singlePrecision && refine) ? 1 : 0;
        o.device = device;
        check(mfs_create(&m_h, &o));
    }
    ~B200Factorizer() {
        if (m_h) mfs_destroy(m_h);
    }
    B200Factorizer(const B200Factorizer &) = delete;
    B200Factorizer &operator=(const B200Factorizer &) = delete;
    B200Factorizer(B200Factorizer &&o) noexcept { *this = std::move(o); }
    B200Factorizer &operator=(B200Factorizer &&o) noexcept {
        std::swap(m_h, o.m_h);
        std::swap(m_n, o.m_n);
        std::swap(m_nr, o.m_nr);
        return *this;
    }

    // ---- factorization
    void factorizeSymbolic(const BlockCSCView &A, const std::vector<size_t> &pinnedVars = {}) {
        std::vector<int64_t> pins(pinnedVars.begin(), pinnedVars.end());
        check(mfs_symbolic(m_h, A.numBlocks, A.Ap, A.Ai, A.blockSize, pins.empty() ? nullptr : pins.data(),
                           int64_t(pins.size()), nullptr, nullptr, 0));
        int64_t nf = 0, nr = 0;
        check(mfs_info(m_h, &nf, &nr, nullptr, nullptr, nullptr, nullptr));
        m_n = size_t(nf);
        m_nr = size_t(nr);
    }
    void factorizeNumeric(const BlockCSCView &A, bool /* isInTryCatch */ = false) {
        check(mfs_numeric(m_h, values(A), nullptr, 0.0, 0));
    }
    void factorizeNumericWithShift(const BlockCSCView &A, double sigma, bool /* isInTryCatch */ = false) {
        check(mfs_numeric(m_h, values(A), nullptr, sigma, 0));
    }
    // A + sigma B, B with A's pattern and layout
    void factorizeNumericWithShift(const BlockCSCView &A, double sigma, const BlockCSCView &B,
                                   bool /* isInTryCatch */ = false) {
        if (B.Ap != A.Ap && (B.numBlocks != A.numBlocks || B.blockSize != A.blockSize))
            throw std::invalid_argument("Shift matrix must have the same sparsity and value layout as A");
        check(mfs_numeric(m_h, values(A), values(B), sigma, 0));
    }
    void factorize(const BlockCSCView &A, const std::vector<size_t> &fixedVars = {}, bool = false) {
        factorizeSymbolic(A, fixedVars);
        factorizeNumeric(A);
    }

    // ---- solves (x may alias b)
    void solve(const std::vector<double> &b, std::vector<double> &x, CholeskySys sys = CholeskySys::A) const {
        if (sys != CholeskySys::A) throw std::runtime_error("Only CholeskySys::A is supported");
        if (b.size() != m_n) throw std::runtime_error("CholeskyFactorizerBase::solve: incorrect b size");
        x = b;
        check(mfs_solve(m_h, x.data(), x.data(), 1, int64_t(m_n), MFS_SOLVE_FULL));
    }
    // column-major B, X (ld rows), nrhs columns
    void solveMultiRHS(const double *B, double *X, int64_t nrhs, int64_t ld) const {
        check(mfs_solve(m_h, B, X, nrhs, ld, MFS_SOLVE_FULL));
    }
    void solveRawReduced(const double *b, double *x, CholeskySys sys = CholeskySys::A,
                         bool alreadyPermuted = false) const {
        if (sys != CholeskySys::A) throw std::runtime_error("Only CholeskySys::A is supported");
        check(mfs_solve(m_h, b, x, 1, int64_t(m_nr),
                        alreadyPermuted ? MFS_SOLVE_REDUCED_PERMUTED : MFS_SOLVE_REDUCED));
    }
    void solveRawReducedInPlace(double *bx, CholeskySys sys = CholeskySys::A, bool alreadyPermuted = false) const {
        solveRawReduced(bx, bx, sys, alreadyPermuted);
    }

    // ---- sizes and introspection
    size_t m() const { return m_n; }
    size_t n() const { return m_n; }
    size_t m_reduced() const { return m_nr; }
    size_t n_reduced() const { return m_nr; }
    FactorizationType factorizationType() const {
        int64_t nf, nr, nnz, nsn;
        double fl;
        int32_t t = 0;
        if (mfs_info(m_h, &nf, &nr, &nnz, &fl, &nsn, &t) != MFS_OK) return FactorizationType::None;
        return FactorizationType(t);
    }
    bool hasFactorization(CholeskySys sys = CholeskySys::A) const {
        const FactorizationType t = factorizationType();
        if (sys == CholeskySys::A || sys == CholeskySys::L || sys == CholeskySys::Lt)
            return t >= FactorizationType::Numeric;
        return t >= FactorizationType::Symbolic;
    }
    size_t getFactorNNZ() const {
        int64_t v = 0;
        check(mfs_info(m_h, nullptr, nullptr, &v, nullptr, nullptr, nullptr));
        return size_t(v);
    }
    double getFlopEstimate() const {
        double v = 0;
        check(mfs_info(m_h, nullptr, nullptr, nullptr, &v, nullptr, nullptr));
        return v;
    }
    std::vector<size_t> getInversePermutation() const {
        std::vector<int64_t> p(m_nr);
        check(mfs_inverse_permutation(m_h, p.data()));
        return std::vector<size_t>(p.begin(), p.end());
    }
    bool preferInPlaceSolve() const { return true; }
    bool supportsPrePermutation() const { return true; }

    // ---- stash (CatamariFactorizer.cc:925-948)
    void stashFactorization() { check(mfs_stash(m_h)); }
    bool hasStashedFactorization() const {
        int32_t v = 0;
        check(mfs_has_stash(m_h, &v));
        return v != 0;
    }
    void swapStashedFactorization() {
        check(mfs_swap_stash(m_h));
        int64_t nf = 0, nr = 0;
        check(mfs_info(m_h, &nf, &nr, nullptr, nullptr, nullptr, nullptr));
        m_n = size_t(nf);
        m_nr = size_t(nr);
    }
    void clearStashedFactorization() { check(mfs_clear_stash(m_h)); }
    // The sizes follow the factorization state, as in the reference: after
    // clearFactors() a solve fails its size check until the next factorizeSymbolic.
    void clearFactors() {
        check(mfs_clear_factors(m_h));
        m_n = 0;
        m_nr = 0;
    }

    mfs_handle *handle() const { return m_h; }

private:
    static const double *values(const BlockCSCView &A) {
        if (!A.Ax) throw std::invalid_argument("matrix has no values (pattern only)");
        return A.Ax;
    }
    void check(mfs_status s) const {
        if (s == MFS_OK) return;
        std::string msg = "mfs status " + std::to_string(int(s));
        if (m_h) {
            char buf[1024];
            if (mfs_last_error(m_h, buf, sizeof buf) == MFS_OK && buf[0]) msg = buf;
        }
        if (s == MFS_INVALID_ARG || s == MFS_SIZE_MISMATCH) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }

    mfs_handle *m_h = nullptr;
    size_t m_n = 0, m_nr = 0;
};

}  // namespace mfs

#endif  // MFS_B200_FACTORIZER_HPP
