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

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mfs {

enum class CholeskySys { A, L, Lt, P, Pt };
enum class FactorizationType { None = 0, Symbolic = 1, Numeric = 2 };

// Separator forest of the last nested-dissection analysis (CholeskyFactorizerBase.hh:55-59):
// CParent per component (postordered, -1 for roots), CMember per analysis variable of the
// reduced ordering graph, at the block size the analysis ran at.
struct NDOrdering {
    std::vector<int64_t> CParent, CMember;
    int blockSize = 1;
};

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
        m_fixed.clear();
        m_rr.clear();
        m_prr.clear();
        check(mfs_symbolic(m_h, A.numBlocks, A.Ap, A.Ai, A.blockSize, pins.empty() ? nullptr : pins.data(),
                           int64_t(pins.size()), nullptr, nullptr, 0));
        int64_t nf = 0, nr = 0;
        check(mfs_info(m_h, &nf, &nr, nullptr, nullptr, nullptr, nullptr));
        m_n = size_t(nf);
        m_nr = size_t(nr);
        m_fixed.assign(pinnedVars.begin(), pinnedVars.end());
        std::sort(m_fixed.begin(), m_fixed.end());
        m_fixed.erase(std::unique(m_fixed.begin(), m_fixed.end()), m_fixed.end());
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
    bool checkPosDef() const { return factorizationType() == FactorizationType::Numeric; }
    // this provider never asks for an early symbolic analysis
    bool wantsSymbolicFactorizationRecompute() const { return false; }
    bool hasFixedVars() const { return !m_fixed.empty(); }
    const std::vector<size_t> &getFixedVars() const { return m_fixed; }

    // Separator forest of the last analysis; empty for orderings other than nested
    // dissection and without a symbolic factorization.
    std::optional<NDOrdering> ndOrdering() const {
        if (factorizationType() < FactorizationType::Symbolic) return std::nullopt;
        int64_t nc = 0, nm = 0;
        if (mfs_nd_ordering(m_h, &nc, &nm, nullptr, nullptr) != MFS_OK || nc == 0) return std::nullopt;
        NDOrdering out;
        out.CParent.resize(size_t(nc));
        out.CMember.resize(size_t(nm));
        check(mfs_nd_ordering(m_h, &nc, &nm, out.CParent.data(), out.CMember.data()));
        int64_t nsn = 0, nst = 0;
        int32_t vb = 1;
        check(mfs_supernodes(m_h, &nsn, &nst, &vb, nullptr, nullptr, nullptr, nullptr, nullptr));
        out.blockSize = vb;
        return out;
    }

    // x (n entries) -> its free entries (n_reduced), in the original order or in the
    // factorization's order (CholeskyFactorizerBase.hh:299-330)
    void removeFixedEntries(const double *x, double *xr, bool permute = false) const {
        const std::vector<int64_t> &map = rowMap(permute);
        for (size_t i = 0; i < m_n; ++i)
            if (map[i] >= 0) xr[map[i]] = x[i];
    }
    // free entries (n_reduced) -> a full vector with zeros on the pinned entries
    // (CholeskyFactorizerBase.hh:331-363)
    void extractFullSolution(const double *xr, double *x, bool permute = false) const {
        const std::vector<int64_t> &map = rowMap(permute);
        for (size_t i = 0; i < m_n; ++i) x[i] = map[i] >= 0 ? xr[map[i]] : 0.0;
    }

    // ---- stash (CatamariFactorizer.cc:925-948)
    void stashFactorization() {
        check(mfs_stash(m_h));
        m_stash_fixed = m_fixed;
    }
    bool hasStashedFactorization() const {
        int32_t v = 0;
        check(mfs_has_stash(m_h, &v));
        return v != 0;
    }
    void swapStashedFactorization() {
        check(mfs_swap_stash(m_h));
        std::swap(m_fixed, m_stash_fixed);
        m_rr.clear();
        m_prr.clear();
        int64_t nf = 0, nr = 0;
        check(mfs_info(m_h, &nf, &nr, nullptr, nullptr, nullptr, nullptr));
        m_n = size_t(nf);
        m_nr = size_t(nr);
    }
    void clearStashedFactorization() {
        check(mfs_clear_stash(m_h));
        m_stash_fixed.clear();
    }
    // The sizes follow the factorization state, as in the reference: after
    // clearFactors() a solve fails its size check until the next factorizeSymbolic.
    void clearFactors() {
        check(mfs_clear_factors(m_h));
        m_n = 0;
        m_nr = 0;
        m_fixed.clear();
        m_rr.clear();
        m_prr.clear();
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

    // full row -> reduced row (-1 when pinned), plain or in the factorization's order
    const std::vector<int64_t> &rowMap(bool permute) const {
        if (m_rr.size() != m_n) {
            if (m_n == 0 || factorizationType() < FactorizationType::Symbolic)
                throw std::runtime_error("no symbolic factorization");
            m_rr.assign(m_n, -1);
            size_t next = 0, f = 0;
            for (size_t i = 0; i < m_n; ++i) {
                while (f < m_fixed.size() && m_fixed[f] < i) ++f;
                if (f < m_fixed.size() && m_fixed[f] == i) continue;
                m_rr[i] = int64_t(next++);
            }
            std::vector<int64_t> iperm(m_nr), perm(m_nr);
            check(mfs_inverse_permutation(m_h, iperm.data()));
            for (size_t k = 0; k < m_nr; ++k) perm[size_t(iperm[k])] = int64_t(k);
            m_prr.assign(m_n, -1);
            for (size_t i = 0; i < m_n; ++i)
                if (m_rr[i] >= 0) m_prr[i] = perm[size_t(m_rr[i])];
        }
        return permute ? m_prr : m_rr;
    }

    mfs_handle *m_h = nullptr;
    size_t m_n = 0, m_nr = 0;
    std::vector<size_t> m_fixed, m_stash_fixed;    // sorted pinned scalar variables (current, stashed)
    mutable std::vector<int64_t> m_rr, m_prr;      // row maps (built on first use)
};

}  // namespace mfs

#endif  // MFS_B200_FACTORIZER_HPP
