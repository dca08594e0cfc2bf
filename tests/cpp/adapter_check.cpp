// Drives the header-only C++ adapter (include/mfs_b200_factorizer.hpp) on an
// analysis-only handle: symbolic factorization of a block path Hessian, sizes,
// nnz / flop estimates, the inverse permutation, and the reference's exception
// classes for calls that need a numeric factorization or a GPU.
#include "mfs_b200_factorizer.hpp"

#include <cstdio>
#include <vector>

int main() {
    const int64_t nb = 20;
    std::vector<int64_t> Ap(1, 0), Ai;
    for (int64_t j = 0; j < nb; ++j) {
        if (j > 0) Ai.push_back(j - 1);
        Ai.push_back(j);
        Ap.push_back(int64_t(Ai.size()));
    }
    mfs::BlockCSCView A;
    A.numBlocks = nb;
    A.blockSize = 3;
    A.Ap = Ap.data();
    A.Ai = Ai.data();
    mfs::B200Factorizer f(false, -1);
    f.factorizeSymbolic(A, {0, 1, 2});
    std::printf("n %zu n_reduced %zu nnz %zu flops %.1f symbolic %d\n", f.n(), f.n_reduced(), f.getFactorNNZ(),
                f.getFlopEstimate(), int(f.hasFactorization(mfs::CholeskySys::P)));
    const auto ip = f.getInversePermutation();
    std::printf("iperm");
    for (size_t k = 0; k < ip.size(); ++k) std::printf(" %zu", ip[k]);
    std::printf("\n");
    int caught = 0;
    try {
        std::vector<double> b(f.n(), 1.0), x;
        f.solve(b, x);
    } catch (const std::runtime_error &) {
        caught |= 1;
    }
    try {
        std::vector<double> vals(9 * Ai.size(), 0.0);
        A.Ax = vals.data();
        f.factorizeNumeric(A);
    } catch (const std::invalid_argument &) {
        caught |= 2;
    }
    try {
        mfs::BlockCSCView bad = A;
        std::vector<int64_t> badAi(Ai);
        badAi[1] = 5;           // a block below the diagonal: not an upper pattern
        bad.Ai = badAi.data();
        f.factorizeSymbolic(bad);
    } catch (const std::invalid_argument &) {
        caught |= 4;
    }
    std::printf("caught %d\n", caught);
    // pins, row maps and the separator forest (a fresh analysis: the failed one above
    // left the handle without a symbolic factorization)
    f.factorizeSymbolic(A, {0, 1, 2, 7});
    std::printf("fixed %d %zu posdef %d\n", int(f.hasFixedVars()), f.getFixedVars().size(), int(f.checkPosDef()));
    std::vector<double> x(f.n()), xr(f.n_reduced()), back(f.n());
    for (size_t i = 0; i < x.size(); ++i) x[i] = double(i) + 0.5;
    for (int permute = 0; permute < 2; ++permute) {
        f.removeFixedEntries(x.data(), xr.data(), permute != 0);
        std::printf("reduced%d", permute);
        for (double v : xr) std::printf(" %g", v);
        std::printf("\n");
        f.extractFullSolution(xr.data(), back.data(), permute != 0);
        std::printf("full%d", permute);
        for (double v : back) std::printf(" %g", v);
        std::printf("\n");
    }
    const auto nd = f.ndOrdering();
    std::printf("nd %d %zu %zu %d\n", int(nd.has_value()), nd ? nd->CParent.size() : 0, nd ? nd->CMember.size() : 0,
                nd ? nd->blockSize : 0);
    return 0;
}
