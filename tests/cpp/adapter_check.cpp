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
    return 0;
}
