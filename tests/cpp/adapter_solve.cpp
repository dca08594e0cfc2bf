// The C++ host interface on the GPU: factor and solve the reference's block path
// matrix (tests/test_catamari_factorizer.cc:100-110 values) in FP64 and in FP32 with
// FP64 refinement; prints the relative residual of each solve.
#include "mfs_b200_factorizer.hpp"

#include <cmath>
#include <cstdio>
#include <vector>

int main() {
    const int64_t nb = 40, bs = 3, n = nb * bs;
    std::vector<int64_t> Ap(1, 0), Ai;
    for (int64_t j = 0; j < nb; ++j) {
        if (j > 0) Ai.push_back(j - 1);
        Ai.push_back(j);
        Ap.push_back(int64_t(Ai.size()));
    }
    // scalar (i, j) of block k at Ax[9k + 3c + r]; dense copy for the residual
    std::vector<double> Ax(9 * Ai.size(), 0.0), M(size_t(n * n), 0.0);
    for (int64_t bj = 0; bj < nb; ++bj)
        for (int64_t k = Ap[bj]; k < Ap[bj + 1]; ++k)
            for (int c = 0; c < bs; ++c)
                for (int r = 0; r < bs; ++r) {
                    const int64_t i = Ai[k] * bs + r, j = bj * bs + c;
                    if (i > j) continue;
                    const double v = (i == j) ? 10.1 : -0.1 * double(1 + (i + j) % 5);
                    Ax[9 * k + 3 * c + r] = v;
                    M[i * n + j] = M[j * n + i] = v;
                }
    mfs::BlockCSCView A;
    A.numBlocks = nb;
    A.blockSize = int32_t(bs);
    A.Ap = Ap.data();
    A.Ai = Ai.data();
    A.Ax = Ax.data();
    std::vector<double> b(n), x;
    for (int64_t i = 0; i < n; ++i) b[i] = std::sin(0.37 * double(i + 1));
    for (int single = 0; single < 2; ++single) {
        mfs::B200Factorizer f(single != 0, 0, true);
        f.factorize(A);
        f.solve(b, x);
        double rn = 0, bn = 0;
        for (int64_t i = 0; i < n; ++i) {
            double s = 0;
            for (int64_t j = 0; j < n; ++j) s += M[i * n + j] * x[j];
            rn += (b[i] - s) * (b[i] - s);
            bn += b[i] * b[i];
        }
        std::printf("%s residual %.3e\n", single ? "fp32+refine" : "fp64", std::sqrt(rn / bn));
    }
    return 0;
}
