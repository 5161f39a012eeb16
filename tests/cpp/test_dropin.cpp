// The reference's own function tests (tests/testcases/function/distributed/
// ttm.cpp TTM1, gram.cpp Gram1) written against the drop-in C++ API at world
// size 1, plus HOOI_ALS / Sp_HOOI_ALS smoke checks.  The input tensor and the
// expected values come from the golden fixture (argv[1], whitespace separated:
// 60 tensor values, 40 TTM1 values, 16 Gram1 values).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "diana/algorithm.hpp"

static int failures = 0;
#define EXPECT(cond, ...)                        \
    do {                                         \
        if (!(cond)) {                           \
            std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
            std::printf(__VA_ARGS__);            \
            std::printf("\n");                   \
            failures++;                          \
        }                                        \
    } while (0)

int main(int argc, char **argv) {
    if (argc < 2) {
        std::printf("usage: test_dropin <known-answers.txt>\n");
        return 2;
    }
    std::ifstream in(argv[1]);
    std::vector<double> tv(60), ttm_gt(40), gram_gt(16);
    for (auto &v : tv) in >> v;
    for (auto &v : ttm_gt) in >> v;
    for (auto &v : gram_gt) in >> v;

    mpi_init();
    auto *distribution = new DistributionCartesianBlock({1, 1, 1}, mpi_rank());
    Tensor<double> t(distribution, {5, 4, 3});
    for (size_t i = 0; i < t.size(); i++) t[i] = tv[i];

    // TTM1
    {
        auto *dis_global = new DistributionGlobal();
        Tensor<double> m1(dis_global, {4, 4});
        for (size_t i = 0; i < m1.size(); i++) m1[i] = (double)i;
        Tensor<double> m2(dis_global, {2, 3});
        for (size_t i = 0; i < m2.size(); i++) m2[i] = (double)i;
        auto r = Function::ttm<double>(t, m1, 1);
        r = Function::ttm<double>(r, m2, 2);
        EXPECT(r.size() == 40, "TTM1 size %zu", r.size());
        for (size_t i = 0; i < r.size(); i++)
            EXPECT(r[i] == ttm_gt[i], "TTM1[%zu] = %.17g, expected %.17g", i, r[i], ttm_gt[i]);
    }
    // Gram1
    {
        auto ans = Function::gram<double>(t, 1);
        for (size_t i = 0; i < ans.size(); i++)
            EXPECT(ans[i] == gram_gt[i], "Gram1[%zu] = %.17g, expected %.17g", i, ans[i],
                   gram_gt[i]);
    }
    // Matrix functions.
    {
        Tensor<double> A({6, 3}, false);
        srand(7);
        A.randn();
        auto [q, r] = Function::reduced_QR<double>(A);
        auto qtq = Function::matmulTN<double>(q, q);
        for (size_t i = 0; i < 3; i++)
            for (size_t j = 0; j < 3; j++)
                EXPECT(std::fabs(qtq[i + 3 * j] - (i == j)) < 1e-13, "Q^T Q");
        auto qr = Function::matmulNN<double>(q, r);
        for (size_t i = 0; i < A.size(); i++) EXPECT(std::fabs(qr[i] - A[i]) < 1e-12, "QR = A");
        auto g = Function::matmulTN<double>(A, A);
        auto gi = Function::inverse<double>(g);
        auto id = Function::matmulNN<double>(g, gi);
        for (size_t i = 0; i < 3; i++)
            for (size_t j = 0; j < 3; j++)
                EXPECT(std::fabs(id[i + 3 * j] - (i == j)) < 1e-10, "G G^-1 = I");
    }
    // HOOI_ALS on a random 30 x 20 x 10 tensor, seeded like the reference's main.
    {
        srand((unsigned int)20000905);
        auto *dist = new DistributionCartesianBlock({1, 1, 1}, mpi_rank());
        Tensor<double> T(dist, {30, 20, 10});
        T.randn();
        auto [G, U] = Algorithm::Tucker::HOOI_ALS(T, {4, 3, 2}, 4);
        EXPECT(G.size() == 24 && U.size() == 3, "HOOI_ALS output shapes");
        const double gn = G.fnorm(), an = T.fnorm();
        EXPECT(gn > 0 && gn <= an, "||G|| %.6g vs ||A|| %.6g", gn, an);
        for (size_t n = 0; n < 3; n++) {
            auto utu = Function::matmulTN<double>(U[n], U[n]);
            const size_t r = U[n].shape()[1];
            for (size_t i = 0; i < r; i++)
                for (size_t j = 0; j < r; j++)
                    EXPECT(std::fabs(utu[i + r * j] - (i == j)) < 1e-12, "U^T U = I");
        }
    }
    // Sp_HOOI_ALS on a small COO tensor built as a data_buffer.
    {
        const size_t nnz = 400;
        auto *dbf = new data_buffer<double>();
        dbf->ndim = 3;
        dbf->nnz = nnz;
        dbf->dims = new size_t[3]{40, 30, 20};
        dbf->index_lists = (size_t **)std::malloc(3 * sizeof(size_t *));
        for (int m = 0; m < 3; m++) dbf->index_lists[m] = (size_t *)std::malloc(nnz * sizeof(size_t));
        dbf->vals = (double *)std::malloc(nnz * sizeof(double));
        srand(3);
        for (size_t e = 0; e < nnz; e++) {
            for (int m = 0; m < 3; m++) dbf->index_lists[m][e] = (size_t)(std::rand() % dbf->dims[m]);
            dbf->vals[e] = 1.0 + (double)(std::rand() % 100) / 10.0;
        }
        SpTensor<double> A(dbf);
        auto [G, Ut] = Algorithm::SpTucker::Sp_HOOI_ALS(A, {4, 4, 4}, 2);
        const double gn = G.fnorm(), an = Function::fnorm(A);
        EXPECT(gn > 0 && gn <= an * (1 + 1e-12), "sparse ||G|| %.6g vs ||A|| %.6g", gn, an);
        EXPECT(Ut.size() == 3 && Ut[0].shape()[0] == 4 && Ut[0].shape()[1] == 40, "Ut shapes");
    }
    // Function::ttmc / mettmc of a sparse tensor to a dense one, against the
    // drop-in's dense Function::ttm chain on the densified tensor.
    {
        const size_t nnz = 300;
        const size_t dims[3] = {12, 9, 7};
        auto *dbf = new data_buffer<double>();
        dbf->ndim = 3;
        dbf->nnz = nnz;
        dbf->dims = (size_t *)std::malloc(3 * sizeof(size_t));
        for (int m = 0; m < 3; m++) dbf->dims[m] = dims[m];
        dbf->index_lists = (size_t **)std::malloc(3 * sizeof(size_t *));
        for (int m = 0; m < 3; m++) dbf->index_lists[m] = (size_t *)std::malloc(nnz * sizeof(size_t));
        dbf->vals = (double *)std::malloc(nnz * sizeof(double));
        srand(11);
        Tensor<double> dense({dims[0], dims[1], dims[2]}, true);
        for (size_t e = 0; e < nnz; e++) {
            size_t lin = 0, st = 1;
            for (int m = 0; m < 3; m++) {
                dbf->index_lists[m][e] = (size_t)(std::rand() % dims[m]);
                lin += dbf->index_lists[m][e] * st;
                st *= dims[m];
            }
            dbf->vals[e] = (double)(std::rand() % 1000) / 100.0 - 5.0;
            dense[lin] += dbf->vals[e];
        }
        SpTensor<double> A(dbf);
        std::vector<Tensor<double>> M;
        for (int m = 0; m < 3; m++) {
            Tensor<double> Mm({(size_t)(3 + m), dims[m]}, false);
            for (size_t i = 0; i < Mm.size(); i++) Mm[i] = std::sin(0.37 * (double)(i + 11 * m));
            M.push_back(Mm);
        }
        auto *dist = new DistributionCartesianBlock({1, 1, 1}, mpi_rank());
        auto Y = Function::ttmc(A, M, {2, 0}, dist, true);
        auto Yd = Function::ttm(Function::ttm(dense, M[2], 2), M[0], 0);
        EXPECT(Y.shape() == Yd.shape(), "ttmc shape");
        double err = 0.0, mx = 0.0;
        for (size_t i = 0; i < Yd.size(); i++) {
            err = std::fmax(err, std::fabs(Y[i] - Yd[i]));
            mx = std::fmax(mx, std::fabs(Yd[i]));
        }
        EXPECT(err <= 1e-12 * mx, "ttmc vs dense chain: %.3g", err / mx);
        for (size_t level = 0; level <= 3; level++) {
            auto Ym = Function::mettmc(A, M, {0, 1, 2}, dist, false, level);
            auto Yf = Function::ttm(Function::ttm(Function::ttm(dense, M[0], 0), M[1], 1), M[2], 2);
            double e2 = 0.0, m2 = 0.0;
            for (size_t i = 0; i < Yf.size(); i++) {
                e2 = std::fmax(e2, std::fabs(Ym[i] - Yf[i]));
                m2 = std::fmax(m2, std::fabs(Yf[i]));
            }
            EXPECT(Ym.shape() == Yf.shape() && e2 <= 1e-12 * m2, "mettmc level %zu: %.3g", level,
                   e2 / m2);
        }
    }
    // read_data on a small .tns file (1-based indices), then SpTensor from it.
    {
        const std::string tns = std::string(argv[1]) + ".tns";
        const char *path = tns.c_str();
        FILE *f = std::fopen(path, "w");
        std::fprintf(f, "1 2 3 1.5\n4 1 2 2.25\n2 2 1 -0.5\n");
        std::fclose(f);
        auto *dbf = new data_buffer<double>();
        read_data<double>(const_cast<char *>(path), dbf);
        EXPECT(dbf->ndim == 3 && dbf->nnz == 3, "read_data ndim %zu nnz %zu", dbf->ndim, dbf->nnz);
        EXPECT(dbf->dims[0] == 4 && dbf->dims[1] == 2 && dbf->dims[2] == 3, "read_data dims");
        EXPECT(dbf->index_lists[0][1] == 3 && dbf->index_lists[2][0] == 2 && dbf->vals[1] == 2.25 &&
                   dbf->vals[2] == -0.5,
               "read_data entries");
        SpTensor<double> A(dbf);
        const double an = Function::fnorm(A);
        EXPECT(std::fabs(an - std::sqrt(1.5 * 1.5 + 2.25 * 2.25 + 0.25)) < 1e-14, "fnorm %.17g", an);
        std::remove(path);
    }
    if (failures == 0) std::printf("ALL PASSED\n");
    return failures == 0 ? 0 : 1;
}
