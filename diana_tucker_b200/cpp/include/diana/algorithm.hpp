// Drop-in C++ host layer: the reference's HOOI entry points
// (include/algorithm.hpp:10-21) over libdt_cuda.so, same signatures and
// return tuple (G, U).
//
// HOOI_ALS draws its initial factors from the caller's current libc rand()
// sequence exactly as hooi_als.tpp:74-81 does (Util::randn per element of each
// I_n x R_n block, then reduced_QR) and runs max_iter sweeps of the ALS_
// subspace step (5 iterations) per mode.  Sp_HOOI_ALS draws R_n x I_n
// Gaussian blocks the same way, orthonormalises them (orth2), and runs
// max_iter sparse power sweeps (sp_hooi_als.tpp:67-118).
#pragma once

#include <tuple>
#include <vector>

#include "function.hpp"

namespace Algorithm {
namespace Tucker {

template <typename Ty>
std::tuple<Tensor<Ty>, std::vector<Tensor<Ty>>> HOOI_ALS(const Tensor<Ty> &A, const shape_t &R,
                                                         size_t max_iter);

template <>
inline std::tuple<Tensor<double>, std::vector<Tensor<double>>> HOOI_ALS(const Tensor<double> &A,
                                                                        const shape_t &R,
                                                                        size_t max_iter) {
    if (R.size() != A.ndim()) diana::fail("HOOI_ALS: one rank per mode expected");
    const size_t N = A.ndim();
    std::vector<int64_t> shape(A.shape().begin(), A.shape().end()), ranks(R.begin(), R.end());
    std::vector<Tensor<double>> U;
    std::vector<double *> Up;
    for (size_t n = 0; n < N; n++) {
        U.emplace_back(shape_t{A.shape()[n], R[n]}, false);
        Up.push_back(U.back().data());
    }
    Tensor<double> G(R, false);
    dt_hooi_opts o;
    dt_hooi_default_opts(&o);
    o.init = DT_INIT_RANDN_LIBC;
    o.seed = DT_SEED_KEEP;
    o.max_sweeps = (int)max_iter;
    o.inner_iters = 5;
    dt_hooi_report rep;
    diana::check(dt_hooi_dense(diana::ctx(), A.data(), DT_F64, (int)N, shape.data(), ranks.data(),
                               &o, G.data(), Up.data(), &rep),
                 "HOOI_ALS");
    return std::make_tuple(G, U);
}

}  // namespace Tucker

namespace SpTucker {

template <typename Ty>
std::tuple<Tensor<Ty>, std::vector<Tensor<Ty>>> Sp_HOOI_ALS(const SpTensor<Ty> &A,
                                                            const shape_t &R, size_t max_iter);

template <>
inline std::tuple<Tensor<double>, std::vector<Tensor<double>>> Sp_HOOI_ALS(
    const SpTensor<double> &A, const shape_t &R, size_t max_iter) {
    const size_t N = A.ndim();
    if (R.size() != N) diana::fail("Sp_HOOI_ALS: one rank per mode expected");
    std::vector<Tensor<double>> Ut;
    std::vector<double *> Up;
    for (size_t n = 0; n < N; n++) {
        Tensor<double> u(shape_t{R[n], A.shape()[n]}, false);
        u.randn();
        diana::check(dt_orth2_f64(diana::ctx(), u.data(), (int64_t)R[n], (int64_t)A.shape()[n]),
                     "orth2");
        Ut.push_back(u);
        Up.push_back(Ut.back().data());
    }
    std::vector<int64_t> ranks(R.begin(), R.end());
    size_t P = 1;
    for (size_t m = 0; m + 1 < N; m++) P *= R[m];
    Tensor<double> G({P, R[N - 1]}, true);
    dt_hooi_report rep;
    diana::check(dt_sp_hooi(diana::ctx(), A.handle(), ranks.data(), (int)max_iter, Up.data(),
                            G.data(), &rep),
                 "Sp_HOOI_ALS");
    return std::make_tuple(G, Ut);
}

}  // namespace SpTucker
}  // namespace Algorithm
