// Drop-in C++ host layer: the reference's namespace Function
// (include/function.hpp:6-94) over libdt_cuda.so.  Same names, argument
// meaning and shape checks; failures end the process through diana::fail
// like the reference's error() / assert.
#pragma once

#include <tuple>
#include <vector>

#include "sp_tensor.hpp"
#include "tensor.hpp"

namespace Function {

namespace detail {
inline std::vector<int64_t> shape64(const shape_t &s) {
    return std::vector<int64_t>(s.begin(), s.end());
}
inline void require(bool c, const char *msg) {
    if (!c) diana::fail(msg);
}
}  // namespace detail

// A x_n M, M is J x I_n (template/function/tensor.tpp:272-335).
template <typename Ty>
Tensor<Ty> ttm(const Tensor<Ty> &A, const Tensor<Ty> &M, size_t n);
template <>
inline Tensor<double> ttm(const Tensor<double> &A, const Tensor<double> &M, size_t n) {
    detail::require(M.is_matrix() && n < A.ndim() && A.shape()[n] == M.shape()[1],
                    "Function::ttm: M must be J x I_n");
    shape_t out = A.shape();
    out[n] = M.shape()[0];
    Tensor<double> ret(A.distribution(), out, false);
    auto s = detail::shape64(A.shape());
    diana::check(dt_ttm_f64(diana::ctx(), A.data(), (int)A.ndim(), s.data(), (int)n, M.data(),
                            (int64_t)M.shape()[0], ret.data()),
                 "Function::ttm");
    return ret;
}

// A_(n) A_(n)^T (tensor.tpp:18-120).
template <typename Ty>
Tensor<Ty> gram(const Tensor<Ty> &A, size_t n);
template <>
inline Tensor<double> gram(const Tensor<double> &A, size_t n) {
    detail::require(n < A.ndim(), "Function::gram: mode out of range");
    const size_t I = A.shape()[n];
    Tensor<double> ret({I, I}, false);
    auto s = detail::shape64(A.shape());
    diana::check(dt_gram_f64(diana::ctx(), A.data(), (int)A.ndim(), s.data(), (int)n, ret.data()),
                 "Function::gram");
    return ret;
}

// A_(n) B_(n)^T (tensor.tpp:132-259).
template <typename Ty>
Tensor<Ty> ttt_except(const Tensor<Ty> &A, const Tensor<Ty> &B, size_t n);
template <>
inline Tensor<double> ttt_except(const Tensor<double> &A, const Tensor<double> &B, size_t n) {
    detail::require(A.ndim() == B.ndim() && n < A.ndim(), "Function::ttt_except: bad modes");
    Tensor<double> ret({A.shape()[n], B.shape()[n]}, false);
    auto sa = detail::shape64(A.shape()), sb = detail::shape64(B.shape());
    diana::check(dt_ttt_except_f64(diana::ctx(), A.data(), sa.data(), B.data(), sb.data(),
                                   (int)A.ndim(), (int)n, ret.data()),
                 "Function::ttt_except");
    return ret;
}

template <typename Ty>
double fnorm(const Tensor<Ty> &A) {
    return A.fnorm();
}

// Matrix functions (template/function/matrix.tpp:6-129).
inline Tensor<double> matmul_(int ta, int tb, const Tensor<double> &A, const Tensor<double> &B) {
    detail::require(A.is_matrix() && B.is_matrix(), "Function::matmul: matrices expected");
    const size_t m = ta ? A.shape()[1] : A.shape()[0];
    const size_t k = ta ? A.shape()[0] : A.shape()[1];
    const size_t kb = tb ? B.shape()[1] : B.shape()[0];
    const size_t n = tb ? B.shape()[0] : B.shape()[1];
    detail::require(k == kb, "Function::matmul: inner dimensions differ");
    Tensor<double> ret({m, n}, false);
    diana::check(dt_matmul_f64(diana::ctx(), ta, tb, (int64_t)m, (int64_t)n, (int64_t)k, A.data(),
                               B.data(), ret.data()),
                 "Function::matmul");
    return ret;
}
template <typename Ty>
Tensor<Ty> matmulNN(const Tensor<Ty> &A, const Tensor<Ty> &B) {
    return matmul_(0, 0, A, B);
}
template <typename Ty>
Tensor<Ty> matmulNT(const Tensor<Ty> &A, const Tensor<Ty> &B) {
    return matmul_(0, 1, A, B);
}
template <typename Ty>
Tensor<Ty> matmulTN(const Tensor<Ty> &A, const Tensor<Ty> &B) {
    return matmul_(1, 0, A, B);
}

template <typename Ty>
Tensor<Ty> inverse(const Tensor<Ty> &A) {
    detail::require(A.is_matrix() && A.shape()[0] == A.shape()[1], "Function::inverse: square");
    Tensor<Ty> ret(A.shape(), false);
    diana::check(dt_inverse_f64(diana::ctx(), A.data(), (int64_t)A.shape()[0], ret.data()),
                 "Function::inverse");
    return ret;
}

template <typename Ty>
std::tuple<Tensor<Ty>, Tensor<Ty>> reduced_QR(const Tensor<Ty> &A) {
    detail::require(A.is_matrix() && A.shape()[0] >= A.shape()[1], "Function::reduced_QR: m >= n");
    const size_t m = A.shape()[0], n = A.shape()[1];
    Tensor<Ty> Q({m, n}, true), R({n, n}, true);
    diana::check(dt_reduced_qr_f64(diana::ctx(), A.data(), (int64_t)m, (int64_t)n, Q.data(),
                                   R.data()),
                 "Function::reduced_QR");
    return std::make_tuple(Q, R);
}

template <typename Ty>
Tensor<Ty> transpose(const Tensor<Ty> &A) {
    detail::require(A.is_matrix(), "Function::transpose: matrix expected");
    const size_t m = A.shape()[0], n = A.shape()[1];
    Tensor<Ty> At({n, m}, false);
    for (size_t i = 0; i < m; i++)
        for (size_t j = 0; j < n; j++) At[j + i * n] = A[i + j * m];
    return At;
}

// Sparse TTMc contractions (template/function/sp_tensor.tpp:236-365).  Factors
// are transposed as in the reference: M[m] is R_m x I_m.
inline Tensor<double> ttmc_mTR(const SpTensor<double> &A, const std::vector<Tensor<double>> &M,
                               size_t n, const Tensor<double> &R) {
    detail::require(n < A.ndim() && A.shape()[n] == R.shape()[1], "Function::ttmc_mTR: shapes");
    std::vector<const double *> ut(A.ndim());
    std::vector<int64_t> rk(A.ndim());
    size_t P = 1;
    for (size_t m = 0; m < A.ndim(); m++) {
        ut[m] = M[m].data();
        rk[m] = (int64_t)M[m].shape()[0];
        if (m != n) P *= M[m].shape()[0];
    }
    Tensor<double> ret({P, R.shape()[0]}, true);
    diana::check(dt_sp_ttmc_mTR(diana::ctx(), A.handle(), ut.data(), rk.data(), (int)n, ret.data()),
                 "Function::ttmc_mTR");
    return ret;
}

inline void ttmc_mTL(const SpTensor<double> &A, const std::vector<Tensor<double>> &M, size_t n,
                     const Tensor<double> &L, Tensor<double> &ret) {
    detail::require(n < A.ndim() && L.shape()[1] == M[n].shape()[0], "Function::ttmc_mTL: shapes");
    std::vector<const double *> ut(A.ndim());
    std::vector<int64_t> rk(A.ndim());
    for (size_t m = 0; m < A.ndim(); m++) {
        ut[m] = M[m].data();
        rk[m] = (int64_t)M[m].shape()[0];
    }
    diana::check(dt_sp_ttmc_mTL(diana::ctx(), A.handle(), ut.data(), rk.data(), (int)n, L.data(),
                                ret.data()),
                 "Function::ttmc_mTL");
}

// Sparse TTMc to a dense tensor (template/function/sp_tensor.tpp:16-192):
// A x_{m in idx} M[m] with M[m] J_m x I_m; the other modes keep their extent.
// The result carries `distribution` (world size 1: the whole tensor);
// to_permu only chooses the reference's internal buffer order and does not
// change the result.
namespace detail {
inline Tensor<double> sp_dense_out(const SpTensor<double> &A, const std::vector<Tensor<double>> &M,
                                   const std::vector<size_t> &idx, Distribution *distribution,
                                   std::vector<const double *> &mp, std::vector<int64_t> &J,
                                   std::vector<int> &ids) {
    shape_t out = A.shape();
    mp.assign(A.ndim(), nullptr);
    J.assign(A.ndim(), 0);
    for (size_t m : idx) {
        require(m < A.ndim() && m < M.size() && M[m].is_matrix() &&
                    M[m].shape()[1] == A.shape()[m],
                "Function::ttmc: M[m] must be J x I_m for every listed mode");
        mp[m] = M[m].data();
        J[m] = (int64_t)M[m].shape()[0];
        out[m] = M[m].shape()[0];
        ids.push_back((int)m);
    }
    return Tensor<double>(distribution, out, false);
}
}  // namespace detail

inline Tensor<double> ttmc(const SpTensor<double> &A, const std::vector<Tensor<double>> &M,
                           const std::vector<size_t> &idx, Distribution *distribution,
                           bool to_permu) {
    (void)to_permu;
    std::vector<const double *> mp;
    std::vector<int64_t> J;
    std::vector<int> ids;
    Tensor<double> ret = detail::sp_dense_out(A, M, idx, distribution, mp, J, ids);
    diana::check(dt_sp_ttmc_dense_f64(diana::ctx(), A.handle(), mp.data(), J.data(), ids.data(),
                                      (int)ids.size(), ret.data()),
                 "Function::ttmc");
    return ret;
}

// mettmc (sp_tensor.tpp:194-211): the same result, the `level` modes of idx
// with the smallest I_m / J_m contracted by dense TTMs after the sparse TTMc.
inline Tensor<double> mettmc(const SpTensor<double> &A, const std::vector<Tensor<double>> &M,
                             const std::vector<size_t> &idx, Distribution *distribution,
                             bool to_permu, size_t level) {
    (void)to_permu;
    std::vector<const double *> mp;
    std::vector<int64_t> J;
    std::vector<int> ids;
    Tensor<double> ret = detail::sp_dense_out(A, M, idx, distribution, mp, J, ids);
    diana::check(dt_sp_mettmc_f64(diana::ctx(), A.handle(), mp.data(), J.data(), ids.data(),
                                  (int)ids.size(), (int)level, ret.data()),
                 "Function::mettmc");
    return ret;
}

inline double fnorm(const SpTensor<double> &A) {
    double out = 0.0;
    diana::check(dt_sp_fnorm(diana::ctx(), A.handle(), &out), "Function::fnorm");
    return out;
}

}  // namespace Function
