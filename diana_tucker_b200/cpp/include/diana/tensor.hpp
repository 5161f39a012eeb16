// Drop-in C++ host layer: the reference's dense Tensor<Ty>
// (include/tensor.hpp:44-182, template/tensor_mpi.tpp) over libdt_cuda.so.
//
// Kept from the reference: column-major storage with stride[0] = 1
// (tensor_mpi.tpp:49-53), shallow copies that share the buffer
// (tensor_mpi.tpp:230-268; here a shared_ptr instead of the global refcount
// map), copy() as the deep copy (:531-542), the constructor set, operator[],
// randn() drawing Util::randn on libc rand() (src/util.cpp:10-18).
// The distribution collapses to one device: every Tensor is the global
// tensor; Distribution arguments are accepted and recorded.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dt_cuda.h"

typedef std::vector<size_t> shape_t;
#ifndef DIANA_CEILDIV
#define DIANA_CEILDIV(n, k) (((n) + (k)-1) / (k))
#endif

namespace diana {

// The reference reports failures with error() -> exit(-3) (logger.hpp:75-84).
// The drop-in does the same by default; define DIANA_DROPIN_THROW to get a
// std::runtime_error instead.
[[noreturn]] inline void fail(const std::string &msg) {
#ifdef DIANA_DROPIN_THROW
    throw std::runtime_error(msg);
#else
    std::fprintf(stderr, "[ERROR] %s\n", msg.c_str());
    std::exit(-3);
#endif
}

inline void check(int code, const char *what) {
    if (code != DT_OK) fail(std::string(what) + ": " + dt_last_error());
}

// One process-wide context on device 0 (the world of size 1).
inline dt_ctx *ctx() {
    static dt_ctx *c = [] {
        dt_ctx *h = nullptr;
        check(dt_ctx_create(0, &h), "dt_ctx_create");
        return h;
    }();
    return c;
}

inline double randn() {  // Util::randn, src/util.cpp:10-18
    for (;;) {
        const double u = ((double)std::rand() / (RAND_MAX)) * 2 - 1;
        const double v = ((double)std::rand() / (RAND_MAX)) * 2 - 1;
        const double r = u * u + v * v;
        if (r == 0 || r > 1) continue;
        return u * std::sqrt(-2 * std::log(r) / r);
    }
}

inline size_t calc_size(const shape_t &s) {
    size_t n = 1;
    for (auto d : s) n *= d;
    return n;
}

}  // namespace diana

// Distribution types of the reference (include/distribution.hpp:14-90); at
// world size 1 every distribution describes the whole tensor on this rank.
class Distribution {
   public:
    enum Type : int { kLocal, kGlobal, kCartesianBlock };
    explicit Distribution(Type t) : type_(t) {}
    virtual ~Distribution() = default;
    Type type() const { return type_; }

   private:
    Type type_;
};
class DistributionLocal : public Distribution {
   public:
    DistributionLocal() : Distribution(kLocal) {}
};
class DistributionGlobal : public Distribution {
   public:
    DistributionGlobal() : Distribution(kGlobal) {}
};
class DistributionCartesianBlock : public Distribution {
   public:
    DistributionCartesianBlock(shape_t partition, int rank)
        : Distribution(kCartesianBlock), partition_(std::move(partition)) {
        for (auto p : partition_)
            if (p != 1) diana::fail("DistributionCartesianBlock: this build runs one rank; use a partition of all 1");
        (void)rank;
    }
    shape_t partition() const { return partition_; }

   private:
    shape_t partition_;
};

inline void mpi_init() {}
inline int mpi_rank() { return 0; }
inline int mpi_size() { return 1; }

template <typename Ty>
class Tensor {
   public:
    Tensor() = default;
    Tensor(Ty *A, const shape_t &shape) : shape_(shape) {  // external buffer, not owned
        data_ = std::shared_ptr<Ty>(A, [](Ty *) {});
        init_strides();
    }
    explicit Tensor(const shape_t &shape, bool zero = true) : shape_(shape) { alloc(zero); }
    Tensor(Distribution *d, Ty *A, const shape_t &shape) : Tensor(A, shape) { dist_ = d; }
    Tensor(Distribution *d, const shape_t &shape, bool zero = true) : shape_(shape), dist_(d) {
        alloc(zero);
    }

    Ty *data() const { return data_.get(); }
    size_t ndim() const { return shape_.size(); }
    size_t size() const { return diana::calc_size(shape_); }
    const shape_t &shape() const { return shape_; }
    const shape_t &shape_global() const { return shape_; }
    size_t size_global() const { return size(); }
    const shape_t &stride() const { return stride_; }
    bool is_matrix() const { return shape_.size() == 2; }
    Distribution *distribution() const { return dist_; }
    int comm_size() const { return 1; }
    int comm_rank() const { return 0; }

    Ty &operator[](size_t i) { return data_.get()[i]; }
    const Ty &operator[](size_t i) const { return data_.get()[i]; }

    void constant(Ty c) {
        for (size_t i = 0; i < size(); i++) data()[i] = c;
    }
    void zeros() { constant(0); }
    void ones() { constant(1); }
    void randn() {
        for (size_t i = 0; i < size(); i++) data()[i] = (Ty)diana::randn();
    }
    void sync(int) {}  // world of size 1: nothing to broadcast
    double fnorm() const;

    Tensor<Ty> copy() const {
        Tensor<Ty> t(shape_, false);
        t.dist_ = dist_;
        std::memcpy(t.data(), data(), size() * sizeof(Ty));
        return t;
    }

   private:
    void init_strides() {
        stride_.assign(shape_.size(), 1);
        for (size_t i = 1; i < shape_.size(); i++) stride_[i] = stride_[i - 1] * shape_[i - 1];
    }
    void alloc(bool zero) {
        init_strides();
        const size_t n = std::max<size_t>(1, size());
        Ty *p = static_cast<Ty *>(std::malloc(n * sizeof(Ty)));
        if (!p) diana::fail("Tensor: host allocation failed");
        if (zero) std::memset(p, 0, n * sizeof(Ty));
        data_ = std::shared_ptr<Ty>(p, [](Ty *q) { std::free(q); });
    }

    shape_t shape_, stride_;
    std::shared_ptr<Ty> data_;
    Distribution *dist_ = nullptr;
};

template <>
inline double Tensor<double>::fnorm() const {
    double out = 0.0;
    diana::check(dt_fnorm_f64(diana::ctx(), data(), (int64_t)size(), &out), "fnorm");
    return out;
}
