// Drop-in C++ host layer: the reference's sparse types data_buffer<Ty>
// (include/read_data.hpp:9-17) and SpTensor<Ty> (include/sp_tensor.hpp:26-51)
// over libdt_cuda.so.
//
// SpTensor keeps the reference's ownership rule -- it takes the index and
// value arrays of the data_buffer (sp_tensor.hpp:189-193) and frees them --
// and builds the device-resident, per-mode sorted copies (the index_buffer
// CSR that sp_tensor.hpp:16-24 declares and ttmc_mTL reads) once.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <vector>

#include "tensor.hpp"

template <typename Ty>
class data_buffer {
   public:
    size_t **index_lists = nullptr;  // index_lists[m][e], 0-based
    size_t ndim = 0;
    size_t nnz = 0;
    Ty *vals = nullptr;
    size_t *dims = nullptr;
};

// read_data<double> (include/read_data.hpp:20-21, src/read_data.cpp:36-129):
// parses the .tns file on the device (dt_tns_read) and fills dbf with
// malloc'd arrays, 0-based size_t indices and dims = max index + 1, as the
// reference does; SpTensor takes them over.
template <typename Ty>
void read_data(char *filename, data_buffer<Ty> *dbf);

template <>
inline void read_data<double>(char *filename, data_buffer<double> *dbf) {
    dt_tns *t = nullptr;
    int nd = 0;
    int64_t nz = 0;
    diana::check(dt_tns_read(diana::ctx(), filename, &t, &nd, &nz), "read_data");
    dbf->ndim = (size_t)nd;
    dbf->nnz = (size_t)nz;
    dbf->dims = (size_t *)std::malloc(nd * sizeof(size_t));
    dbf->index_lists = (size_t **)std::malloc(nd * sizeof(size_t *));
    std::vector<int64_t *> idx(nd);
    for (int m = 0; m < nd; m++) {
        dbf->index_lists[m] = (size_t *)std::malloc(nz * sizeof(size_t));
        idx[m] = reinterpret_cast<int64_t *>(dbf->index_lists[m]);
    }
    dbf->vals = (double *)std::malloc(nz * sizeof(double));
    const int rc = dt_tns_copy(diana::ctx(), t, reinterpret_cast<int64_t *>(dbf->dims), idx.data(),
                               dbf->vals);
    dt_tns_destroy(t);
    diana::check(rc, "read_data");
}

template <typename Ty>
class SpTensor;

template <>
class SpTensor<double> {
   public:
    explicit SpTensor(data_buffer<double> *dbf) {
        ndim_ = dbf->ndim;
        nnz_ = dbf->nnz;
        for (size_t m = 0; m < ndim_; m++) dims_.push_back(dbf->dims[m]);
        index_lists_ = dbf->index_lists;
        vals_ = dbf->vals;
        std::vector<const int64_t *> idx(ndim_);
        std::vector<int64_t> shape(ndim_);
        for (size_t m = 0; m < ndim_; m++) {
            static_assert(sizeof(size_t) == sizeof(int64_t), "size_t indices are 64-bit");
            idx[m] = reinterpret_cast<const int64_t *>(index_lists_[m]);
            shape[m] = (int64_t)dims_[m];
        }
        diana::check(dt_sptensor_create(diana::ctx(), (int64_t)nnz_, (int)ndim_, idx.data(), vals_,
                                        shape.data(), &h_),
                     "SpTensor");
    }
    SpTensor(const SpTensor &) = delete;
    SpTensor &operator=(const SpTensor &) = delete;
    ~SpTensor() {
        if (h_) dt_sptensor_destroy(h_);
        for (size_t m = 0; m < ndim_; m++) std::free(index_lists_[m]);
        std::free(index_lists_);
        std::free(vals_);
    }
    size_t ndim() const { return ndim_; }
    size_t nnz() const { return nnz_; }
    const shape_t &shape() const { return dims_; }
    size_t **index_lists() const { return index_lists_; }
    const double *vals() const { return vals_; }
    dt_sptensor *handle() const { return h_; }

   private:
    size_t ndim_ = 0, nnz_ = 0;
    shape_t dims_;
    size_t **index_lists_ = nullptr;
    double *vals_ = nullptr;
    dt_sptensor *h_ = nullptr;
};
