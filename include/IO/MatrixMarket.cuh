// MatrixMarket.cuh -- Matrix Market coordinate reader (drop-in for
// include/IO/MatrixMarket.cuh:14-31 of Mgepahmge/ThermoFEM: HostCsr with the
// same fields, readMatrixMarket(std::istream&) with the same acceptance
// rules and std::runtime_error messages).  The stream is read in large
// blocks by the library's reader (tf_read_matrix_market_stream): real or
// integer, general or symmetric (one triangle, mirrored), duplicates kept,
// each row's entries in input order.  No CUDA needed.
#pragma once

#include <thermofem_b200.h>

#include <cstddef>
#include <istream>
#include <stdexcept>
#include <string>
#include <vector>

namespace thermofem::io {

struct HostCsr {
    int rows_{};
    int columns_{};
    std::vector<int> offsets_;
    std::vector<int> indices_;
    std::vector<double> values_;
};

namespace detail {
inline std::size_t readBlock(void *user, char *buffer, std::size_t capacity) {
    auto &in = *static_cast<std::istream *>(user);
    if (in.bad()) return static_cast<std::size_t>(-1);
    in.read(buffer, static_cast<std::streamsize>(capacity));
    if (in.bad()) return static_cast<std::size_t>(-1);
    return static_cast<std::size_t>(in.gcount());
}
}  // namespace detail

inline HostCsr readMatrixMarket(std::istream &input) {
    tf_host_csr raw{};
    const int status = tf_read_matrix_market_stream(detail::readBlock, &input, &raw);
    if (status != TF_OK) {
        const char *why = tf_last_error();
        throw std::runtime_error(why && *why ? why : "Matrix Market input read failure");
    }
    HostCsr out;
    out.rows_ = raw.rows;
    out.columns_ = raw.cols;
    out.offsets_.assign(raw.offsets, raw.offsets + raw.rows + 1);
    out.indices_.assign(raw.indices, raw.indices + raw.nnz);
    out.values_.assign(raw.values, raw.values + raw.nnz);
    tf_host_csr_free(&raw);
    return out;
}

}  // namespace thermofem::io
