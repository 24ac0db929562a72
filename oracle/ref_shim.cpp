// ref_shim.cpp -- C entry points over the reference's own host aggregation
// oracle (test/support/NativeAggregationOracle.cu) and Matrix Market reader
// (src/IO/MatrixMarket.cu), compiled from the reference sources where they
// lie by oracle/Makefile into oracle/_ref/libref_oracle.so.
//
// TEST INFRASTRUCTURE ONLY: it pins oracle/oracle.c and generates the golden
// fixtures under tests/golden/.  Nothing in the product links it.
#include <IO/MatrixMarket.cuh>
#include <support/NativeAggregationOracle.cuh>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <sstream>
#include <string>

namespace {
namespace to = thermofem::testoracle;
using thermofem::io::HostCsr;

struct RefCsr {
    int rows, cols;
    int64_t nnz;
    int *offsets;
    int *indices;
    double *values;
};

template <class V>
typename V::value_type *dup(const V &v) {
    auto *p = static_cast<typename V::value_type *>(std::malloc(sizeof(typename V::value_type) * (v.size() ? v.size() : 1)));
    if (!v.empty()) std::memcpy(p, v.data(), sizeof(typename V::value_type) * v.size());
    return p;
}

void put(const HostCsr &h, RefCsr *out) {
    out->rows = h.rows_;
    out->cols = h.columns_;
    out->nnz = static_cast<int64_t>(h.values_.size());
    out->offsets = dup(h.offsets_);
    out->indices = dup(h.indices_);
    out->values = dup(h.values_);
}

HostCsr get(int n, const int *rp, const int *ci, const double *v) {
    HostCsr h;
    h.rows_ = h.columns_ = n;
    h.offsets_.assign(rp, rp + n + 1);
    h.indices_.assign(ci, ci + rp[n]);
    h.values_.assign(v, v + rp[n]);
    return h;
}

thread_local std::string lastError;
}  // namespace

extern "C" {
const char *ref_last_error() { return lastError.c_str(); }

void ref_csr_free(RefCsr *a) {
    std::free(a->offsets);
    std::free(a->indices);
    std::free(a->values);
}

int ref_canonical(int n, const int *rp, const int *ci, const double *v, RefCsr *out) {
    try {
        put(to::canonicalMatrix(get(n, rp, ci, v)), out);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

int ref_strength(int n, const int *rp, const int *ci, const double *v, double theta, RefCsr *out) {
    try {
        put(to::strengthGraph(get(n, rp, ci, v), theta).edges_, out);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// Aggregates a strength graph: map[n], offsets[coarse+1], members[n], hist[4].
int ref_aggregate(int n, const int *rp, const int *ci, const double *v, int rounds, int absorb, int *map,
                  int *offsets, int *members, int *coarse, int64_t *hist) {
    try {
        to::StrengthGraph g{get(n, rp, ci, v)};
        auto t = to::aggregate(g, rounds, absorb != 0);
        std::memcpy(map, t.fineToCoarse_.data(), sizeof(int) * t.fineToCoarse_.size());
        std::memcpy(offsets, t.offsets_.data(), sizeof(int) * t.offsets_.size());
        std::memcpy(members, t.members_.data(), sizeof(int) * t.members_.size());
        *coarse = t.coarseRows();
        for (int k = 0; k < 4; ++k) hist[k] = static_cast<int64_t>(t.histogram_[k]);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

int ref_galerkin(int n, const int *rp, const int *ci, const double *v, const int *map, int coarse,
                 const int *offsets, const int *members, RefCsr *out) {
    try {
        to::AggregateMap t;
        t.fineToCoarse_.assign(map, map + n);
        t.offsets_.assign(offsets, offsets + coarse + 1);
        t.members_.assign(members, members + n);
        put(to::aggregateGalerkin(get(n, rp, ci, v), t), out);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// Parses Matrix Market text; returns 0, or -1 with ref_last_error() set.
int ref_read_matrix_market(const char *text, RefCsr *out) {
    try {
        std::istringstream in{std::string(text)};
        auto h = thermofem::io::readMatrixMarket(in);
        out->rows = h.rows_;
        out->cols = h.columns_;
        out->nnz = static_cast<int64_t>(h.values_.size());
        out->offsets = dup(h.offsets_);
        out->indices = dup(h.indices_);
        out->values = dup(h.values_);
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return -1;
    }
}

// std::mt19937 stream, to pin the oracle's own MT19937 used by sample(n).
void ref_std_mt19937(uint32_t seed, int count, uint32_t *out) {
    std::mt19937 g(seed);
    for (int i = 0; i < count; ++i) out[i] = static_cast<uint32_t>(g());
}
}
