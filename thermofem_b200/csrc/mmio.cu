// mmio.cu -- Matrix Market coordinate reader (host code), the input stage of
// the solve driver.  Accepts `matrix coordinate real|integer
// general|symmetric`, skips blank and '%' lines, expands a symmetric
// triangle (mixed triangles rejected), keeps duplicates and, within a row,
// the input order (a stable counting sort by row).  The acceptance rules and
// messages follow the reference reader (src/IO/MatrixMarket.cu:35-122) so a
// file accepted or rejected there is accepted or rejected here.
#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

using tfb::fail;

bool next_line(std::istream &in, std::string &line) {
    while (std::getline(in, line)) {
        const auto first = line.find_first_not_of(" \t\r");
        if (first != std::string::npos && line[first] != '%') return true;
    }
    return false;
}

void require_end(std::istringstream &row) {
    std::string extra;
    if (row >> extra) fail(TF_ERR_RUNTIME, "Unexpected Matrix Market field");
}

struct Entry {
    int row, col;
    double value;
};

void parse(std::istream &input, tf_host_csr *out) {
    std::string line, banner, object, format, field, symmetry;
    if (!std::getline(input, line)) fail(TF_ERR_RUNTIME, "Missing Matrix Market header");
    std::istringstream header(line);
    if (!(header >> banner >> object >> format >> field >> symmetry) || banner != "%%MatrixMarket" ||
        object != "matrix" || format != "coordinate" || (field != "real" && field != "integer") ||
        (symmetry != "general" && symmetry != "symmetric"))
        fail(TF_ERR_RUNTIME, "Unsupported Matrix Market header");
    require_end(header);
    if (!next_line(input, line)) fail(TF_ERR_RUNTIME, "Missing Matrix Market dimensions");
    long long rows = 0, cols = 0, count = 0;
    std::istringstream dims(line);
    constexpr long long limit = std::numeric_limits<int>::max();
    if (!(dims >> rows >> cols >> count) || rows < 0 || cols < 0 || count < 0 || rows > limit || cols > limit ||
        count > limit || (symmetry == "symmetric" && rows != cols))
        fail(TF_ERR_RUNTIME, "Invalid Matrix Market dimensions");
    require_end(dims);
    std::vector<Entry> entries;
    entries.reserve(static_cast<size_t>(count));
    int triangle = 0;
    for (long long k = 0; k < count; ++k) {
        if (!next_line(input, line)) fail(TF_ERR_RUNTIME, "Truncated Matrix Market entries");
        std::istringstream rec(line);
        long long r = 0, c = 0;
        double v = 0;
        if (!(rec >> r >> c >> v) || r < 1 || r > rows || c < 1 || c > cols || !std::isfinite(v) ||
            (field == "integer" && std::trunc(v) != v))
            fail(TF_ERR_RUNTIME, "Invalid Matrix Market entry");
        require_end(rec);
        const bool mirror = symmetry == "symmetric" && r != c;
        if (mirror) {
            const int side = r > c ? 1 : -1;
            if (triangle && triangle != side) fail(TF_ERR_RUNTIME, "Mixed triangles in symmetric storage");
            triangle = side;
        }
        const size_t added = mirror ? 2 : 1;
        if (entries.size() > static_cast<size_t>(limit) - added) fail(TF_ERR_RUNTIME, "Expanded CSR exceeds index range");
        entries.push_back({static_cast<int>(r - 1), static_cast<int>(c - 1), v});
        if (mirror) entries.push_back({static_cast<int>(c - 1), static_cast<int>(r - 1), v});
    }
    if (next_line(input, line)) fail(TF_ERR_RUNTIME, "Extra Matrix Market entries");
    if (input.bad()) fail(TF_ERR_RUNTIME, "Matrix Market input read failure");
    const size_t m = entries.size();
    out->rows = static_cast<int>(rows);
    out->cols = static_cast<int>(cols);
    out->nnz = static_cast<int64_t>(m);
    out->offsets = static_cast<int32_t *>(std::calloc(static_cast<size_t>(rows) + 1, sizeof(int32_t)));
    out->indices = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * (m ? m : 1)));
    out->values = static_cast<double *>(std::malloc(sizeof(double) * (m ? m : 1)));
    if (!out->offsets || !out->indices || !out->values) fail(TF_ERR_NOMEM, "host allocation failed");
    for (const auto &e : entries) ++out->offsets[e.row + 1];
    for (long long r = 0; r < rows; ++r) out->offsets[r + 1] += out->offsets[r];
    std::vector<int32_t> pos(out->offsets, out->offsets + rows);
    for (const auto &e : entries) {
        const int32_t p = pos[static_cast<size_t>(e.row)]++;
        out->indices[p] = e.col;
        out->values[p] = e.value;
    }
}

void reset(tf_host_csr *out) {
    out->rows = out->cols = 0;
    out->nnz = 0;
    out->offsets = nullptr;
    out->indices = nullptr;
    out->values = nullptr;
}

}  // namespace

extern "C" {

int tf_read_matrix_market(const char *text, size_t length, tf_host_csr *out) {
    return tfb::guard([&] {
        tfb::require(out != nullptr && (text != nullptr || length == 0), "null argument");
        reset(out);
        std::istringstream in(std::string(text ? text : "", length));
        try {
            parse(in, out);
        } catch (...) {
            tf_host_csr_free(out);
            throw;
        }
    });
}

int tf_read_matrix_market_file(const char *path, tf_host_csr *out) {
    return tfb::guard([&] {
        tfb::require(out != nullptr && path != nullptr, "null argument");
        reset(out);
        std::ifstream file(path);
        if (!file) fail(TF_ERR_RUNTIME, "Cannot open matrix file");
        try {
            parse(file, out);
        } catch (...) {
            tf_host_csr_free(out);
            throw;
        }
    });
}

void tf_host_csr_free(tf_host_csr *m) {
    if (!m) return;
    std::free(m->offsets);
    std::free(m->indices);
    std::free(m->values);
    reset(m);
}

}  // extern "C"
