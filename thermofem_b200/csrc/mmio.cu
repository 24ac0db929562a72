// mmio.cu -- Matrix Market coordinate reader (host code), the input stage of
// the solve driver.
//
// What it accepts is the reference reader's contract
// (src/IO/MatrixMarket.cu:35-122): `%%MatrixMarket matrix coordinate
// real|integer general|symmetric`, blank and '%' lines skipped after the
// banner, a symmetric file gives one triangle (its mirror added right after
// each off-diagonal entry), duplicates kept, entries of a row in input order.
// Every rule of that contract, with the message it raises, is one row of the
// rules below, so a file accepted or rejected there is accepted or rejected
// here with the same message.
//
// How it reads is its own: input arrives in large blocks (a whole text buffer,
// a file read 16 MB at a time, or a caller's read callback), lines are cut
// out of the block without copying, and each field is scanned in place with
// the number grammar of the C++ stream extractors (so a field ends exactly
// where `stream >> value` would end it) and converted with std::from_chars.
// Entries land in three flat arrays and one stable counting sort by row
// builds the CSR.  No per-line string streams: the reference's reader spends
// most of its time constructing them.
#include <clocale>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <locale.h>
#include <string>
#include <string_view>
#include <vector>

#include "common.cuh"

namespace {

using tfb::fail;

// ---- the contract, one rule per row ---------------------------------------
enum Rule {
    kNoBanner,        // the input has no first line
    kBadBanner,       // the first line is not one of the accepted banners
    kBannerTail,      // the banner has a sixth field
    kNoSize,          // no size line after the banner
    kBadSize,         // size fields missing, negative, beyond INT_MAX, or a non-square symmetric matrix
    kSizeTail,        // the size line has a fourth field
    kShortEntries,    // fewer entry lines than the size line announces
    kBadEntry,        // an entry's row/column/value is missing or out of range, nonfinite, or non-integral in an integer file
    kEntryTail,       // an entry line has a fourth field
    kBothTriangles,   // a symmetric file gives entries above and below the diagonal
    kTooManyEntries,  // the expanded entry count exceeds INT_MAX
    kExtraEntries,    // a content line after the announced entries
    kReadError,       // the input could not be read
    kRuleCount
};

constexpr const char *kMessage[kRuleCount] = {
    "Missing Matrix Market header",
    "Unsupported Matrix Market header",
    "Unexpected Matrix Market field",
    "Missing Matrix Market dimensions",
    "Invalid Matrix Market dimensions",
    "Unexpected Matrix Market field",
    "Truncated Matrix Market entries",
    "Invalid Matrix Market entry",
    "Unexpected Matrix Market field",
    "Mixed triangles in symmetric storage",
    "Expanded CSR exceeds index range",
    "Extra Matrix Market entries",
    "Matrix Market input read failure",
};

[[noreturn]] void reject(Rule r) { fail(TF_ERR_RUNTIME, kMessage[r]); }

// The banner: five words, each from its own set of accepted spellings.  The
// index of the matching spelling at positions 3 and 4 gives the field
// (0 real, 1 integer) and the symmetry (0 general, 1 symmetric).
constexpr std::string_view kBannerWords[5][2] = {
    {"%%MatrixMarket", {}}, {"matrix", {}}, {"coordinate", {}}, {"real", "integer"}, {"general", "symmetric"}};

constexpr long long kIndexLimit = std::numeric_limits<int>::max();

// ---- lines -----------------------------------------------------------------
// Produces the input's lines, cut at '\n' (a final line without '\n' counts
// when it holds at least one character), as views into a block buffer that
// stay valid until the next call.
class Lines {
public:
    using ReadFn = size_t (*)(void *user, char *buf, size_t capacity);

    // A caller-owned text: lines are views straight into it.
    Lines(const char *text, size_t length) : fixed_(text), fixed_end_(text + length) {}
    // A block source: `read` fills up to `capacity` bytes and returns how many
    // (0 at the end, (size_t)-1 on a read error).
    Lines(ReadFn read, void *user) : read_(read), user_(user), buf_(kBlock) {}

    bool next(std::string_view &line) {
        if (!read_) {
            if (fixed_ == fixed_end_) return false;
            const char *nl = static_cast<const char *>(std::memchr(fixed_, '\n', fixed_end_ - fixed_));
            const char *stop = nl ? nl : fixed_end_;
            line = std::string_view(fixed_, stop - fixed_);
            fixed_ = nl ? nl + 1 : fixed_end_;
            return true;
        }
        for (;;) {
            const char *base = buf_.data();
            if (const void *nl = std::memchr(base + pos_, '\n', len_ - pos_)) {
                const size_t at = static_cast<const char *>(nl) - base;
                line = std::string_view(base + pos_, at - pos_);
                pos_ = at + 1;
                return true;
            }
            if (done_) {
                if (pos_ == len_) return false;
                line = std::string_view(base + pos_, len_ - pos_);
                pos_ = len_;
                return true;
            }
            refill();
        }
    }

    bool failed() const { return failed_; }

private:
    static constexpr size_t kBlock = size_t(16) << 20;

    // Moves the unfinished line to the front, grows the buffer if that line
    // fills it, and appends the next block.
    void refill() {
        const size_t keep = len_ - pos_;
        if (keep && pos_) std::memmove(buf_.data(), buf_.data() + pos_, keep);
        pos_ = 0;
        len_ = keep;
        if (buf_.size() - len_ < kBlock / 2) buf_.resize(buf_.size() * 2);
        const size_t got = read_(user_, buf_.data() + len_, buf_.size() - len_);
        if (got == static_cast<size_t>(-1)) {
            failed_ = true;
            done_ = true;
        } else if (got == 0) {
            done_ = true;
        } else {
            len_ += got;
        }
    }

    const char *fixed_ = nullptr, *fixed_end_ = nullptr;
    ReadFn read_ = nullptr;
    void *user_ = nullptr;
    std::vector<char> buf_;
    size_t pos_ = 0, len_ = 0;
    bool done_ = false, failed_ = false;
};

// A line that holds something other than ' ', '\t', '\r' and does not start
// (after those) with '%'.
bool is_content(std::string_view line) {
    for (char c : line) {
        if (c == ' ' || c == '\t' || c == '\r') continue;
        return c != '%';
    }
    return false;
}

bool next_content(Lines &in, std::string_view &line) {
    while (in.next(line))
        if (is_content(line)) return true;
    return false;
}

// ---- fields ----------------------------------------------------------------
// A cursor over one line.  Fields are separated by the C locale's white space;
// numbers follow the grammar of the stream extractors: an optional sign, then
// digits (integers) or digits, an optional '.' and digits, and an exponent
// that needs a digit before it (reals).
struct Cursor {
    const char *p, *e;

    static bool space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
    static bool digit(char c) { return c >= '0' && c <= '9'; }

    void skip() {
        while (p != e && space(*p)) ++p;
    }
    bool empty_after_space() {
        skip();
        return p == e;
    }
    bool word(std::string_view &w) {
        skip();
        const char *s = p;
        while (p != e && !space(*p)) ++p;
        w = std::string_view(s, p - s);
        return p != s;
    }
    bool integer(long long &v) {
        skip();
        bool negative = false;
        if (p != e && (*p == '+' || *p == '-')) negative = *p++ == '-';
        const char *d = p;
        while (p != e && digit(*p)) ++p;
        if (p == d) return false;
        // from_chars takes no '+'; the sign is applied by parsing "-digits"
        const auto r = negative ? std::from_chars(d - 1, p, v) : std::from_chars(d, p, v);
        return r.ec == std::errc() && r.ptr == p;
    }
    bool real(double &v) {
        skip();
        const char *s = p;
        if (p != e && (*p == '+' || *p == '-')) ++p;
        bool mantissa = false, point = false;
        for (; p != e; ++p) {
            if (digit(*p)) {
                mantissa = true;
            } else if (*p == '.' && !point) {
                point = true;
            } else {
                break;
            }
        }
        if (mantissa && p != e && (*p == 'e' || *p == 'E')) {
            ++p;
            if (p != e && (*p == '+' || *p == '-')) ++p;
            while (p != e && digit(*p)) ++p;
        }
        return convert(s, p, v);
    }

    // The whole of [s, t) must be one number, as strtod would read it; a value
    // too small for a double becomes its nearest double (0 or subnormal) as
    // the stream extractor gives it, a value too large is rejected.
    static bool convert(const char *s, const char *t, double &v) {
        if (s == t) return false;
        const char *b = *s == '+' ? s + 1 : s;
        if (b == t || *b == '+') return false;
        const auto r = std::from_chars(b, t, v);
        if (r.ptr != t) return false;
        if (r.ec == std::errc()) return true;
        if (r.ec != std::errc::result_out_of_range) return false;
        std::string copy(s, t);
        static locale_t c_locale = newlocale(LC_ALL_MASK, "C", nullptr);
        char *stop = nullptr;
        v = c_locale ? strtod_l(copy.c_str(), &stop, c_locale) : std::strtod(copy.c_str(), &stop);
        return stop == copy.c_str() + copy.size() && std::isfinite(v);
    }
};

// ---- the reader ------------------------------------------------------------
void parse(Lines &in, tf_host_csr *out) {
    std::string_view line;
    if (!in.next(line)) reject(in.failed() ? kReadError : kNoBanner);

    int choice[5] = {};
    {
        Cursor c{line.data(), line.data() + line.size()};
        for (int k = 0; k < 5; ++k) {
            std::string_view w;
            if (!c.word(w)) reject(kBadBanner);
            choice[k] = -1;
            for (int a = 0; a < 2; ++a)
                if (!kBannerWords[k][a].empty() && w == kBannerWords[k][a]) choice[k] = a;
            if (choice[k] < 0) reject(kBadBanner);
        }
        if (!c.empty_after_space()) reject(kBannerTail);
    }
    const bool integer_field = choice[3] == 1;
    const bool symmetric = choice[4] == 1;

    if (!next_content(in, line)) reject(in.failed() ? kReadError : kNoSize);
    long long rows = 0, cols = 0, count = 0;
    {
        Cursor c{line.data(), line.data() + line.size()};
        if (!c.integer(rows) || !c.integer(cols) || !c.integer(count)) reject(kBadSize);
        if (rows < 0 || cols < 0 || count < 0 || rows > kIndexLimit || cols > kIndexLimit || count > kIndexLimit ||
            (symmetric && rows != cols))
            reject(kBadSize);
        if (!c.empty_after_space()) reject(kSizeTail);
    }

    std::vector<int32_t> er, ec;
    std::vector<double> ev;
    const size_t hint = static_cast<size_t>(std::min<long long>(count, 1LL << 24)) * (symmetric ? 2 : 1);
    er.reserve(hint);
    ec.reserve(hint);
    ev.reserve(hint);
    int side = 0;  // symmetric: +1 lower triangle given, -1 upper
    for (long long k = 0; k < count; ++k) {
        if (!next_content(in, line)) reject(in.failed() ? kReadError : kShortEntries);
        Cursor c{line.data(), line.data() + line.size()};
        long long r = 0, col = 0;
        double v = 0;
        if (!c.integer(r) || !c.integer(col) || !c.real(v) || r < 1 || r > rows || col < 1 || col > cols ||
            !std::isfinite(v) || (integer_field && std::trunc(v) != v))
            reject(kBadEntry);
        if (!c.empty_after_space()) reject(kEntryTail);
        const bool mirror = symmetric && r != col;
        if (mirror) {
            const int s = r > col ? 1 : -1;
            if (side && side != s) reject(kBothTriangles);
            side = s;
        }
        if (static_cast<long long>(er.size()) + (mirror ? 2 : 1) > kIndexLimit) reject(kTooManyEntries);
        er.push_back(static_cast<int32_t>(r - 1));
        ec.push_back(static_cast<int32_t>(col - 1));
        ev.push_back(v);
        if (mirror) {
            er.push_back(static_cast<int32_t>(col - 1));
            ec.push_back(static_cast<int32_t>(r - 1));
            ev.push_back(v);
        }
    }
    if (next_content(in, line)) reject(kExtraEntries);
    if (in.failed()) reject(kReadError);

    // stable counting sort by row
    const size_t m = er.size();
    out->rows = static_cast<int>(rows);
    out->cols = static_cast<int>(cols);
    out->nnz = static_cast<int64_t>(m);
    out->offsets = static_cast<int32_t *>(std::calloc(static_cast<size_t>(rows) + 1, sizeof(int32_t)));
    out->indices = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * (m ? m : 1)));
    out->values = static_cast<double *>(std::malloc(sizeof(double) * (m ? m : 1)));
    if (!out->offsets || !out->indices || !out->values) fail(TF_ERR_NOMEM, "host allocation failed");
    int32_t *off = out->offsets;
    for (size_t j = 0; j < m; ++j) ++off[er[j] + 1];
    for (long long i = 0; i < rows; ++i) off[i + 1] += off[i];
    std::vector<int32_t> fill(off, off + rows);
    for (size_t j = 0; j < m; ++j) {
        const int32_t at = fill[er[j]]++;
        out->indices[at] = ec[j];
        out->values[at] = ev[j];
    }
}

void reset(tf_host_csr *out) {
    out->rows = out->cols = 0;
    out->nnz = 0;
    out->offsets = nullptr;
    out->indices = nullptr;
    out->values = nullptr;
}

template <class F>
int read_into(tf_host_csr *out, F &&make_lines) {
    return tfb::guard([&] {
        tfb::require(out != nullptr, "null argument");
        reset(out);
        try {
            make_lines([&](Lines &in) { parse(in, out); });
        } catch (...) {
            tf_host_csr_free(out);
            throw;
        }
    });
}

size_t read_file(void *user, char *buf, size_t capacity) {
    FILE *f = static_cast<FILE *>(user);
    const size_t got = std::fread(buf, 1, capacity, f);
    if (got == 0 && std::ferror(f)) return static_cast<size_t>(-1);
    return got;
}

}  // namespace

extern "C" {

int tf_read_matrix_market(const char *text, size_t length, tf_host_csr *out) {
    if (!text && length) return tfb::guard([] { tfb::require(false, "null argument"); });
    return read_into(out, [&](auto &&run) {
        Lines in(text ? text : "", text ? length : 0);
        run(in);
    });
}

int tf_read_matrix_market_file(const char *path, tf_host_csr *out) {
    if (!path) return tfb::guard([] { tfb::require(false, "null argument"); });
    return read_into(out, [&](auto &&run) {
        FILE *f = std::fopen(path, "rb");
        if (!f) fail(TF_ERR_RUNTIME, "Cannot open matrix file");
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{f};
        Lines in(read_file, f);
        run(in);
    });
}

int tf_read_matrix_market_stream(size_t (*read)(void *user, char *buf, size_t capacity), void *user,
                                 tf_host_csr *out) {
    if (!read) return tfb::guard([] { tfb::require(false, "null argument"); });
    return read_into(out, [&](auto &&run) {
        Lines in(read, user);
        run(in);
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
