// MatrixMarket text and binary I/O of matrix data (host code, no CUDA).
//
// Follows core/base/mtx_io.cpp of the reference:
//   - text reading (mtx_io::read, :73-81): the header line is the first
//     non-empty line, lower-cased and matched against
//     "%%matrixmarket matrix <layout> <field> <modifier>" as a prefix
//     (:612-650); the dimension line is the first following line that does
//     not start with '%' (:652-659); entries are read with the number rules
//     of a C++ input stream and the rest of each entry's line is discarded
//     (coordinate :400-440, array :462-492); symmetric, skew-symmetric and
//     hermitian storage add the mirrored entry (:305-381); the result is
//     sorted by (row, column) (:79);
//   - text writing (:980-1004 with :442-460 and :494-525): values in the
//     default stream format, six significant digits;
//   - the binary format (:760-978).
// The parser is a cursor over the whole buffer instead of an istream: one
// pass, no per-token allocation.
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <exception>
#include <new>
#include <numeric>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/ginkgo_b200.h"

namespace b2s {
void set_error(const char* fmt, ...);
}

namespace {

struct MtxData {
    int value_type = B2S_MTX_F64;
    int index_type = B2S_MTX_I32;
    int64_t rows = 0;
    int64_t cols = 0;
    std::vector<int64_t> r;  // entries, already converted to the index type
    std::vector<int64_t> c;
    std::vector<double> v;   // entries, already rounded to the value type
    std::string bytes;       // formatted output of a write
};

// A failure with the reference's StreamError message.
struct MtxError {
    std::string msg;
};

[[noreturn]] void fail(const std::string& msg) { throw MtxError{msg}; }

double round_to(int value_type, double x)
{
    return value_type == B2S_MTX_F32 ? double(float(x)) : x;
}

inline bool is_digit(char ch) { return ch >= '0' && ch <= '9'; }

// A signed decimal integer at p (no leading whitespace) within [lo, hi];
// all its digits are consumed even when it overflows.
bool scan_int(const char*& p, const char* end, int64_t lo, int64_t hi, int64_t& out)
{
    const char* q = p;
    bool neg = false;
    if (q < end && (*q == '+' || *q == '-')) neg = *q++ == '-';
    if (q >= end || !is_digit(*q)) return false;
    // magnitude up to 2^63 (the most negative int64)
    const uint64_t lim = uint64_t(std::numeric_limits<int64_t>::max()) + (neg ? 1 : 0);
    uint64_t mag = 0;
    bool over = false;
    for (; q < end && is_digit(*q); ++q) {
        const unsigned d = unsigned(*q - '0');
        if (mag > (lim - d) / 10) over = true;
        else mag = mag * 10 + d;
    }
    p = q;
    if (over) return false;
    const int64_t val = neg ? (mag == (uint64_t(1) << 63) ? std::numeric_limits<int64_t>::min()
                                                        : -int64_t(mag))
                            : int64_t(mag);
    if (val < lo || val > hi) return false;
    out = val;
    return true;
}

// A double at p (no leading whitespace) with the stream's grammar:
// [sign] digits [. digits] [(e|E) [sign] digits], at least one mantissa
// digit.  An exponent marker without digits fails, and so does a value that
// overflows to infinity (the stream's conversion sets failbit for both,
// LWG 23); an underflow gives the correctly rounded tiny value or zero.
bool scan_double(const char*& p, const char* end, double& out)
{
    const char* s = p;
    const char* q = p;
    bool plus = false;
    if (q < end && (*q == '+' || *q == '-')) plus = *q++ == '+';
    bool digits = false;
    while (q < end && is_digit(*q)) ++q, digits = true;
    if (q < end && *q == '.') {
        ++q;
        while (q < end && is_digit(*q)) ++q, digits = true;
    }
    if (!digits) {
        p = q;
        return false;
    }
    if (q < end && (*q == 'e' || *q == 'E')) {
        const char* e = q + 1;
        if (e < end && (*e == '+' || *e == '-')) ++e;
        if (e >= end || !is_digit(*e)) {
            p = e;
            return false;
        }
        while (e < end && is_digit(*e)) ++e;
        q = e;
    }
    p = q;
    // from_chars takes no leading '+'; it is correctly rounded, as strtod
    const char* f = plus ? s + 1 : s;
    const auto r = std::from_chars(f, q, out);
    if (r.ec == std::errc()) return true;
    const std::string t(f, q);
    const double x = std::strtod(t.c_str(), nullptr);
    if (std::isinf(x)) return false;
    out = x;
    return true;
}

// Cursor over the input with the extraction rules of a C++ stream in the
// classic locale: leading whitespace is skipped, a number is the longest
// prefix that fits its grammar.
struct Cursor {
    const char* p;
    const char* end;

    static bool space(char ch)
    {
        return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\v' || ch == '\f' ||
               ch == '\r';
    }
    void skip_ws()
    {
        while (p < end && space(*p)) ++p;
    }
    bool at_end() const { return p >= end; }
    // istream::ignore(max, '\n')
    void skip_line()
    {
        const void* nl = std::memchr(p, '\n', size_t(end - p));
        p = nl ? static_cast<const char*>(nl) + 1 : end;
    }
    // std::getline: false only when nothing is left to read
    bool get_line(std::string& out)
    {
        if (p >= end) return false;
        const void* nl = std::memchr(p, '\n', size_t(end - p));
        const char* e = nl ? static_cast<const char*>(nl) : end;
        out.assign(p, e);
        p = nl ? e + 1 : end;
        return true;
    }
    // signed decimal integer within [lo, hi]
    bool read_int(int64_t lo, int64_t hi, int64_t& out)
    {
        skip_ws();
        return scan_int(p, end, lo, hi, out);
    }
    // unsigned decimal size (a leading '-' is rejected)
    bool read_size(int64_t& out)
    {
        skip_ws();
        if (p < end && *p == '-') return false;
        return read_int(0, std::numeric_limits<int64_t>::max(), out);
    }
    bool read_double(double& out)
    {
        skip_ws();
        return scan_double(p, end, out);
    }
};

enum class Layout { coordinate, array };
enum class Field { real, integer, complex, pattern };
enum class Modifier { general, symmetric, skew_symmetric, hermitian };

// prefix match of one of the words at *pos, in the reference's order
template <typename E, size_t N>
bool match_word(const std::string& line, size_t& pos, const char* const (&words)[N],
                const E (&vals)[N], E& out)
{
    for (size_t i = 0; i < N; ++i) {
        const size_t len = std::strlen(words[i]);
        if (line.compare(pos, len, words[i]) == 0) {
            out = vals[i];
            pos += len;
            return true;
        }
    }
    return false;
}

void parse_header(const std::string& raw, Layout& layout, Field& field, Modifier& modifier)
{
    std::string line = raw;
    for (auto& ch : line) ch = char(std::tolower(static_cast<unsigned char>(ch)));
    static const char* const kLayouts[] = {"coordinate", "array"};
    static const Layout kLayoutVals[] = {Layout::coordinate, Layout::array};
    static const char* const kFields[] = {"real", "integer", "complex", "pattern"};
    static const Field kFieldVals[] = {Field::real, Field::integer, Field::complex,
                                       Field::pattern};
    static const char* const kMods[] = {"general", "symmetric", "skew-symmetric",
                                        "hermitian"};
    static const Modifier kModVals[] = {Modifier::general, Modifier::symmetric,
                                        Modifier::skew_symmetric, Modifier::hermitian};
    const std::string lead = "%%matrixmarket matrix ";
    size_t pos = 0;
    bool ok = line.compare(0, lead.size(), lead) == 0;
    pos = lead.size();
    ok = ok && match_word(line, pos, kLayouts, kLayoutVals, layout);
    ok = ok && line.compare(pos, 1, " ") == 0 && (++pos, true);
    ok = ok && match_word(line, pos, kFields, kFieldVals, field);
    ok = ok && line.compare(pos, 1, " ") == 0 && (++pos, true);
    ok = ok && match_word(line, pos, kMods, kModVals, modifier);
    if (!ok) {
        fail("error parsing the header line, the header format should have the "
             "following structure:\n    %%MatrixMarket matrix <LAYOUT-TYPE> "
             "<VALUE-TYPE> <LAYOUT-MODIFIER>\nwhere:\n    <LAYOUT-TYPE>     is one "
             "of: coordinate, array\n    <VALUE-TYPE>      is one of: real, integer, "
             "complex, pattern\n    <LAYOUT-MODIFIER> is one of: general, symmetric, "
             "skew-symmetric, hermitian\nFound the following header instead: " +
             line);
    }
}

struct Reader {
    MtxData& d;
    Field field;
    Modifier modifier;
    int64_t ilo, ihi;  // index type range

    double entry(Cursor& cur, const char* what)
    {
        if (field == Field::complex) {
            fail("trying to read a complex matrix into a real storage type");
        }
        if (field == Field::pattern) return 1.0;
        double x;
        if (!cur.read_double(x)) fail(what);
        return round_to(d.value_type, x);
    }
    void insert(int64_t row, int64_t col, double val)
    {
        d.r.push_back(row);
        d.c.push_back(col);
        d.v.push_back(val);
        if (row == col || modifier == Modifier::general) return;
        d.r.push_back(col);
        d.c.push_back(row);
        d.v.push_back(modifier == Modifier::skew_symmetric ? -val : val);
    }
    int64_t row_start(int64_t col) const
    {
        switch (modifier) {
        case Modifier::general: return 0;
        case Modifier::skew_symmetric: return col + 1;
        default: return col;
        }
    }
};

// Threads for a host pass over `bytes` bytes: at most the hardware threads
// (64 at most), at least 4 MiB each.
unsigned io_threads(size_t bytes)
{
    unsigned hw = std::thread::hardware_concurrency();
    hw = hw == 0 ? 1 : std::min(hw, 64u);
    return std::max(1u, std::min<unsigned>(hw, unsigned(std::min<size_t>(bytes >> 22, 64))));
}

// Runs f(0) .. f(T - 1), on T threads when T > 1; parts whose thread
// cannot be started run on the calling thread.
template <typename F>
void parallel_for(unsigned T, F&& f)
{
    std::vector<std::thread> pool;
    pool.reserve(T);
    unsigned t = 1;
    try {
        for (; t < T; ++t) pool.emplace_back(f, t);
    } catch (const std::system_error&) {
        for (; t < T; ++t) f(t);
    }
    f(0u);
    for (auto& th : pool) th.join();
}

// Stable sort of entries [b, e) of one row by column: insertion sort for
// short rows, a stable sort of an index range for long ones.
void sort_row_by_column(std::vector<int64_t>& c, std::vector<double>& v, size_t b, size_t e)
{
    if (e - b < 2) return;
    if (e - b <= 64) {
        for (size_t i = b + 1; i < e; ++i) {
            const int64_t ci = c[i];
            const double vi = v[i];
            size_t j = i;
            while (j > b && c[j - 1] > ci) {
                c[j] = c[j - 1];
                v[j] = v[j - 1];
                --j;
            }
            c[j] = ci;
            v[j] = vi;
        }
        return;
    }
    std::vector<size_t> perm(e - b);
    std::iota(perm.begin(), perm.end(), b);
    std::stable_sort(perm.begin(), perm.end(), [&](size_t x, size_t y) { return c[x] < c[y]; });
    std::vector<int64_t> cc(e - b);
    std::vector<double> vv(e - b);
    for (size_t k = 0; k < perm.size(); ++k) {
        cc[k] = c[perm[k]];
        vv[k] = v[perm[k]];
    }
    std::copy(cc.begin(), cc.end(), c.begin() + b);
    std::copy(vv.begin(), vv.end(), v.begin() + b);
}

// matrix_data::sort_row_major with equal coordinates kept in input order:
// a counting sort by row (rows inside [0, rows) and not far more rows than
// entries), then each row by column; otherwise a comparison sort.
void sort_row_major(MtxData& d)
{
    const size_t n = d.r.size();
    bool sorted = true;
    for (size_t i = 1; i < n && sorted; ++i) {
        sorted = d.r[i - 1] < d.r[i] || (d.r[i - 1] == d.r[i] && d.c[i - 1] <= d.c[i]);
    }
    if (sorted) return;
    bool counting = d.rows <= int64_t(4 * n + 1024);
    for (size_t i = 0; i < n && counting; ++i) counting = d.r[i] >= 0 && d.r[i] < d.rows;
    std::vector<int64_t> r(n), c(n);
    std::vector<double> v(n);
    if (counting) {
        // two stable passes on T threads: entries into B buckets of
        // consecutive rows (each thread's range in order), then a counting
        // sort by row inside each bucket and a column sort of every row
        const unsigned T = io_threads(n * 24);
        const uint64_t R = uint64_t(d.rows);
        const uint64_t B = std::min<uint64_t>(4096, R);
        auto bucket = [&](int64_t row) { return size_t(uint64_t(row) * B / R); };
        std::vector<size_t> off(size_t(T) * B, 0);
        parallel_for(T, [&](unsigned t) {
            size_t* cnt = &off[size_t(t) * B];
            for (size_t i = n * t / T; i < n * (t + 1) / T; ++i) ++cnt[bucket(d.r[i])];
        });
        std::vector<size_t> bstart(B + 1, 0);
        size_t run = 0;
        for (size_t b = 0; b < B; ++b) {
            bstart[b] = run;
            for (unsigned t = 0; t < T; ++t) {
                const size_t k = off[size_t(t) * B + b];
                off[size_t(t) * B + b] = run;
                run += k;
            }
        }
        bstart[B] = run;
        std::vector<int64_t> tr(n), tc(n);
        std::vector<double> tv(n);
        parallel_for(T, [&](unsigned t) {
            size_t* pos = &off[size_t(t) * B];
            for (size_t i = n * t / T; i < n * (t + 1) / T; ++i) {
                const size_t k = pos[bucket(d.r[i])]++;
                tr[k] = d.r[i];
                tc[k] = d.c[i];
                tv[k] = d.v[i];
            }
        });
        parallel_for(T, [&](unsigned t) {
            std::vector<size_t> start;
            for (size_t b = B * t / T; b < B * (t + 1) / T; ++b) {
                // rows of bucket b: [ceil(b R / B), ceil((b + 1) R / B))
                const int64_t lo = int64_t((b * R + B - 1) / B);
                const int64_t hi = int64_t(((b + 1) * R + B - 1) / B);
                start.assign(size_t(hi - lo) + 1, 0);
                for (size_t i = bstart[b]; i < bstart[b + 1]; ++i) ++start[size_t(tr[i] - lo) + 1];
                for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
                for (size_t i = bstart[b]; i < bstart[b + 1]; ++i) {
                    const size_t k = bstart[b] + start[size_t(tr[i] - lo)]++;
                    r[k] = tr[i];
                    c[k] = tc[i];
                    v[k] = tv[i];
                }
                // each row by column, stable (start[] now holds row ends)
                size_t rb = bstart[b];
                for (int64_t row = lo; row < hi; ++row) {
                    const size_t re = bstart[b] + start[size_t(row - lo)];
                    sort_row_by_column(c, v, rb, re);
                    rb = re;
                }
            }
        });
    } else {
        std::vector<size_t> perm(n);
        std::iota(perm.begin(), perm.end(), size_t(0));
        std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) {
            return d.r[a] < d.r[b] || (d.r[a] == d.r[b] && d.c[a] < d.c[b]);
        });
        for (size_t i = 0; i < n; ++i) {
            r[i] = d.r[perm[i]];
            c[i] = d.c[perm[i]];
            v[i] = d.v[perm[i]];
        }
    }
    d.r.swap(r);
    d.c.swap(c);
    d.v.swap(v);
}

inline bool line_space(char ch)
{
    return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\v' || ch == '\f';
}

// Coordinate entries of a large file, speculatively in parallel: the text
// after the dimension line is cut at line starts, every chunk counts its
// non-blank lines, then parses them as one entry per line ("row col
// [value] [anything]").  Valid only when each of the first nnz entries sits
// on its own line; otherwise (a token on the next line, a malformed or
// missing entry) it returns false and the serial reader, which follows the
// stream's rules exactly, runs instead.  Blank lines are skipped by both.
bool read_coordinate_parallel(const char* p, const char* end, int64_t nnz, const Reader& rd,
                              MtxData& d)
{
    const size_t bytes = size_t(end - p);
    const unsigned T = io_threads(bytes);
    if (T < 2 || nnz < (int64_t(1) << 16)) return false;
    std::vector<const char*> cut(T + 1);
    cut[0] = p;
    cut[T] = end;
    for (unsigned t = 1; t < T; ++t) {
        const char* q = std::max(p + bytes * t / T, cut[t - 1]);
        const void* nl = q < end ? std::memchr(q, '\n', size_t(end - q)) : nullptr;
        cut[t] = nl ? static_cast<const char*>(nl) + 1 : end;
    }
    std::vector<int64_t> count(T, 0);
    parallel_for(T, [&](unsigned t) {
        int64_t k = 0;
        bool blank = true;
        for (const char* q = cut[t]; q < cut[t + 1]; ++q) {
            if (*q == '\n') {
                k += !blank;
                blank = true;
            } else if (!line_space(*q)) {
                blank = false;
            }
        }
        count[t] = k + !blank;
    });
    std::vector<int64_t> first(T + 1, 0);
    for (unsigned t = 0; t < T; ++t) first[t + 1] = first[t] + count[t];
    if (first[T] < nnz) return false;
    struct Part {
        std::vector<int64_t> r, c;
        std::vector<double> v;
        bool ok = true;
    };
    std::vector<Part> part(T);
    const bool pattern = rd.field == Field::pattern;
    const bool general = rd.modifier == Modifier::general;
    const bool skew = rd.modifier == Modifier::skew_symmetric;
    parallel_for(T, [&](unsigned t) {
        int64_t idx = first[t];
        if (idx >= nnz) return;
        Part& o = part[t];
        const size_t want = size_t(std::min(nnz, first[t + 1]) - idx) * (general ? 1 : 2);
        o.r.reserve(want);
        o.c.reserve(want);
        o.v.reserve(want);
        const char* q = cut[t];
        const char* e = cut[t + 1];
        while (q < e && idx < nnz) {
            const void* nl = std::memchr(q, '\n', size_t(e - q));
            const char* le = nl ? static_cast<const char*>(nl) : e;
            const char* x = q;
            q = nl ? le + 1 : e;
            while (x < le && line_space(*x)) ++x;
            if (x == le) continue;
            int64_t row, col;
            if (!scan_int(x, le, rd.ilo, rd.ihi, row)) return void(o.ok = false);
            while (x < le && line_space(*x)) ++x;
            if (!scan_int(x, le, rd.ilo, rd.ihi, col)) return void(o.ok = false);
            double val = 1.0;
            if (!pattern) {
                while (x < le && line_space(*x)) ++x;
                if (!scan_double(x, le, val)) return void(o.ok = false);
                val = round_to(rd.d.value_type, val);
            }
            --row;
            --col;
            o.r.push_back(row);
            o.c.push_back(col);
            o.v.push_back(val);
            if (!general && row != col) {
                o.r.push_back(col);
                o.c.push_back(row);
                o.v.push_back(skew ? -val : val);
            }
            ++idx;
        }
    });
    for (const auto& o : part) {
        if (!o.ok) return false;
    }
    std::vector<size_t> off(T + 1, 0);
    for (unsigned t = 0; t < T; ++t) off[t + 1] = off[t] + part[t].r.size();
    d.r.resize(off[T]);
    d.c.resize(off[T]);
    d.v.resize(off[T]);
    parallel_for(T, [&](unsigned t) {
        std::copy(part[t].r.begin(), part[t].r.end(), d.r.begin() + off[t]);
        std::copy(part[t].c.begin(), part[t].c.end(), d.c.begin() + off[t]);
        std::copy(part[t].v.begin(), part[t].v.end(), d.v.begin() + off[t]);
    });
    return true;
}

void read_text(const char* buf, int64_t len, MtxData& d)
{
    Cursor cur{buf, buf + len};
    std::string line;
    do {
        if (!cur.get_line(line)) fail("error when reading the header line");
    } while (line.empty());
    Layout layout;
    Field field;
    Modifier modifier;
    parse_header(line, layout, field, modifier);
    std::string dims;
    do {
        if (!cur.get_line(dims)) fail("error when reading the dimensions line");
    } while (!dims.empty() && dims[0] == '%');
    Cursor dc{dims.data(), dims.data() + dims.size()};
    Reader rd{d, field, modifier, 0, 0};
    if (d.index_type == B2S_MTX_I32) {
        rd.ilo = std::numeric_limits<int32_t>::min();
        rd.ihi = std::numeric_limits<int32_t>::max();
    } else {
        rd.ilo = std::numeric_limits<int64_t>::min();
        rd.ihi = std::numeric_limits<int64_t>::max();
    }
    if (layout == Layout::coordinate) {
        int64_t nnz;
        if (!dc.read_size(d.rows) || !dc.read_size(d.cols) || !dc.read_size(nnz)) {
            fail("error when determining matrix size, expected: rows cols nnz");
        }
        if (field != Field::complex &&
            read_coordinate_parallel(cur.p, cur.end, nnz, rd, d)) {
            sort_row_major(d);
            return;
        }
        // reserve no more than the text can hold (two bytes per entry at least)
        const int64_t mult = modifier == Modifier::general ? 1 : 2;
        const int64_t cap = std::min<int64_t>(nnz, len / 2 + 1) * mult;
        d.r.reserve(size_t(cap));
        d.c.reserve(size_t(cap));
        d.v.reserve(size_t(cap));
        for (int64_t i = 0; i < nnz; ++i) {
            int64_t row, col;
            if (!cur.read_int(rd.ilo, rd.ihi, row) || !cur.read_int(rd.ilo, rd.ihi, col)) {
                fail("error when reading coordinates of matrix entry " + std::to_string(i));
            }
            const double val = rd.entry(cur, "error while reading matrix entry");
            rd.insert(row - 1, col - 1, val);
            cur.skip_line();
        }
    } else {
        if (!dc.read_size(d.rows) || !dc.read_size(d.cols)) {
            fail("error when determining matrix size, expected: rows cols");
        }
        for (int64_t col = 0; col < d.cols; ++col) {
            for (int64_t row = rd.row_start(col); row < d.rows; ++row) {
                const double val = rd.entry(cur, "error while reading matrix entry");
                rd.insert(row, col, val);
                cur.skip_line();
            }
        }
    }
    sort_row_major(d);
}

// IEEE binary16 and bfloat16 to double (both exact)
double half_to_double(uint16_t h)
{
    const int sign = h >> 15;
    const int exp = (h >> 10) & 0x1f;
    const int man = h & 0x3ff;
    double v;
    if (exp == 0) {
        v = std::ldexp(double(man), -24);
    } else if (exp == 31) {
        v = man ? std::numeric_limits<double>::quiet_NaN()
                : std::numeric_limits<double>::infinity();
    } else {
        v = std::ldexp(double(man | 0x400), exp - 25);
    }
    return sign ? -v : v;
}

double bf16_to_double(uint16_t b)
{
    const uint32_t bits = uint32_t(b) << 16;
    float f;
    std::memcpy(&f, &bits, 4);
    return double(f);
}

constexpr char kMagic[6] = {'G', 'I', 'N', 'K', 'G', 'O'};

void read_binary(const char* buf, int64_t len, MtxData& d)
{
    if (len < 32) fail("failed reading header");
    uint64_t hdr[4];
    std::memcpy(hdr, buf, 32);
    const char* magic = buf;
    const char vt = magic[6];
    const char it = magic[7];
    const bool real = vt == 'D' || vt == 'S' || vt == 'H' || vt == 'B';
    const bool cplx = vt == 'Z' || vt == 'C' || vt == 'X' || vt == 'Y';
    if (std::memcmp(magic, kMagic, 6) != 0 || !(real || cplx) || !(it == 'I' || it == 'L')) {
        fail("invalid header magic number '" + std::string(buf, 8) + "'");
    }
    const uint64_t rows = hdr[1], cols = hdr[2], entries = hdr[3];
    const uint64_t imax = d.index_type == B2S_MTX_I32
                              ? uint64_t(std::numeric_limits<int32_t>::max())
                              : uint64_t(std::numeric_limits<int64_t>::max());
    if (rows > imax || cols > imax) {
        fail("cannot read into this format, its index type would overflow");
    }
    if (cplx) fail("cannot read into this format, would assign complex to real");
    const size_t isz = it == 'I' ? 4 : 8;
    const size_t vsz = vt == 'D' ? 8 : vt == 'S' ? 4 : 2;
    const size_t esz = 2 * isz + vsz;
    const uint64_t avail = uint64_t(len - 32) / esz;
    if (entries > avail) fail("failed reading entry " + std::to_string(avail));
    d.rows = int64_t(rows);
    d.cols = int64_t(cols);
    d.r.resize(size_t(entries));
    d.c.resize(size_t(entries));
    d.v.resize(size_t(entries));
    const char* q = buf + 32;
    for (uint64_t i = 0; i < entries; ++i, q += esz) {
        int64_t row, col;
        if (isz == 4) {
            int32_t a, b;
            std::memcpy(&a, q, 4);
            std::memcpy(&b, q + 4, 4);
            row = a;
            col = b;
        } else {
            std::memcpy(&row, q, 8);
            std::memcpy(&col, q + 8, 8);
        }
        if (d.index_type == B2S_MTX_I32) {
            // the reference assigns the file index to the narrower type
            row = int64_t(int32_t(uint32_t(uint64_t(row))));
            col = int64_t(int32_t(uint32_t(uint64_t(col))));
        }
        const char* pv = q + 2 * isz;
        double val;
        if (vt == 'D') {
            std::memcpy(&val, pv, 8);
        } else if (vt == 'S') {
            float f;
            std::memcpy(&f, pv, 4);
            val = f;
        } else {
            uint16_t h;
            std::memcpy(&h, pv, 2);
            val = vt == 'H' ? half_to_double(h) : bf16_to_double(h);
        }
        d.r[i] = row;
        d.c[i] = col;
        d.v[i] = round_to(d.value_type, val);
    }
    sort_row_major(d);
}

// The stream's default floating-point format is printf's %g with six
// significant digits; to_chars with chars_format::general and precision 6
// is specified to produce exactly that text.
inline char* put_value(char* b, char* e, double v)
{
    return std::to_chars(b, e, v, std::chars_format::general, 6).ptr;
}

inline char* put_int(char* b, char* e, int64_t v) { return std::to_chars(b, e, v).ptr; }

void append_int(std::string& o, int64_t v)
{
    char b[24];
    o.append(b, size_t(put_int(b, b + sizeof(b), v) - b));
}

void write_text(MtxData& d, bool array)
{
    std::string& o = d.bytes;
    o = array ? "%%MatrixMarket matrix array real general\n"
              : "%%MatrixMarket matrix coordinate real general\n";
    const size_t n = d.r.size();
    if (!array) {
        append_int(o, d.rows);
        o += ' ';
        append_int(o, d.cols);
        o += ' ';
        append_int(o, int64_t(n));
        o += '\n';
        // entries in the given order; ranges formatted on separate threads
        const unsigned T = io_threads(n * 24);
        std::vector<std::string> part(T);
        parallel_for(T, [&](unsigned t) {
            const size_t b = n * t / T, e = n * (t + 1) / T;
            std::string& s = part[t];
            s.reserve((e - b) * 24);
            char line[96];
            for (size_t i = b; i < e; ++i) {
                char* q = put_int(line, line + 24, d.r[i] + 1);
                *q++ = ' ';
                q = put_int(q, q + 24, d.c[i] + 1);
                *q++ = ' ';
                q = put_value(q, q + 40, d.v[i]);
                *q++ = '\n';
                s.append(line, size_t(q - line));
            }
        });
        size_t total = o.size();
        for (const auto& s : part) total += s.size();
        o.reserve(total);
        for (const auto& s : part) o += s;
        return;
    }
    // column-major walk over every position; entries in (column, row) order
    std::vector<size_t> perm(n);
    std::iota(perm.begin(), perm.end(), size_t(0));
    std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) {
        return d.c[a] < d.c[b] || (d.c[a] == d.c[b] && d.r[a] < d.r[b]);
    });
    append_int(o, d.rows);
    o += ' ';
    append_int(o, d.cols);
    o += '\n';
    size_t pos = 0;
    char line[48];
    for (int64_t j = 0; j < d.cols; ++j) {
        for (int64_t i = 0; i < d.rows; ++i) {
            char* q;
            if (pos >= n || d.r[perm[pos]] != i || d.c[perm[pos]] != j) {
                q = put_value(line, line + 40, 0.0);
            } else {
                q = put_value(line, line + 40, d.v[perm[pos]]);
                ++pos;
            }
            *q++ = '\n';
            o.append(line, size_t(q - line));
        }
    }
}

void write_binary(MtxData& d)
{
    const bool i32 = d.index_type == B2S_MTX_I32;
    const bool f32 = d.value_type == B2S_MTX_F32;
    const size_t isz = i32 ? 4 : 8, vsz = f32 ? 4 : 8, esz = 2 * isz + vsz;
    const size_t n = d.r.size();
    std::string& o = d.bytes;
    o.resize(32 + n * esz);
    char* q = &o[0];
    std::memcpy(q, kMagic, 6);
    q[6] = f32 ? 'S' : 'D';
    q[7] = i32 ? 'I' : 'L';
    const uint64_t sizes[3] = {uint64_t(d.rows), uint64_t(d.cols), uint64_t(n)};
    std::memcpy(q + 8, sizes, 24);
    q += 32;
    for (size_t i = 0; i < n; ++i, q += esz) {
        if (i32) {
            const int32_t a = int32_t(d.r[i]), b = int32_t(d.c[i]);
            std::memcpy(q, &a, 4);
            std::memcpy(q + 4, &b, 4);
        } else {
            std::memcpy(q, &d.r[i], 8);
            std::memcpy(q + 8, &d.c[i], 8);
        }
        if (f32) {
            const float f = float(d.v[i]);
            std::memcpy(q + 2 * isz, &f, 4);
        } else {
            std::memcpy(q + 2 * isz, &d.v[i], 8);
        }
    }
}

bool valid_types(int value_type, int index_type)
{
    return (value_type == B2S_MTX_F64 || value_type == B2S_MTX_F32) &&
           (index_type == B2S_MTX_I32 || index_type == B2S_MTX_I64);
}

}  // namespace

extern "C" {

int b2s_mtx_read(const void* bytes, int64_t num_bytes, int format, int value_type,
                 int index_type, void* handle_out)
{
    if (handle_out == nullptr || num_bytes < 0 || (bytes == nullptr && num_bytes > 0) ||
        !valid_types(value_type, index_type) ||
        (format != B2S_MTX_TEXT && format != B2S_MTX_BINARY && format != B2S_MTX_GENERIC)) {
        b2s::set_error("b2s_mtx_read: invalid argument");
        return B2S_ERR_INVALID_ARG;
    }
    *static_cast<void**>(handle_out) = nullptr;
    MtxData* d = new (std::nothrow) MtxData;
    if (d == nullptr) {
        b2s::set_error("b2s_mtx_read: out of host memory");
        return B2S_ERR_INVALID_ARG;
    }
    d->value_type = value_type;
    d->index_type = index_type;
    const char* buf = static_cast<const char*>(bytes);
    try {
        if (format == B2S_MTX_GENERIC) {
            if (num_bytes == 0) fail("failed reading from stream");
            format = buf[0] == '%' ? B2S_MTX_TEXT : B2S_MTX_BINARY;
        }
        if (format == B2S_MTX_TEXT) {
            read_text(buf, num_bytes, *d);
        } else {
            read_binary(buf, num_bytes, *d);
        }
    } catch (const MtxError& e) {
        delete d;
        b2s::set_error("%s", e.msg.c_str());
        return B2S_ERR_INVALID_ARG;
    } catch (const std::bad_alloc&) {
        delete d;
        b2s::set_error("b2s_mtx_read: out of host memory");
        return B2S_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        delete d;
        b2s::set_error("b2s_mtx_read: %s", e.what());
        return B2S_ERR_INVALID_ARG;
    }
    *static_cast<void**>(handle_out) = d;
    return B2S_OK;
}

int b2s_mtx_write(int64_t num_rows, int64_t num_cols, int64_t num_entries,
                  const void* row_idxs, const void* col_idxs, const void* values,
                  int value_type, int index_type, int format, void* handle_out)
{
    if (handle_out == nullptr || num_rows < 0 || num_cols < 0 || num_entries < 0 ||
        (num_entries > 0 && (row_idxs == nullptr || col_idxs == nullptr || values == nullptr)) ||
        !valid_types(value_type, index_type) ||
        (format != B2S_MTX_COORDINATE && format != B2S_MTX_ARRAY && format != B2S_MTX_BINARY)) {
        b2s::set_error("b2s_mtx_write: invalid argument");
        return B2S_ERR_INVALID_ARG;
    }
    *static_cast<void**>(handle_out) = nullptr;
    MtxData* d = new (std::nothrow) MtxData;
    if (d == nullptr) {
        b2s::set_error("b2s_mtx_write: out of host memory");
        return B2S_ERR_INVALID_ARG;
    }
    try {
        d->value_type = value_type;
        d->index_type = index_type;
        d->rows = num_rows;
        d->cols = num_cols;
        const size_t n = size_t(num_entries);
        d->r.resize(n);
        d->c.resize(n);
        d->v.resize(n);
        for (size_t i = 0; i < n; ++i) {
            if (index_type == B2S_MTX_I32) {
                d->r[i] = static_cast<const int32_t*>(row_idxs)[i];
                d->c[i] = static_cast<const int32_t*>(col_idxs)[i];
            } else {
                d->r[i] = static_cast<const int64_t*>(row_idxs)[i];
                d->c[i] = static_cast<const int64_t*>(col_idxs)[i];
            }
            d->v[i] = value_type == B2S_MTX_F32 ? double(static_cast<const float*>(values)[i])
                                                : static_cast<const double*>(values)[i];
        }
        if (format == B2S_MTX_BINARY) {
            write_binary(*d);
        } else {
            write_text(*d, format == B2S_MTX_ARRAY);
        }
    } catch (const std::bad_alloc&) {
        delete d;
        b2s::set_error("b2s_mtx_write: out of host memory");
        return B2S_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        delete d;
        b2s::set_error("b2s_mtx_write: %s", e.what());
        return B2S_ERR_INVALID_ARG;
    }
    *static_cast<void**>(handle_out) = d;
    return B2S_OK;
}

int b2s_mtx_sizes(const void* handle, int64_t* sizes_out)
{
    if (handle == nullptr || sizes_out == nullptr) {
        b2s::set_error("b2s_mtx_sizes: null argument");
        return B2S_ERR_INVALID_ARG;
    }
    const MtxData* d = static_cast<const MtxData*>(handle);
    sizes_out[0] = d->rows;
    sizes_out[1] = d->cols;
    sizes_out[2] = int64_t(d->r.size());
    sizes_out[3] = int64_t(d->bytes.size());
    return B2S_OK;
}

int b2s_mtx_copy(const void* handle, void* row_idxs, void* col_idxs, void* values, void* bytes)
{
    if (handle == nullptr) {
        b2s::set_error("b2s_mtx_copy: null handle");
        return B2S_ERR_INVALID_ARG;
    }
    const MtxData* d = static_cast<const MtxData*>(handle);
    const size_t n = d->r.size();
    const bool i32 = d->index_type == B2S_MTX_I32;
    for (size_t i = 0; i < n; ++i) {
        if (row_idxs) {
            if (i32) static_cast<int32_t*>(row_idxs)[i] = int32_t(d->r[i]);
            else static_cast<int64_t*>(row_idxs)[i] = d->r[i];
        }
        if (col_idxs) {
            if (i32) static_cast<int32_t*>(col_idxs)[i] = int32_t(d->c[i]);
            else static_cast<int64_t*>(col_idxs)[i] = d->c[i];
        }
        if (values) {
            if (d->value_type == B2S_MTX_F32) static_cast<float*>(values)[i] = float(d->v[i]);
            else static_cast<double*>(values)[i] = d->v[i];
        }
    }
    if (bytes && !d->bytes.empty()) std::memcpy(bytes, d->bytes.data(), d->bytes.size());
    return B2S_OK;
}

int b2s_mtx_free(void* handle)
{
    delete static_cast<MtxData*>(handle);
    return B2S_OK;
}

}  // extern "C"
