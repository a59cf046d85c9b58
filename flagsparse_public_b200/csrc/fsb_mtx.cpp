// fsb_mtx.cpp -- Matrix Market (.mtx) coordinate files to CSR on the host.
//
// Semantics follow FlagSparse's loader (load_mtx_to_csr_torch,
// tests/test_spmv.py:103-178), bit for bit:
//   * the header "%%MatrixMarket ... <field> <symmetry>" (lower-cased; real /
//     general when it has fewer than five tokens); other '%' lines and blank
//     lines are skipped anywhere; the first remaining line gives
//     "n_rows n_cols [nnz]" (a missing nnz -- "array" files -- reads as 0,
//     i.e. an empty matrix);
//   * the first nnz data lines are read; "pattern" entries are 1.0, otherwise
//     the third token (the real part for complex fields);
//   * entries outside the matrix are dropped; duplicates are summed in file
//     order starting from 0.0 (float64); symmetric and hermitian files mirror
//     off-diagonal entries (c, r) += v, skew-symmetric ones (c, r) -= v,
//     each mirror right after its entry;
//   * explicit zeros stay; columns are sorted within each row.
// Parsing runs on several threads (line ranges), the per-row column sort and
// duplicate sums too; the float64 values are rounded to the caller's type by
// the caller.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/flagsparse_b200.h"

namespace fsb_host {
void set_error(const char* fmt, ...);
}

namespace {

struct Entry {
    int64_t row, col;
    double v;
    int64_t order;  // file order of the contribution (mirror right after its entry)
    int neg;        // skew-symmetric mirror: subtract
};

struct MtxResult {
    int64_t n_rows = 0, n_cols = 0;
    std::vector<int64_t> indptr, indices;
    std::vector<double> values;
};

bool read_file(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(&out[0], 1, (size_t)n, f) : 0;
    std::fclose(f);
    return got == out.size();
}

// Python str.strip() of ASCII whitespace
inline void strip(const char*& b, const char*& e) {
    while (b < e && std::isspace((unsigned char)*b)) ++b;
    while (e > b && std::isspace((unsigned char)e[-1])) --e;
}

inline int split(const char* b, const char* e, const char** tb, const char** te, int max_tokens) {
    int n = 0;
    while (b < e && n < max_tokens) {
        while (b < e && std::isspace((unsigned char)*b)) ++b;
        if (b >= e) break;
        tb[n] = b;
        while (b < e && !std::isspace((unsigned char)*b)) ++b;
        te[n++] = b;
    }
    return n;
}

bool parse_int(const char* b, const char* e, int64_t* out) {
    std::string s(b, e);
    char* end = nullptr;
    errno = 0;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (errno || end != s.c_str() + s.size() || s.empty()) return false;
    *out = v;
    return true;
}

bool parse_double(const char* b, const char* e, double* out) {
    std::string s(b, e);
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end != s.c_str() + s.size() || s.empty()) return false;
    *out = v;
    return true;
}

}  // namespace

extern "C" void* fsb_mtx_open(const char* path, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int threads) {
    if (!path || !n_rows || !n_cols || !nnz) {
        fsb_host::set_error("fsb_mtx_open: null argument");
        return nullptr;
    }
    std::string text;
    if (!read_file(path, text)) {
        fsb_host::set_error("fsb_mtx_open: cannot read %s", path);
        return nullptr;
    }
    // line starts (sequential scan: cheap next to parsing)
    std::vector<std::pair<size_t, size_t>> lines;
    {
        size_t s = 0;
        for (size_t i = 0; i <= text.size(); ++i) {
            if (i == text.size() || text[i] == '\n') {
                if (i > s || i < text.size()) lines.emplace_back(s, i);
                s = i + 1;
            }
        }
    }
    std::string field = "real", symmetry = "general";
    bool have_header = false;
    int64_t hr = 0, hc = 0, hn = 0;
    std::vector<std::pair<size_t, size_t>> data;
    for (const auto& ln : lines) {
        const char* b = text.data() + ln.first;
        const char* e = text.data() + ln.second;
        strip(b, e);
        if ((size_t)(e - b) >= 14 && std::strncmp(b, "%%MatrixMarket", 14) == 0) {
            const char *tb[8], *te[8];
            const int nt = split(b, e, tb, te, 8);
            if (nt >= 5) {
                field.assign(tb[3], te[3]);
                symmetry.assign(tb[4], te[4]);
                for (auto& ch : field) ch = (char)std::tolower((unsigned char)ch);
                for (auto& ch : symmetry) ch = (char)std::tolower((unsigned char)ch);
            }
            continue;
        }
        if (b < e && *b == '%') continue;
        if (!have_header && b < e) {
            const char *tb[4], *te[4];
            const int nt = split(b, e, tb, te, 4);
            if (nt < 2 || !parse_int(tb[0], te[0], &hr) || !parse_int(tb[1], te[1], &hc) ||
                (nt > 2 && !parse_int(tb[2], te[2], &hn))) {
                fsb_host::set_error("fsb_mtx_open: cannot parse the size line of %s", path);
                return nullptr;
            }
            if (nt == 2) hn = 0;
            have_header = true;
            continue;
        }
        if (b < e) data.emplace_back((size_t)(b - text.data()), (size_t)(e - text.data()));
    }
    if (!have_header) {
        fsb_host::set_error("Cannot parse .mtx header: %s", path);
        return nullptr;
    }
    if (hr < 0 || hc < 0 || hn < 0) {
        fsb_host::set_error("fsb_mtx_open: negative sizes in %s", path);
        return nullptr;
    }
    auto* res = new MtxResult();
    res->n_rows = hr;
    res->n_cols = hc;
    res->indptr.assign((size_t)hr + 1, 0);
    const bool pattern = field == "pattern";
    const bool sym = symmetry == "symmetric" || symmetry == "hermitian";
    const bool skew = symmetry == "skew-symmetric";
    const int64_t n_data = hn < (int64_t)data.size() ? hn : (int64_t)data.size();
    if (hn == 0 || n_data == 0) {
        *n_rows = hr;
        *n_cols = hc;
        *nnz = 0;
        return res;
    }
    // parse entries in parallel over line ranges: entry i owns orders 2i, 2i+1
    int nth = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (nth < 1) nth = 1;
    if (nth > 64) nth = 64;
    if (n_data < 65536) nth = 1;
    std::vector<std::vector<Entry>> parts((size_t)nth);
    std::vector<int> bad((size_t)nth, 0);
    auto work = [&](int t) {
        const int64_t lo = n_data * t / nth, hi = n_data * (t + 1) / nth;
        auto& out = parts[(size_t)t];
        out.reserve((size_t)(hi - lo) * (sym || skew ? 2 : 1));
        for (int64_t i = lo; i < hi; ++i) {
            const char* b = text.data() + data[(size_t)i].first;
            const char* e = text.data() + data[(size_t)i].second;
            const char *tb[4], *te[4];
            const int nt = split(b, e, tb, te, 4);
            int64_t r, c;
            double v = 1.0;
            if (nt < 2 || !parse_int(tb[0], te[0], &r) || !parse_int(tb[1], te[1], &c) ||
                (!pattern && (nt < 3 || !parse_double(tb[2], te[2], &v)))) {
                bad[(size_t)t] = 1;
                return;
            }
            r -= 1;
            c -= 1;
            if (r >= 0 && r < hr && c >= 0 && c < hc) {
                out.push_back(Entry{r, c, v, 2 * i, 0});
                if (r != c && (sym || skew) && c < hr && r < hc) out.push_back(Entry{c, r, v, 2 * i + 1, skew ? 1 : 0});
            }
        }
    };
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < nth; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
    }
    for (int t = 0; t < nth; ++t)
        if (bad[(size_t)t]) {
            delete res;
            fsb_host::set_error("fsb_mtx_open: malformed entry line in %s", path);
            return nullptr;
        }
    // bucket by row (stable: thread parts in order, entries in order)
    std::vector<int64_t> count((size_t)hr + 1, 0);
    for (const auto& p : parts)
        for (const auto& en : p) ++count[(size_t)en.row + 1];
    for (int64_t r = 0; r < hr; ++r) count[(size_t)r + 1] += count[(size_t)r];
    std::vector<Entry> by_row((size_t)count[(size_t)hr]);
    {
        std::vector<int64_t> fill(count.begin(), count.end() - 1);
        for (const auto& p : parts)
            for (const auto& en : p) by_row[(size_t)fill[(size_t)en.row]++] = en;
    }
    parts.clear();
    // per row: stable sort by column (file order kept among duplicates), then
    // sum each column's contributions in file order starting from 0.0
    std::vector<int64_t> row_nnz((size_t)hr, 0);
    auto rows_work = [&](int t, bool emit) {
        const int64_t lo = hr * t / nth, hi = hr * (t + 1) / nth;
        for (int64_t r = lo; r < hi; ++r) {
            auto b = by_row.begin() + count[(size_t)r], e = by_row.begin() + count[(size_t)r + 1];
            if (!emit)
                std::stable_sort(b, e, [](const Entry& x, const Entry& y) {
                    return x.col < y.col || (x.col == y.col && x.order < y.order);
                });
            int64_t k = emit ? res->indptr[(size_t)r] : 0;
            for (auto it = b; it != e;) {
                const int64_t col = it->col;
                double acc = 0.0;
                for (; it != e && it->col == col; ++it) acc = it->neg ? acc - it->v : acc + it->v;
                if (emit) {
                    res->indices[(size_t)k] = col;
                    res->values[(size_t)k] = acc;
                }
                ++k;
            }
            if (!emit) row_nnz[(size_t)r] = k;
        }
    };
    if (hr < 4096) nth = 1;
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < nth; ++t) pool.emplace_back(rows_work, t, false);
        rows_work(0, false);
        for (auto& th : pool) th.join();
    }
    for (int64_t r = 0; r < hr; ++r) res->indptr[(size_t)r + 1] = res->indptr[(size_t)r] + row_nnz[(size_t)r];
    const int64_t total = res->indptr[(size_t)hr];
    res->indices.resize((size_t)total);
    res->values.resize((size_t)total);
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < nth; ++t) pool.emplace_back(rows_work, t, true);
        rows_work(0, true);
        for (auto& th : pool) th.join();
    }
    *n_rows = hr;
    *n_cols = hc;
    *nnz = total;
    return res;
}

extern "C" int fsb_mtx_read(void* handle, int64_t* indptr, int64_t* indices, double* values) {
    auto* res = static_cast<MtxResult*>(handle);
    if (!res || !indptr || (!res->indices.empty() && (!indices || !values))) {
        fsb_host::set_error("fsb_mtx_read: null argument");
        return FSB_ERR_INVALID;
    }
    std::memcpy(indptr, res->indptr.data(), res->indptr.size() * sizeof(int64_t));
    if (!res->indices.empty()) {
        std::memcpy(indices, res->indices.data(), res->indices.size() * sizeof(int64_t));
        std::memcpy(values, res->values.data(), res->values.size() * sizeof(double));
    }
    return FSB_OK;
}

extern "C" void fsb_mtx_close(void* handle) { delete static_cast<MtxResult*>(handle); }
