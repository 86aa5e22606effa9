// Matrix Market reader -> CSR (host).
//
// Replaces csr::matrix_market_reader (common/csr/matrix_market_reader.h:
// 48-673).  Same accepted files and the same CSR: a "%%MatrixMarket matrix
// coordinate <type> <symmetry>" banner (type real / integer / pattern /
// complex; symmetry general or symmetric -- a symmetric file's off-diagonal
// entries are mirrored, hermitian and skew-symmetric are refused, as there),
// '%' comment lines (an "%%AMGX" block-size line included), 1-based indices
// checked against the declared size, entries stably sorted by (row, column)
// with duplicates kept, pattern entries read as 1.
//
// The file is read in one piece and parsed with strtol/strtod straight from
// the buffer (strtod rounds correctly, so values equal the reference's
// operator>> into double); the COO->CSR step is a counting sort by row
// followed by a stable sort of each row by column, O(nnz) plus the per-row
// sorts, instead of a global stable_sort of the triples.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/hpblas1.h"

namespace {

thread_local char g_mm_error[512];

int mm_fail(int status, const char* fmt, const char* arg = "") {
    std::snprintf(g_mm_error, sizeof(g_mm_error), fmt, arg);
    return status;
}

std::string lower(std::string s) {
    for (char& c : s) c = char(std::tolower(static_cast<unsigned char>(c)));
    return s;
}

struct Entry {
    int32_t row, col;
    double re, im;
};

}  // namespace

extern "C" {

const char* hpb_mm_last_error(void) { return g_mm_error; }

void hpb_mm_free(hpb_mm_csr* m) {
    if (m == nullptr) return;
    std::free(m->row_ptr);
    std::free(m->col_ind);
    std::free(m->val);
    m->row_ptr = nullptr;
    m->col_ind = nullptr;
    m->val = nullptr;
}

int hpb_mm_read_csr(const char* path, hpb_mm_csr* out) {
    g_mm_error[0] = 0;
    if (path == nullptr || out == nullptr) return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: null argument");
    *out = hpb_mm_csr{};
    std::FILE* f = std::fopen(path, "rb");
    if (f == nullptr) return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: cannot open %s", path);
    std::vector<char> buf;
    {
        std::fseek(f, 0, SEEK_END);
        const long len = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        if (len < 0) {
            std::fclose(f);
            return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: cannot read %s", path);
        }
        buf.resize(size_t(len) + 1);
        const size_t got = std::fread(buf.data(), 1, size_t(len), f);
        std::fclose(f);
        buf[got] = '\0';
        buf.resize(got + 1);
    }
    char* p = buf.data();
    char* const end = buf.data() + buf.size() - 1;
    auto next_line = [&](char*& q) {
        while (q < end && *q != '\n') ++q;
        if (q < end) ++q;
    };
    // banner
    std::string banner;
    {
        char* q = p;
        next_line(q);
        banner.assign(p, size_t(q - p));
        p = q;
    }
    std::vector<std::string> tok;
    {
        size_t i = 0;
        while (i < banner.size()) {
            while (i < banner.size() && std::isspace(static_cast<unsigned char>(banner[i]))) ++i;
            size_t j = i;
            while (j < banner.size() && !std::isspace(static_cast<unsigned char>(banner[j]))) ++j;
            if (j > i) tok.push_back(banner.substr(i, j - i));
            i = j;
        }
    }
    if (tok.size() != 5 || tok[0] != "%%MatrixMarket" || lower(tok[1]) != "matrix")
        return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: invalid MatrixMarket banner");
    const std::string storage = lower(tok[2]), type = lower(tok[3]), symmetry = lower(tok[4]);
    if (storage != "coordinate")
        return mm_fail(HPB_ERROR_NOT_SUPPORTED, "hpb_mm_read_csr: storage format [%s] is not supported (coordinate only)",
                       storage.c_str());
    if (type != "real" && type != "integer" && type != "pattern" && type != "complex")
        return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: invalid MatrixMarket data type [%s]", type.c_str());
    if (symmetry == "hermitian" || symmetry == "skew-symmetric")
        return mm_fail(HPB_ERROR_NOT_SUPPORTED, "hpb_mm_read_csr: %s matrices are not supported", symmetry.c_str());
    if (symmetry != "general" && symmetry != "symmetric")
        return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: invalid MatrixMarket symmetry [%s]", symmetry.c_str());
    // comments and blank lines, then the size line
    for (;;) {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
        if (p < end && (*p == '%' || *p == '\n')) {
            next_line(p);
            continue;
        }
        break;
    }
    errno = 0;
    char* q = nullptr;
    const long long nr = std::strtoll(p, &q, 10);
    const long long nc = (q != p) ? std::strtoll(p = q, &q, 10) : -1;
    const long long ne = (q != p) ? std::strtoll(p = q, &q, 10) : -1;
    if (q == p || errno != 0 || nr < 0 || nc < 0 || ne < 0 || nr > INT32_MAX - 1 || nc > INT32_MAX)
        return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: error while reading sizes");
    p = q;
    const bool cplx = type == "complex", pattern = type == "pattern", sym = symmetry == "symmetric";
    std::vector<Entry> e;
    try {
        e.reserve(size_t(ne) * (sym ? 2 : 1));
    } catch (const std::bad_alloc&) {
        return mm_fail(HPB_ERROR_OUT_OF_MEMORY, "hpb_mm_read_csr: out of host memory");
    }
    for (long long k = 0; k < ne; ++k) {
        Entry t{0, 0, 1.0, 0.0};
        const long long r = std::strtoll(p, &q, 10);
        if (q == p) return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: unexpected end of file in the entries");
        p = q;
        const long long c = std::strtoll(p, &q, 10);
        if (q == p) return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: unexpected end of file in the entries");
        p = q;
        if (!pattern) {
            t.re = std::strtod(p, &q);
            if (q == p) return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: unexpected end of file in the entries");
            p = q;
            if (cplx) {
                t.im = std::strtod(p, &q);
                if (q == p)
                    return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: unexpected end of file in the entries");
                p = q;
            }
        }
        if (r < 1 || c < 1)
            return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: found invalid %s index (index < 1)",
                           r < 1 ? "row" : "column");
        if (r > nr || c > nc)
            return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: found invalid %s index (index > size)",
                           r > nr ? "row" : "column");
        t.row = int32_t(r - 1);
        t.col = int32_t(c - 1);
        e.push_back(t);
    }
    if (sym) {  // mirror the off-diagonal entries, appended after the file's entries
        const size_t n0 = e.size();
        for (size_t k = 0; k < n0; ++k)
            if (e[k].row != e[k].col) e.push_back(Entry{e[k].col, e[k].row, e[k].re, e[k].im});
    }
    if (e.size() > size_t(INT32_MAX))
        return mm_fail(HPB_ERROR_INVALID_VALUE, "hpb_mm_read_csr: more than 2^31 - 1 entries");
    // COO -> CSR: stable counting sort by row, then a stable sort of each row
    // by column (together: the stable order by (row, column))
    const size_t nnz = e.size();
    auto* rp = static_cast<int32_t*>(std::calloc(size_t(nr) + 1, sizeof(int32_t)));
    auto* ci = static_cast<int32_t*>(std::malloc(std::max<size_t>(nnz, 1) * sizeof(int32_t)));
    auto* val = static_cast<double*>(std::malloc(std::max<size_t>(nnz, 1) * sizeof(double) * (cplx ? 2 : 1)));
    std::vector<uint32_t> order;
    bool order_ok = true;
    try {
        order.resize(nnz);
    } catch (const std::bad_alloc&) {
        order_ok = false;
    }
    if (rp == nullptr || ci == nullptr || val == nullptr || !order_ok) {
        std::free(rp);
        std::free(ci);
        std::free(val);
        return mm_fail(HPB_ERROR_OUT_OF_MEMORY, "hpb_mm_read_csr: out of host memory");
    }
    for (const Entry& t : e) ++rp[t.row + 1];
    for (long long r = 0; r < nr; ++r) rp[r + 1] += rp[r];
    {
        std::vector<int32_t> fill(rp, rp + nr);
        for (size_t k = 0; k < nnz; ++k) order[size_t(fill[size_t(e[k].row)]++)] = uint32_t(k);
    }
    for (long long r = 0; r < nr; ++r)
        std::stable_sort(order.begin() + rp[r], order.begin() + rp[r + 1],
                         [&](uint32_t a, uint32_t b) { return e[a].col < e[b].col; });
    for (size_t k = 0; k < nnz; ++k) {
        const Entry& t = e[order[k]];
        ci[k] = t.col;
        if (cplx) {
            val[2 * k] = t.re;
            val[2 * k + 1] = t.im;
        } else {
            val[k] = t.re;
        }
    }
    out->rows = int32_t(nr);
    out->cols = int32_t(nc);
    out->nnz = int64_t(nnz);
    out->is_complex = cplx ? 1 : 0;
    out->symmetric = sym ? 1 : 0;
    out->row_ptr = rp;
    out->col_ind = ci;
    out->val = val;
    return HPB_SUCCESS;
}

}  // extern "C"
