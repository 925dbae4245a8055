// mmio.cpp -- Matrix Market coordinate reader to CSR (the role of the
// reference's read_Dmatrix_32, src/biio2.0/src/biio.h:153, with
// mmio_info/mmio_data of mmio_highlevel.h:7-321).
//
// Same result as the reference reader: 1-based -> 0-based, pattern entries
// read as 1.0, integer entries converted to double, complex entries keep the
// real part; a symmetric (or hermitian) file gets, for every off-diagonal
// entry (i,j), the entry (i,j) in row i and (j,i) in row j; entries of a row
// keep file order (columns are not sorted).  Unlike the reference, a
// malformed file is reported as MF_ERR_IO instead of being read past its end.
// Large files are parsed by several threads (same numbers: std::from_chars
// rounds as strtod does).
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "mf.h"

namespace mf {
void set_last_error(const char *fmt, ...);
}

namespace {

struct Reader {
    const char *p, *e;
    bool eol() const { return p >= e; }
    void skip_space()
    {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) p++;
    }
    bool next_long(long long &v)
    {
        skip_space();
        if (p >= e) return false;
        char *end;
        v = strtoll(p, &end, 10);
        if (end == p) return false;
        p = end;
        return true;
    }
    bool next_double(double &v)
    {
        skip_space();
        if (p >= e) return false;
        char *end;
        v = strtod(p, &end);
        if (end == p) return false;
        p = end;
        return true;
    }
};

std::string lower(std::string s)
{
    for (auto &c : s) c = (char)tolower((unsigned char)c);
    return s;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

// One whitespace-delimited number for the parallel parser: std::from_chars
// (correctly rounded, so the same double as strtod), with strtoll / strtod
// for what from_chars does not take (a leading '+', hexadecimal floats).
inline bool tok_ll(const char *&p, const char *e, long long &v)
{
    while (p < e && is_space(*p)) p++;
    if (p >= e) return false;
    const char *q = (*p == '+') ? p + 1 : p;
    const auto r = std::from_chars(q, e, v);
    if (r.ec == std::errc() && (r.ptr == e || is_space(*r.ptr))) {
        p = r.ptr;
        return true;
    }
    char *end;
    v = strtoll(p, &end, 10);
    if (end == p) return false;
    p = end;
    return true;
}

inline bool tok_d(const char *&p, const char *e, double &v)
{
    while (p < e && is_space(*p)) p++;
    if (p >= e) return false;
    const char *q = (*p == '+') ? p + 1 : p;
    const auto r = std::from_chars(q, e, v);
    if (r.ec == std::errc() && (r.ptr == e || is_space(*r.ptr))) {
        p = r.ptr;
        return true;
    }
    char *end;
    v = strtod(p, &end);
    if (end == p) return false;
    p = end;
    return true;
}

// Entries of a coordinate file parsed by several threads: the entry lines
// are cut at line starts into one piece per thread, each piece's numbers
// are counted (so that every piece knows its first entry), then parsed into
// place.  Returns false -- and the caller parses serially, which also
// gives the exact error -- unless every piece holds whole entries and every
// entry parses with its indices in range.
bool parse_entries_parallel(const char *p, const char *e, long long NZ, long long M, long long N, bool pattern,
                            bool complex_, bool integer, int nthreads, std::vector<int> &ri, std::vector<int> &ci,
                            std::vector<double> &vv)
{
    const int per = 2 + (pattern ? 0 : (complex_ ? 2 : 1));  // numbers per entry
    const int T = nthreads;
    std::vector<const char *> b((size_t)T + 1);
    b[0] = p;
    b[T] = e;
    for (int t = 1; t < T; t++) {
        const char *q = p + (size_t)(e - p) * (size_t)t / (size_t)T;
        if (q < b[t - 1]) q = b[t - 1];
        const char *nl = (const char *)memchr(q, '\n', (size_t)(e - q));
        b[t] = nl ? nl + 1 : e;
    }
    std::vector<long long> cnt((size_t)T, 0);
    auto count = [&](int t) {
        long long c = 0;
        const char *q = b[t], *qe = b[t + 1];
        while (q < qe) {
            while (q < qe && is_space(*q)) q++;
            if (q >= qe) break;
            c++;
            while (q < qe && !is_space(*q)) q++;
        }
        cnt[t] = c;
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < T; t++) th.emplace_back(count, t);
        count(0);
        for (auto &x : th) x.join();
    }
    std::vector<long long> first((size_t)T + 1, 0);
    for (int t = 0; t < T; t++) {
        if (cnt[t] % per != 0) return false;  // an entry spans two pieces: not one entry per line
        first[t + 1] = first[t] + cnt[t] / per;
    }
    if (first[T] < NZ) return false;  // truncated: the serial parser reports where
    std::vector<char> bad((size_t)T, 0);
    auto parse = [&](int t) {
        const char *q = b[t];
        const char *qe = b[t + 1];
        const long long k1 = std::min(first[t + 1], NZ);
        for (long long k = first[t]; k < k1; k++) {
            long long i, j;
            double v = 1.0, im;
            if (!tok_ll(q, qe, i) || !tok_ll(q, qe, j)) {
                bad[t] = 1;
                return;
            }
            if (!pattern) {
                if (integer) {
                    long long iv;
                    if (!tok_ll(q, qe, iv)) {
                        bad[t] = 1;
                        return;
                    }
                    v = (double)(int)iv;
                } else if (!tok_d(q, qe, v)) {
                    bad[t] = 1;
                    return;
                }
                if (complex_ && !tok_d(q, qe, im)) {
                    bad[t] = 1;
                    return;
                }
            }
            if (i < 1 || i > M || j < 1 || j > N) {
                bad[t] = 1;
                return;
            }
            ri[k] = (int)(i - 1);
            ci[k] = (int)(j - 1);
            vv[k] = v;
        }
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < T; t++) th.emplace_back(parse, t);
        parse(0);
        for (auto &x : th) x.join();
    }
    for (int t = 0; t < T; t++)
        if (bad[t]) return false;
    return true;
}

}  // namespace

namespace mf {

// The entries of a Matrix Market coordinate file in file order (0-based
// row, column, value), its sizes and whether it is symmetric (or
// hermitian); a symmetric file's off-diagonal entries are checked to mirror
// inside the rows.  The CSR is built from these by mf_read_matrix_market
// (host) or mf_matrix_create_mtx (device).
mf_status mtx_read_coo(const char *path, long long &M, long long &N, long long &NZ, bool &sym, std::vector<int> &ri,
                       std::vector<int> &ci, std::vector<double> &vv)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        mf::set_last_error("cannot open %s: %s", path, strerror(errno));
        return MF_ERR_IO;
    }
    std::vector<char> buf;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize((size_t)sz + 1);
    size_t got = fread(buf.data(), 1, (size_t)sz, f);
    fclose(f);
    buf[got] = 0;
    const char *p = buf.data(), *e = buf.data() + got;
    // banner
    const char *nl = (const char *)memchr(p, '\n', e - p);
    std::string banner(p, nl ? nl : e);
    std::string bl = lower(banner);
    if (bl.rfind("%%matrixmarket", 0) != 0 || bl.find("coordinate") == std::string::npos) {
        mf::set_last_error("%s: not a Matrix Market coordinate file", path);
        return MF_ERR_IO;
    }
    const bool pattern = bl.find("pattern") != std::string::npos;
    const bool complex_ = bl.find("complex") != std::string::npos;
    const bool integer = bl.find("integer") != std::string::npos;
    sym = bl.find("symmetric") != std::string::npos || bl.find("hermitian") != std::string::npos;
    p = nl ? nl + 1 : e;
    // skip comments / blank lines
    while (p < e) {
        const char *q = p;
        while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) q++;
        if (q < e && (*q == '%' || *q == '\n')) {
            const char *n2 = (const char *)memchr(q, '\n', e - q);
            p = n2 ? n2 + 1 : e;
            continue;
        }
        break;
    }
    Reader rd{p, e};
    if (!rd.next_long(M) || !rd.next_long(N) || !rd.next_long(NZ) || M < 0 || N < 0 || NZ < 0 || M > 0x7fffffff ||
        N > 0x7fffffff) {
        mf::set_last_error("%s: bad size line", path);
        return MF_ERR_IO;
    }
    ri.assign((size_t)NZ, 0);
    ci.assign((size_t)NZ, 0);
    vv.assign((size_t)NZ, 0.0);
    // entries in parallel on files of 200,000 entries or more, serially
    // otherwise or when the file is not one entry per line;
    // MF_MTX_THREADS=<t> sets the threads for every file (1: serial)
    int nth = (int)std::thread::hardware_concurrency();
    if (NZ < 200000) nth = 1;
    if (const char *env = getenv("MF_MTX_THREADS")) nth = atoi(env);
    nth = std::max(1, std::min(nth, 64));
    bool parsed = nth > 1 && parse_entries_parallel(rd.p, e, NZ, M, N, pattern, complex_, integer, nth, ri, ci, vv);
    for (long long k = 0; !parsed && k < NZ; k++) {
        long long i, j;
        double v = 1.0, im;
        if (!rd.next_long(i) || !rd.next_long(j)) {
            mf::set_last_error("%s: truncated at entry %lld", path, k);
            return MF_ERR_IO;
        }
        if (!pattern) {
            if (integer) {
                long long iv;
                if (!rd.next_long(iv)) {
                    mf::set_last_error("%s: bad value at entry %lld", path, k);
                    return MF_ERR_IO;
                }
                v = (double)(int)iv;
            } else if (!rd.next_double(v)) {
                mf::set_last_error("%s: bad value at entry %lld", path, k);
                return MF_ERR_IO;
            }
            if (complex_ && !rd.next_double(im)) {
                mf::set_last_error("%s: bad imaginary part at entry %lld", path, k);
                return MF_ERR_IO;
            }
        }
        if (i < 1 || i > M || j < 1 || j > N) {
            mf::set_last_error("%s: entry %lld index out of range", path, k);
            return MF_ERR_IO;
        }
        ri[k] = (int)(i - 1);
        ci[k] = (int)(j - 1);
        vv[k] = v;
    }
    if (sym)
        for (long long k = 0; k < NZ; k++)
            if (ri[k] != ci[k] && ci[k] >= M) {
                mf::set_last_error("%s: symmetric entry mirrors outside the rows", path);
                return MF_ERR_IO;
            }
    return MF_OK;
}

}  // namespace mf

extern "C" mf_status mf_read_matrix_market(const char *path, int *m_out, int *n_out, int *nnz_out, int **rowptr,
                                           int **colidx, double **val, int *is_symmetric)
{
    if (!path || !m_out || !n_out || !nnz_out || !rowptr || !colidx || !val) return MF_ERR_INVALID_ARG;
    long long M, N, NZ;
    bool sym = false;
    std::vector<int> ri, ci;
    std::vector<double> vv;
    const mf_status st = mf::mtx_read_coo(path, M, N, NZ, sym, ri, ci, vv);
    if (st != MF_OK) return st;
    // CSR: a row's entries in file order, a symmetric entry's mirror placed
    // when the entry is read
    std::vector<long long> cnt((size_t)M + 1, 0);
    for (long long k = 0; k < NZ; k++) {
        cnt[ri[k]]++;
        if (sym && ri[k] != ci[k]) cnt[ci[k]]++;
    }
    // exclusive scan
    long long run = 0;
    for (long long r = 0; r <= M; r++) {
        long long c = cnt[r];
        cnt[r] = run;
        run += c;
    }
    if (run > 0x7fffffff) {
        mf::set_last_error("%s: more than 2^31-1 entries", path);
        return MF_ERR_UNSUPPORTED;
    }
    int *rp = (int *)malloc(sizeof(int) * (M + 1));
    int *cc = (int *)malloc(sizeof(int) * (run > 0 ? run : 1));
    double *va = (double *)malloc(sizeof(double) * (run > 0 ? run : 1));
    if (!rp || !cc || !va) {
        free(rp);
        free(cc);
        free(va);
        return MF_ERR_NO_MEMORY;
    }
    for (long long r = 0; r <= M; r++) rp[r] = (int)cnt[r];
    std::vector<long long> fill((size_t)M + 1, 0);
    for (long long k = 0; k < NZ; k++) {
        int i = ri[k], j = ci[k];
        long long o = rp[i] + fill[i]++;
        cc[o] = j;
        va[o] = vv[k];
        if (sym && i != j) {
            o = rp[j] + fill[j]++;
            cc[o] = i;
            va[o] = vv[k];
        }
    }
    *m_out = (int)M;
    *n_out = (int)N;
    *nnz_out = (int)run;
    *rowptr = rp;
    *colidx = cc;
    *val = va;
    if (is_symmetric) *is_symmetric = sym ? 1 : 0;
    return MF_OK;
}

// ---- binary CSR (.cbd) ------------------------------------------------
//
// The reference's binary cache of a parsed matrix (binary_read_csr /
// binary_write_csr, src/biio2.0/src/biio.h:22-94): int32 rows, int32 cols,
// int64 nnz, then int64 row_ptr[rows + 1], int32 col_idx[nnz] and double
// val[nnz], in the machine's byte order.  The layout is kept because files
// written by the reference must read here and the other way round.  Unlike
// the reference, the reader checks the file length against the header and
// the row pointers and column indices against the sizes, and reports a
// malformed file as MF_ERR_IO.

extern "C" mf_status mf_read_cbd(const char *path, int *m_out, int *n_out, int *nnz_out, int **rowptr, int **colidx,
                                 double **val)
{
    if (!path || !m_out || !n_out || !nnz_out || !rowptr || !colidx || !val) return MF_ERR_INVALID_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) {
        mf::set_last_error("cannot open %s: %s", path, strerror(errno));
        return MF_ERR_IO;
    }
    fseek(f, 0, SEEK_END);
    const long long fsz = (long long)ftell(f);
    fseek(f, 0, SEEK_SET);
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;
    if (fread(&rows, 4, 1, f) != 1 || fread(&cols, 4, 1, f) != 1 || fread(&nnz, 8, 1, f) != 1) {
        fclose(f);
        mf::set_last_error("%s: truncated header", path);
        return MF_ERR_IO;
    }
    if (rows < 0 || cols < 0 || nnz < 0 || nnz > 0x7fffffffLL ||
        fsz != 16 + 8LL * ((long long)rows + 1) + 12LL * (long long)nnz) {
        fclose(f);
        if (nnz > 0x7fffffffLL) {
            mf::set_last_error("%s: more than 2^31-1 entries", path);
            return MF_ERR_UNSUPPORTED;
        }
        mf::set_last_error("%s: header (%d x %d, %lld entries) does not match the file length %lld", path, rows, cols,
                           (long long)nnz, fsz);
        return MF_ERR_IO;
    }
    std::vector<int64_t> rp64((size_t)rows + 1);
    int *rp = (int *)malloc(sizeof(int) * ((size_t)rows + 1));
    int *cc = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    double *va = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    auto fail = [&](mf_status st, const char *what) {
        fclose(f);
        free(rp);
        free(cc);
        free(va);
        if (what) mf::set_last_error("%s: %s", path, what);
        return st;
    };
    if (!rp || !cc || !va) return fail(MF_ERR_NO_MEMORY, nullptr);
    if (fread(rp64.data(), 8, (size_t)rows + 1, f) != (size_t)rows + 1 ||
        fread(cc, 4, (size_t)nnz, f) != (size_t)nnz || fread(va, 8, (size_t)nnz, f) != (size_t)nnz)
        return fail(MF_ERR_IO, "truncated arrays");
    if (rp64[0] != 0 || rp64[rows] != nnz) return fail(MF_ERR_IO, "row pointers do not span the entries");
    for (int r = 0; r < rows; r++) {
        if (rp64[r + 1] < rp64[r]) return fail(MF_ERR_IO, "row pointers decrease");
        rp[r] = (int)rp64[r];
    }
    rp[rows] = (int)nnz;
    for (int64_t k = 0; k < nnz; k++)
        if (cc[k] < 0 || cc[k] >= cols) return fail(MF_ERR_IO, "column index out of range");
    fclose(f);
    *m_out = rows;
    *n_out = cols;
    *nnz_out = (int)nnz;
    *rowptr = rp;
    *colidx = cc;
    *val = va;
    return MF_OK;
}

extern "C" mf_status mf_write_cbd(const char *path, int m, int n, int nnz, const int *rowptr, const int *colidx,
                                  const double *val)
{
    if (!path || m < 0 || n < 0 || nnz < 0 || !rowptr || (nnz > 0 && (!colidx || !val))) return MF_ERR_INVALID_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) {
        mf::set_last_error("cannot create %s: %s", path, strerror(errno));
        return MF_ERR_IO;
    }
    const int32_t rows = m, cols = n;
    const int64_t nz = nnz;
    std::vector<int64_t> rp64((size_t)m + 1);
    for (int r = 0; r <= m; r++) rp64[r] = rowptr[r];
    bool ok = fwrite(&rows, 4, 1, f) == 1 && fwrite(&cols, 4, 1, f) == 1 && fwrite(&nz, 8, 1, f) == 1 &&
              fwrite(rp64.data(), 8, (size_t)m + 1, f) == (size_t)m + 1 &&
              (nnz == 0 || (fwrite(colidx, 4, (size_t)nnz, f) == (size_t)nnz &&
                            fwrite(val, 8, (size_t)nnz, f) == (size_t)nnz));
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        mf::set_last_error("%s: write failed", path);
        return MF_ERR_IO;
    }
    return MF_OK;
}

// The reference CLIs' reader (read_Dmatrix_32, src/biio2.0/src/biio.h:153-194):
// the file name's extension picks the format, ".cbd" binary CSR or ".mtx"
// Matrix Market.  A binary file holds the matrix as stored, so
// *is_symmetric is 0 for it.
extern "C" mf_status mf_read_matrix(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx,
                                    double **val, int *is_symmetric)
{
    if (!path) return MF_ERR_INVALID_ARG;
    const size_t len = strlen(path);
    if (len >= 3 && !strcmp(path + len - 3, "cbd")) {
        const mf_status st = mf_read_cbd(path, m, n, nnz, rowptr, colidx, val);
        if (st == MF_OK && is_symmetric) *is_symmetric = 0;
        return st;
    }
    if (len >= 3 && !strcmp(path + len - 3, "mtx"))
        return mf_read_matrix_market(path, m, n, nnz, rowptr, colidx, val, is_symmetric);
    mf::set_last_error("%s: unsupported file type (expected .mtx or .cbd)", path);
    return MF_ERR_IO;
}
