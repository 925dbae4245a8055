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
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
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

}  // namespace

extern "C" mf_status mf_read_matrix_market(const char *path, int *m_out, int *n_out, int *nnz_out, int **rowptr,
                                           int **colidx, double **val, int *is_symmetric)
{
    if (!path || !m_out || !n_out || !nnz_out || !rowptr || !colidx || !val) return MF_ERR_INVALID_ARG;
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
    const bool sym = bl.find("symmetric") != std::string::npos || bl.find("hermitian") != std::string::npos;
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
    long long M, N, NZ;
    if (!rd.next_long(M) || !rd.next_long(N) || !rd.next_long(NZ) || M < 0 || N < 0 || NZ < 0 || M > 0x7fffffff ||
        N > 0x7fffffff) {
        mf::set_last_error("%s: bad size line", path);
        return MF_ERR_IO;
    }
    std::vector<int> ri((size_t)NZ), ci((size_t)NZ);
    std::vector<double> vv((size_t)NZ);
    std::vector<long long> cnt((size_t)M + 1, 0);
    for (long long k = 0; k < NZ; k++) {
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
        cnt[ri[k]]++;
        if (sym && ri[k] != ci[k]) {
            if (ci[k] >= M) {
                mf::set_last_error("%s: symmetric entry mirrors outside the rows", path);
                return MF_ERR_IO;
            }
            cnt[ci[k]]++;
        }
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
