/*
 * mf_oracle.c -- CPU oracle (test infrastructure only; see mf_oracle.h).
 *
 * Plain C restatement of the reference's CPU algorithms.  Each function
 * names the reference file:line it follows.  Sums are written as separate
 * multiply and add statements and the file is compiled with
 * -ffp-contract=off so that no fused multiply-add changes a rounding.
 */
#include "mf_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TILE 16

static int ceil_div(int a, int b) { return (a + b - 1) / b; }

/* ---- Tile_create: src/csr2block.h:267-422 (steps 1-4 at 6-265) ---------- */

typedef struct { int jc; int src; } orc_pair;

static int pair_cmp(const void *a, const void *b)
{
    const orc_pair *x = (const orc_pair *)a, *y = (const orc_pair *)b;
    if (x->jc != y->jc) return x->jc < y->jc ? -1 : 1;
    return (x->src > y->src) - (x->src < y->src);
}

void orc_tiles_free(orc_tiles *t)
{
    free(t->tile_ptr); free(t->tile_columnidx); free(t->tile_nnz); free(t->blknnz);
    free(t->blknnznnz); free(t->csr_offset); free(t->csrptr_offset); free(t->Blockcsr_Val);
    free(t->Blockcsr_Val_Low); free(t->Tile_csr_Col); free(t->Blockcsr_Ptr);
    memset(t, 0, sizeof(*t));
}

/* Returns 0 on success, -1 on an out-of-range column index. */
int orc_tile_create(int rowA, int colA, const int *rowptr, const int *colidx,
                    const double *val, const float *val_low, orc_tiles *out)
{
    memset(out, 0, sizeof(*out));
    int tilem = ceil_div(rowA, TILE), tilen = ceil_div(colA, TILE);
    out->tilem = tilem; out->tilen = tilen;
    int nnz_used = rowA > 0 ? rowptr[rowA] - rowptr[0] : 0;
    for (int k = rowptr[0]; k < rowptr[0] + nnz_used; k++)
        if (colidx[k] < 0 || colidx[k] >= colA) return -1;

    /* step 1 (csr2block.h:6-41): distinct tile columns per tile-row */
    out->tile_ptr = (int *)calloc(tilem + 1, sizeof(int));
    int maxrow = 0;
    for (int bi = 0; bi < tilem; bi++) {
        int s = bi * TILE, e = (bi == tilem - 1) ? rowA : (bi + 1) * TILE;
        if (rowptr[e] - rowptr[s] > maxrow) maxrow = rowptr[e] - rowptr[s];
    }
    orc_pair *pairs = (orc_pair *)malloc((size_t)(maxrow > 0 ? maxrow : 1) * sizeof(orc_pair));
    for (int bi = 0; bi < tilem; bi++) {
        int s = bi * TILE, e = (bi == tilem - 1) ? rowA : (bi + 1) * TILE;
        int m = 0;
        for (int k = rowptr[s]; k < rowptr[e]; k++) { pairs[m].jc = colidx[k] / TILE; pairs[m].src = k; m++; }
        qsort(pairs, m, sizeof(orc_pair), pair_cmp);
        int cnt = 0;
        for (int q = 0; q < m; q++) if (q == 0 || pairs[q].jc != pairs[q - 1].jc) cnt++;
        out->tile_ptr[bi] = cnt;
    }
    /* exclusive scan (utils.h:34-49) */
    {
        int run = 0;
        for (int bi = 0; bi <= tilem; bi++) { int v = out->tile_ptr[bi]; out->tile_ptr[bi] = run; run += v; }
    }
    int T = out->tile_ptr[tilem];
    out->tilenum = T;

    /* step 2 (csr2block.h:43-107): tile columns, per-tile nnz, per-row u8 counts */
    out->tile_columnidx = (int *)calloc(T > 0 ? T : 1, sizeof(int));
    out->tile_nnz = (int *)calloc(T + 1, sizeof(int));
    unsigned char *row_cnt = (unsigned char *)calloc((size_t)(T > 0 ? T : 1) * TILE, 1);
    for (int bi = 0; bi < tilem; bi++) {
        int s = bi * TILE, e = (bi == tilem - 1) ? rowA : (bi + 1) * TILE;
        int m = 0;
        for (int k = rowptr[s]; k < rowptr[e]; k++) { pairs[m].jc = colidx[k] / TILE; pairs[m].src = k; m++; }
        qsort(pairs, m, sizeof(orc_pair), pair_cmp);
        int t = out->tile_ptr[bi] - 1;
        for (int q = 0; q < m; q++) {
            if (q == 0 || pairs[q].jc != pairs[q - 1].jc) { t++; out->tile_columnidx[t] = pairs[q].jc; }
            out->tile_nnz[t]++;
        }
        for (int r = s; r < e; r++)
            for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
                int jc = colidx[k] / TILE;
                /* locate tile of jc in this tile-row (linear, as step 4 does) */
                for (int tt = out->tile_ptr[bi]; tt < out->tile_ptr[bi + 1]; tt++)
                    if (out->tile_columnidx[tt] == jc) { row_cnt[(size_t)tt * TILE + (r - s)]++; break; }
            }
    }
    {
        int run = 0;
        for (int i = 0; i <= T; i++) { int v = out->tile_nnz[i]; out->tile_nnz[i] = run; run += v; }
    }

    /* step 3 (csr2block.h:109-150) + scans (csr2block.h:346-376) */
    out->blknnz = (int *)calloc(T + 1, sizeof(int));
    out->blknnznnz = (unsigned char *)calloc(T + 1, 1);
    out->csr_offset = (int *)calloc(T + 1, sizeof(int));
    out->csrptr_offset = (int *)calloc(T + 1, sizeof(int));
    int csrsize = 0, csrptrlen = 0;
    for (int bi = 0; bi < tilem; bi++) {
        int rowlen = (bi == tilem - 1) ? rowA - (tilem - 1) * TILE : TILE;
        for (int t = out->tile_ptr[bi]; t < out->tile_ptr[bi + 1]; t++) {
            int nz = out->tile_nnz[t + 1] - out->tile_nnz[t];
            out->blknnz[t] = nz; out->csr_offset[t] = nz; out->csrptr_offset[t] = rowlen;
            csrsize += nz; csrptrlen += rowlen;
        }
    }
    for (int i = 0; i <= T; i++) out->blknnznnz[i] = (unsigned char)out->blknnz[i];
    {
        int r1 = 0, r2 = 0, r3 = 0;
        for (int i = 0; i <= T; i++) {
            int a = out->blknnz[i], b = out->csr_offset[i], c = out->csrptr_offset[i];
            out->blknnz[i] = r1; out->csr_offset[i] = r2; out->csrptr_offset[i] = r3;
            r1 += a; r2 += b; r3 += c;
        }
    }
    out->csrsize = csrsize; out->csrptrlen = csrptrlen;

    /* step 4 (csr2block.h:152-265): scatter in CSR order, u8 row pointers */
    out->Blockcsr_Val = (double *)calloc(csrsize > 0 ? csrsize : 1, sizeof(double));
    out->Blockcsr_Val_Low = (float *)calloc(csrsize > 0 ? csrsize : 1, sizeof(float));
    out->Tile_csr_Col = (unsigned char *)calloc(csrsize > 0 ? csrsize : 1, 1);
    out->Blockcsr_Ptr = (unsigned char *)calloc(csrptrlen > 0 ? csrptrlen : 1, 1);
    int *fill = (int *)calloc(T > 0 ? T : 1, sizeof(int));
    for (int bi = 0; bi < tilem; bi++) {
        int s = bi * TILE, e = (bi == tilem - 1) ? rowA : (bi + 1) * TILE;
        int rowlen = e - s;
        for (int k = rowptr[s]; k < rowptr[e]; k++) {
            int jc = colidx[k] / TILE;
            for (int t = out->tile_ptr[bi]; t < out->tile_ptr[bi + 1]; t++) {
                if (out->tile_columnidx[t] != jc) continue;
                int dst = out->csr_offset[t] + fill[t]++;
                out->Blockcsr_Val[dst] = val[k];
                out->Blockcsr_Val_Low[dst] = val_low ? val_low[k] : (float)val[k];
                out->Tile_csr_Col[dst] = (unsigned char)(colidx[k] - jc * TILE);
                break;
            }
        }
        for (int t = out->tile_ptr[bi]; t < out->tile_ptr[bi + 1]; t++) {
            /* exclusive_scan_char over rowlen entries (utils.h:50-65) */
            unsigned char run = 0;
            for (int r = 0; r < rowlen; r++) {
                unsigned char v = row_cnt[(size_t)t * TILE + r];
                out->Blockcsr_Ptr[out->csrptr_offset[t] + r] = run;
                run = (unsigned char)(run + v);
            }
        }
    }
    free(fill); free(row_cnt); free(pairs);
    return 0;
}

/* ---- encode / decode: src/encode.h:29-72 -------------------------------- */

void orc_encode(const unsigned char *str, unsigned char *res, int str_len, int offset)
{
    int pairs = str_len / 2;
    for (int p = 0; p < pairs; p++)
        res[offset + p] = (unsigned char)((str[2 * p] << 4) + str[2 * p + 1]);
    if (str_len % 2) res[offset + pairs] = (unsigned char)(str[str_len - 1] << 4);
}

void orc_decode(const unsigned char *str, unsigned char *res, int res_len)
{
    for (int i = 0; i + 1 < res_len; i += 2) {
        res[i] = (unsigned char)((str[i / 2] & 240) >> 4);
        res[i + 1] = (unsigned char)(str[i / 2] & 15);
    }
    if (res_len % 2) res[res_len - 1] = (unsigned char)(str[res_len / 2] >> 4);
}

/* ---- blockspmv_cpu: src/blockspmv_cpu.h:2-112 --------------------------- */

#define PREFETCH_TH 4

int orc_rowblkblock_count(const orc_tiles *t)
{
    int c = 0;
    for (int bi = 0; bi < t->tilem; bi++) {
        int k = t->tile_ptr[bi + 1] - t->tile_ptr[bi];
        c += (k <= PREFETCH_TH) ? 1 : ceil_div(k, PREFETCH_TH);
    }
    return c;
}

void orc_blockspmv(const orc_tiles *t, int rowA, int colA, const unsigned char *cidx,
                   int *ptroffset1, int *ptroffset2, unsigned int *rowidx, int *colstart,
                   int *colstop, const double *x, double *y)
{
    (void)colA;
    int e = 0;
    for (int bi = 0; bi < t->tilem; bi++) {
        int k = t->tile_ptr[bi + 1] - t->tile_ptr[bi];
        if (k <= PREFETCH_TH) { rowidx[e] = (unsigned)bi; colstart[e] = 0; colstop[e] = 0; e++; continue; }
        int parts = ceil_div(k, PREFETCH_TH);
        int len = ceil_div(k, parts);
        for (int p = 0; p < parts; p++) {
            rowidx[e] = (unsigned)bi | 0x80000000u;
            colstart[e] = t->tile_ptr[bi] + p * len;
            colstop[e] = (p == parts - 1) ? t->tile_ptr[bi] + k : t->tile_ptr[bi] + (p + 1) * len;
            e++;
        }
    }
    int valoff = 0, ptroff = 0;
    for (int bi = 0; bi < t->tilem; bi++) {
        int rowlen = (bi == t->tilem - 1) ? rowA - (t->tilem - 1) * TILE : TILE;
        for (int r = 0; r < TILE; r++) y[bi * TILE + r] = 0;
        for (int tt = t->tile_ptr[bi]; tt < t->tile_ptr[bi + 1]; tt++) {
            int xo = t->tile_columnidx[tt] * TILE;
            ptroffset1[tt] = valoff; ptroffset2[tt] = ptroff;
            int nz = t->blknnz[tt + 1] - t->blknnz[tt];
            for (int r = 0; r < rowlen; r++) {
                double sum = 0;
                int stop = (r == rowlen - 1) ? nz : t->Blockcsr_Ptr[ptroff + r + 1];
                for (int k = t->Blockcsr_Ptr[ptroff + r]; k < stop; k++) {
                    int g = valoff + k;
                    int c = (g % 2 == 0) ? (cidx[g / 2] & 240) >> 4 : (cidx[g / 2] & 15);
                    double prod = x[xo + c] * t->Blockcsr_Val[g];
                    sum = sum + prod;
                }
                y[bi * TILE + r] = y[bi * TILE + r] + sum;
            }
            valoff += nz; ptroff += rowlen;
        }
    }
}

void orc_tiled_spmv(const orc_tiles *t, int rowA, const double *x, double *y)
{
    for (int bi = 0; bi < t->tilem; bi++) {
        int rowlen = (bi == t->tilem - 1) ? rowA - (t->tilem - 1) * TILE : TILE;
        for (int r = 0; r < rowlen; r++) y[bi * TILE + r] = 0;
        for (int tt = t->tile_ptr[bi]; tt < t->tile_ptr[bi + 1]; tt++) {
            int xo = t->tile_columnidx[tt] * TILE;
            int off = t->tile_nnz[tt], nz = t->tile_nnz[tt + 1] - off, po = t->csrptr_offset[tt];
            for (int r = 0; r < rowlen; r++) {
                double sum = 0;
                int stop = (r == rowlen - 1) ? nz : t->Blockcsr_Ptr[po + r + 1];
                for (int k = t->Blockcsr_Ptr[po + r]; k < stop; k++) {
                    double prod = x[xo + t->Tile_csr_Col[off + k]] * t->Blockcsr_Val[off + k];
                    sum = sum + prod;
                }
                y[bi * TILE + r] = y[bi * TILE + r] + sum;
            }
        }
    }
}

/* ---- non-empty-row compaction: src/main-cg.cu:1231-1288 ----------------- */

static int row_stop(const orc_tiles *t, int tt, int r, int rowlen)
{
    int po = t->csrptr_offset[tt];
    return (r == rowlen - 1) ? (t->blknnz[tt + 1] - t->blknnz[tt]) : t->Blockcsr_Ptr[po + r + 1];
}

int orc_nonzero_rows_count(const orc_tiles *t, int rowA)
{
    int c = 0;
    for (int bi = 0; bi < t->tilem; bi++) {
        int rowlen = (bi == t->tilem - 1) ? rowA - (t->tilem - 1) * TILE : TILE;
        for (int tt = t->tile_ptr[bi]; tt < t->tile_ptr[bi + 1]; tt++) {
            c += 1;
            for (int r = 0; r < rowlen; r++)
                if (row_stop(t, tt, r, rowlen) != t->Blockcsr_Ptr[t->csrptr_offset[tt] + r]) c++;
        }
    }
    return c;
}

void orc_nonzero_rows(const orc_tiles *t, int rowA, int *nzr, int *tile_rowidx,
                      unsigned char *rowid, unsigned char *ptrnew, int *block_signal)
{
    int T = t->tilenum, run = 0;
    for (int bi = 0; bi < t->tilem; bi++) {
        int rowlen = (bi == t->tilem - 1) ? rowA - (t->tilem - 1) * TILE : TILE;
        block_signal[bi] = t->tile_ptr[bi + 1] - t->tile_ptr[bi];
        for (int tt = t->tile_ptr[bi]; tt < t->tile_ptr[bi + 1]; tt++) {
            tile_rowidx[tt] = bi;
            nzr[tt] = run;
            rowid[run] = 0; ptrnew[run] = 0; run++;
            for (int r = 0; r < rowlen; r++) {
                int stop = row_stop(t, tt, r, rowlen);
                if (stop != t->Blockcsr_Ptr[t->csrptr_offset[tt] + r]) {
                    rowid[run] = (unsigned char)r; ptrnew[run] = (unsigned char)stop; run++;
                }
            }
        }
    }
    nzr[T] = run;
    rowid[run] = 0; ptrnew[run] = 0;
    block_signal[t->tilem] = 0;
}

/* ---- nnz load balancer (cg_solve_inc): src/main-cg.cu:1290-1454 ---------- */

static int balance_count(const int *nz, int T, int budget)
{
    int i = 0, j = T - 1, cnt = 0, index = 1;
    while (i < j) {
        if (nz[i] + cnt < budget) { cnt += nz[i]; i++; } else { i++; index++; cnt = 0; }
        if (nz[j] + cnt < budget) { cnt += nz[j]; j--; } else { j--; index++; cnt = 0; }
    }
    return index;
}

/* Returns 0 on success; -1 where the reference would loop forever (no
 * budget in its list gives fewer than 6912 warps) or return early. */
int orc_balance(const orc_tiles *t, int nnzR, int *index_out, int *budget_out,
                int *bptr, int *row_new, int *idx_new, int *vew32, int *vt32)
{
    int T = t->tilenum;
    int *nz = (int *)malloc((size_t)(T + 1) * sizeof(int));
    int *row = (int *)malloc((size_t)(T + 1) * sizeof(int));
    for (int bi = 0; bi < t->tilem; bi++)
        for (int tt = t->tile_ptr[bi]; tt < t->tile_ptr[bi + 1]; tt++) {
            nz[tt] = t->blknnz[tt + 1] - t->blknnz[tt]; row[tt] = bi;
        }
    int list[12] = {16, 32, 64, 96, 128, 256, 512, 1024, 2048, 4096, nnzR / 6912, 0};
    int budget = -1, index = 0;
    for (int k = 0; k < 12; k++) {
        index = balance_count(nz, T, list[k]);
        if (index < 6912) { budget = list[k]; break; }
    }
    if (budget < 0) { free(nz); free(row); return -1; }
    *vew32 = 0; *vt32 = 0;
    if (index < t->tilem) {
        int vew16 = ceil_div(t->tilem, index);
        int tilem32 = ceil_div(t->tilem, 2);
        *vew32 = vew16 * 2;
        *vt32 = (tilem32 / *vew32 / 8) * 8;
    }
    for (int q = 0; q <= index; q++) bptr[q] = 0;
    for (int q = 0; q <= T; q++) { row_new[q] = 0; idx_new[q] = 0; }
    int i = 0, j = T - 1, cnt = 0, step = 0;
    index = 1;
    while (i < j) {
        if (nz[i] + cnt < budget) { cnt += nz[i]; idx_new[step] = i; row_new[step] = row[i]; i++; step++; }
        else { idx_new[step] = i; row_new[step] = row[i]; i++; step++; bptr[index] = step; index++; cnt = 0; }
        if (nz[j] + cnt < budget) { cnt += nz[j]; idx_new[step] = j; row_new[step] = row[j]; j--; step++; }
        else { idx_new[step] = j; row_new[step] = row[j]; j--; step++; bptr[index] = step; index++; cnt = 0; }
        if (i == j) { idx_new[step] = j; row_new[step] = row[j]; step++; bptr[index] = step; }
        if (i > j) { idx_new[step] = j; row_new[step] = row[j]; bptr[index] = step; }
    }
    *index_out = index; *budget_out = budget;
    free(nz); free(row);
    return 0;
}

/* ---- payload casts: src/main-cg-mixed.cu:2325-2342 ---------------------- */

/* IEEE-754 binary32 -> binary16, round to nearest even (the rounding that
 * the reference's (half)(float)v conversion performs). */
uint16_t orc_f32_to_f16_bits(float f)
{
    uint32_t x; memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ex = (x >> 23) & 0xffu, man = x & 0x7fffffu;
    if (ex == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u | (man >> 13) : 0u));
    int e = (int)ex - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t m = man | 0x800000u;
        int shift = 14 - e;
        uint32_t q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (q & 1u))) q++;
        return (uint16_t)(sign | q);
    }
    uint32_t q = man >> 13, rem = man & 0x1fffu;
    uint32_t h = sign | ((uint32_t)e << 10) | q;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) h++;
    return (uint16_t)h;
}

float orc_f16_bits_to_f32(uint16_t h)
{
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16, ex = (h >> 10) & 0x1fu, man = h & 0x3ffu, x;
    if (ex == 0) {
        if (man == 0) x = sign;
        else { float v = (float)man * 0x1p-24f; memcpy(&x, &v, 4); x |= sign; }
    } else if (ex == 31) x = sign | 0x7f800000u | (man << 13);
    else x = sign | ((ex - 15 + 127) << 23) | (man << 13);
    float f; memcpy(&f, &x, 4); return f;
}

void orc_payload_casts(const double *v, int n, float *f32, uint16_t *f16, int8_t *i8)
{
    for (int i = 0; i < n; i++) {
        float f = (float)v[i];
        if (f32) f32[i] = f;
        if (f16) f16[i] = orc_f32_to_f16_bits(f);
        if (i8) {
            /* (int8_t)v as compiled for x86-64: truncate toward zero to a
             * 32-bit integer, keep the low byte (two's complement). */
            double tv = trunc(v[i]);
            int32_t w = (tv >= 2147483648.0 || tv < -2147483648.0 || tv != tv) ? INT32_MIN : (int32_t)tv;
            i8[i] = (int8_t)(uint8_t)(uint32_t)w;
        }
    }
}

/* Race-free restatement of the per-segment rule of
 * src/main-cg-mixed.cu:415-460: the most precise class demanded by any
 * element of the segment wins, i.e. the class follows the largest |dp|.
 * Codes follow the reference: 0 fp64, 4 fp32, 3 fp16, 2 int8, 1 bypass. */
int orc_rule_class(double v)
{
    if (v > 1e-5) return 0;
    if (v > 1e-6) return 4;
    if (v > 1e-7) return 3;
    if (v > 1e-8) return 2;
    return 1;
}

/* The rule's per-tile decision and working class for FP32 directions
 * pn / po (n entries), as the library computes them: scaled = 0 takes the
 * reference's absolute thresholds on v = max_seg |pn - po| in FP64
 * (src/main-cg-mixed.cu:415-460, most precise demand wins), scaled = 1 the
 * same thresholds (without the FP64 class) on max_seg |pn - po| / max |pn|
 * in FP32.  A tile takes its column segment's decision; the working class
 * maps FP64 / FP32 decisions to FP32, FP16 to FP16, INT8 to INT8 on integer
 * tiles (static class INT8) and FP16 otherwise, BYPASS to BYPASS under the
 * scaled rule and like INT8 under the absolute one, and keeps a narrower
 * exact static class (INT8, FP16); an inexact tile whose FP16 payload is not
 * finite (bit 0 of f16ok[t] clear; NULL: all finite) runs FP16 in FP32. */
void orc_rule_tiles(int n, int tilen, int T, const int *tile_col, const unsigned char *static_cls,
                    const unsigned char *f16ok, const float *pn, const float *po, int scaled, unsigned char *decision,
                    unsigned char *working)
{
    int *seg = (int *)malloc(sizeof(int) * (tilen > 0 ? tilen : 1));
    float pmax = 0.f;
    for (int j = 0; j < n; j++) {
        float a = fabsf(pn[j]);
        if (a > pmax) pmax = a;
    }
    for (int s = 0; s < tilen; s++) {
        if (!scaled) {
            double v = 0.0;
            for (int j = s * 16; j < s * 16 + 16 && j < n; j++) {
                double d = fabs((double)pn[j] - (double)po[j]);
                if (d > v) v = d;
            }
            seg[s] = orc_rule_class(v);
        } else {
            float dp = 0.f;
            for (int j = s * 16; j < s * 16 + 16 && j < n; j++) {
                float d = fabsf(pn[j] - po[j]);
                if (d > dp) dp = d;
            }
            float v = pmax > 0.f ? dp / pmax : 0.f;
            seg[s] = v > 1e-6f ? 4 : v > 1e-7f ? 3 : v > 1e-8f ? 2 : 1;
        }
    }
    for (int t = 0; t < T; t++) {
        int d = seg[tile_col[t]], c = static_cls[t], w;
        if (d == 0 || d == 4) w = 4;
        else if (d == 3) w = 3;
        else if (d == 2 || !scaled) w = (c == 2) ? 2 : 3;  /* absolute rule: BYPASS runs as INT8 */
        else w = 1;
        if (w == 4 && (c == 3 || c == 2)) w = c;
        if (w == 3 && c == 2) w = c;
        if (w == 3 && c != 3 && f16ok && !(f16ok[t] & 1)) w = 4;
        decision[t] = (unsigned char)d;
        working[t] = (unsigned char)w;
    }
    free(seg);
}

/* ---- batched solver: storage and the chunk policy ------------------------- */

/* IEEE binary16 bits of a double, rounded to nearest even directly from the
 * double (no intermediate float rounding). */
uint16_t orc_f64_to_f16_bits(double v)
{
    uint64_t x; memcpy(&x, &v, 8);
    uint16_t sign = (uint16_t)((x >> 48) & 0x8000u);
    int ex = (int)((x >> 52) & 0x7ffu);
    uint64_t man = x & 0xfffffffffffffull;
    if (ex == 0x7ff) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u : 0u));
    if (ex == 0 && man == 0) return sign;
    int e = ex - 1023;                      /* unbiased exponent (normal doubles) */
    uint64_t m = man | (1ull << 52);        /* 53-bit significand */
    if (ex == 0) return sign;               /* double subnormals are far below half's range */
    if (e > 15) return (uint16_t)(sign | 0x7c00u);
    int shift;                              /* bits dropped from the 53-bit significand */
    uint32_t base;
    if (e >= -14) { shift = 42; base = (uint32_t)(e + 15) << 10; }
    else { shift = 42 + (-14 - e); base = 0; if (shift > 63) return sign; }
    uint64_t q = m >> shift, rem = m & ((1ull << shift) - 1ull), half = 1ull << (shift - 1);
    if (e >= -14) q &= 0x3ffu;              /* implicit bit lives in the exponent field */
    uint32_t h = base + (uint32_t)q;
    if (rem > half || (rem == half && (h & 1u))) h++;   /* carries into the exponent as IEEE does */
    return (uint16_t)(sign | h);
}

/* Per row of one system (CSR rp/ci/val, n rows): the FP16 copy of the
 * off-diagonal values scaled by 2^-e (e = exponent of the row's largest
 * off-diagonal magnitude - 14; diagonal entries 0), the row scale 2^e as a
 * float (0 when e leaves FP32's normal range or the diagonal is not finite
 * within FP32), the FP32 diagonal (sum of the row's diagonal entries), and
 * the flag bit 0 = every value exact in that storage, bit 1 = FP16-capable;
 * rowstat[4] per row: max |a| (diagonal included), min nonzero |a|,
 * S / max(a_ii - S, 1e-30 S) with S the off-diagonal |a| sum, and the
 * off-diagonal max / min (1 without off-diagonals). */
void orc_batch_rows(int n, const int *rp, const int *ci, const double *val, uint16_t *val16, float *rscale,
                    float *diag32, unsigned char *flag, float *rowstat)
{
    for (int i = 0; i < n; i++) {
        double offmax = 0.0, offmin = 0.0, S = 0.0, d = 0.0, amin = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            double v = val[k], av = fabs(v);
            if (av > 0.0 && (amin == 0.0 || av < amin)) amin = av;
            if (ci[k] == i) d += v;
            else {
                S += av;
                if (av > offmax) offmax = av;
                if (av > 0.0 && (offmin == 0.0 || av < offmin)) offmin = av;
            }
        }
        int e = offmax > 0.0 ? ilogb(offmax) - 14 : 0;
        int ok = e >= -126 && e <= 127 && isfinite(d) && fabs(d) <= 3.0e38;
        int exact = ok && (double)(float)d == d;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            uint16_t h = 0;
            if (ok && ci[k] != i) {
                h = orc_f64_to_f16_bits(ldexp(val[k], -e));
                if ((double)orc_f16_bits_to_f32(h) * ldexp(1.0, e) != val[k]) exact = 0;
            }
            val16[k] = h;
        }
        rscale[i] = ok ? ldexpf(1.f, e) : 0.f;
        diag32[i] = (float)d;
        double margin = d - S;
        double lo = 1e-30 * (S > 1e-300 ? S : 1e-300);
        rowstat[4 * i + 0] = (float)(offmax > fabs(d) ? offmax : fabs(d));
        rowstat[4 * i + 1] = (float)amin;
        rowstat[4 * i + 2] = (float)(S / (margin > lo ? margin : lo));
        rowstat[4 * i + 3] = offmin > 0.0 ? (float)(offmax / offmin) : 1.f;
        flag[i] = (unsigned char)((exact ? 1 : 0) | (ok ? 2 : 0));
    }
}

static float slog10f(float v) { return log10f(v > 1e-30f ? v : 1e-30f); }

/* The network: one unit at a time from its bias, products added in input
 * order with fused multiply-adds (FP32). */
void orc_pn_forward(const float *w, const float *x, float *out)
{
    float h1[32], h2[32];
    for (int j = 0; j < 32; j++) {
        float s = w[512 + j];
        for (int k = 0; k < 16; k++) s = fmaf(w[j * 16 + k], x[k], s);
        h1[j] = s > 0.f ? s : 0.f;
    }
    for (int j = 0; j < 32; j++) {
        float s = w[1568 + j];
        for (int k = 0; k < 32; k++) s = fmaf(w[544 + j * 32 + k], h1[k], s);
        h2[j] = s > 0.f ? s : 0.f;
    }
    for (int o = 0; o < 4; o++) {
        float s = w[1728 + o];
        for (int k = 0; k < 32; k++) s = fmaf(w[1600 + o * 32 + k], h2[k], s);
        out[o] = s;
    }
}

/* The chunk policy of the batched solver on one system: static chunk
 * features from the rows (chunk c = rows [crow[c], crow[c+1]), entries
 * [cent[c], cent[c+1])), checkpoint features from r, pn, po, q, relres and
 * refs (history from prev[4 * c] when have_prev, else the current ones;
 * prev receives the current features 6-9), the network with weights w, and
 * the class: 1 (FP16) when P(label <= 1) >= 0.9 or the chunk is exact in
 * FP16, 0 (FP32) when it is not FP16-capable or otherwise.  feat: 16 floats
 * per chunk.  margin (may be NULL): the decision's distance from its
 * threshold, (e0 + e1) / z - 0.9. */
void orc_batch_classify(int n, const int *rp, const int *ci, const double *val, int nch, const int *crow,
                        const int *cent, const double *r, const double *pn, const double *po, const double *q,
                        double relres, int refs, int have_prev, float *prev, const float *w, float *feat,
                        unsigned char *cls, double *margin)
{
    uint16_t *v16 = (uint16_t *)malloc(sizeof(uint16_t) * (rp[n] > 0 ? rp[n] : 1));
    float *rs = (float *)malloc(sizeof(float) * (n + 1)), *d32 = (float *)malloc(sizeof(float) * (n + 1));
    float *rst = (float *)malloc(sizeof(float) * 4 * (n + 1));
    unsigned char *fl = (unsigned char *)malloc((size_t)n + 1);
    orc_batch_rows(n, rp, ci, val, v16, rs, d32, fl, rst);
    float gr = 0.f, gp = 0.f;
    float *mx = (float *)malloc(sizeof(float) * 4 * (nch + 1));
    for (int c = 0; c < nch; c++) {
        float mr = 0.f, mp = 0.f, mdp = 0.f, mq = 0.f;
        for (int i = crow[c]; i < crow[c + 1]; i++) {
            float a;
            a = (float)fabs(r[i]); if (a > mr) mr = a;
            a = (float)fabs(pn[i]); if (a > mp) mp = a;
            a = (float)fabs(pn[i] - po[i]); if (a > mdp) mdp = a;
            a = (float)fabs(q[i]); if (a > mq) mq = a;
        }
        mx[4 * c] = mr; mx[4 * c + 1] = mp; mx[4 * c + 2] = mdp; mx[4 * c + 3] = mq;
        if (mr > gr) gr = mr;
        if (mp > gp) gp = mp;
    }
    for (int c = 0; c < nch; c++) {
        float amax = 0.f, amin = 3e38f, dd = 0.f, rng = 1.f;
        unsigned fg = 3u;
        for (int i = crow[c]; i < crow[c + 1]; i++) {
            const float *s = rst + 4 * i;
            if (s[0] > amax) amax = s[0];
            if (s[1] > 0.f && s[1] < amin) amin = s[1];
            if (s[2] > dd) dd = s[2];
            if (s[3] > rng) rng = s[3];
            fg &= fl[i];
        }
        float *x = feat + 16 * (size_t)c;
        const float *d = mx + 4 * c;
        x[0] = slog10f(amax) * 0.1f;
        x[1] = slog10f(amin < 3e38f ? amin : 0.f) * 0.1f;
        x[2] = (float)(cent[c + 1] - cent[c]) * (1.f / 2048.f);
        x[3] = slog10f(dd) * 0.1f;
        x[4] = slog10f(rng) * 0.1f;
        x[5] = slog10f((float)relres) * 0.1f;
        x[6] = slog10f(gr > 0.f ? d[0] / gr : 0.f) * 0.1f;
        x[7] = slog10f(gp > 0.f ? d[1] / gp : 0.f) * 0.1f;
        x[8] = slog10f(d[1] > 0.f ? d[2] / d[1] : 0.f) * 0.1f;
        x[9] = slog10f(d[1] > 0.f && amax > 0.f ? d[3] / (d[1] * amax) : 0.f) * 0.1f;
        for (int k = 0; k < 4; k++) x[10 + k] = have_prev ? prev[4 * c + k] : x[6 + k];
        x[14] = (float)refs * (1.f / 16.f);
        x[15] = 1.f;
        for (int k = 0; k < 4; k++) prev[4 * c + k] = x[6 + k];
        float o[4];
        orc_pn_forward(w, x, o);
        float m = o[0];
        for (int k = 1; k < 4; k++) if (o[k] > m) m = o[k];
        float e[4], z = 0.f;
        for (int k = 0; k < 4; k++) { e[k] = expf(o[k] - m); z += e[k]; }
        int c16 = (e[0] + e[1] >= 0.9f * z) ? 1 : 0;
        if (fg & 1u) c16 = 1;
        if (!(fg & 2u)) c16 = 0;
        cls[c] = (unsigned char)c16;
        if (margin) margin[c] = (double)(e[0] + e[1]) / (double)z - 0.9;
    }
    free(mx); free(v16); free(rs); free(d32); free(rst); free(fl);
}

/* ---- the batched configuration's generator --------------------------------- */

/* A C restatement of the library's seeded random SPD generator (SplitMix64
 * counter streams; the written definition the Python mirror also follows),
 * so that the CPU baseline builds its systems without the product library.
 * Row i draws k_i = 8 + floor(25 U) columns uniform in [0, n) (self
 * references dropped) with values N(0,1) 10^U[-4,4] / 2, mirrored; duplicates
 * summed in draw order; diagonal = row |sum| + 1.  Arrays malloc'd (free
 * with orc_free). */
#define ORC_GAMMA 0x9E3779B97F4A7C15ull

static uint64_t orc_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t orc_key(uint64_t seed, uint64_t stream) { return orc_mix64(seed * ORC_GAMMA ^ orc_mix64(stream + ORC_GAMMA)); }
static double orc_u01(uint64_t key, uint64_t i) { return (double)(orc_mix64(key + (i + 1) * ORC_GAMMA) >> 11) * 0x1.0p-53; }
static double orc_normal01(uint64_t key, uint64_t m)
{
    double a = orc_u01(key, 2 * m), b = orc_u01(key, 2 * m + 1);
    return sqrt(-2.0 * log(1.0 - a)) * cos(6.283185307179586 * b);
}

int orc_random_spd_size(uint64_t seed)
{
    double u = orc_u01(orc_key(seed, 3), 0);
    return (int)llround(exp(log(1000.0) + u * (log(64000.0) - log(1000.0))));
}

void orc_xstar(uint64_t seed, int n, double *out)
{
    uint64_t k = orc_key(seed, 1);
    for (int i = 0; i < n; i++) out[i] = -1.0 + 2.0 * orc_u01(k, i);
}

typedef struct { long long key, ord; double v; } orc_trip;

static int orc_trip_cmp(const void *pa, const void *pb)
{
    const orc_trip *a = (const orc_trip *)pa, *b = (const orc_trip *)pb;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->ord < b->ord ? -1 : (a->ord > b->ord ? 1 : 0);
}

int orc_random_spd(uint64_t seed, int n, int *nnz_out, int **rowptr, int **colidx, double **val)
{
    if (n <= 0) n = orc_random_spd_size(seed);
    uint64_t kl = orc_key(seed, 4), ks = orc_key(seed, 2), kc = orc_key(seed, 5), kv = orc_key(seed, 6);
    size_t cap = (size_t)n * 66 + 16, nt = 0;
    orc_trip *tr = (orc_trip *)malloc(sizeof(orc_trip) * cap);
    long long ord = 0;
    for (int i = 0; i < n; i++) {
        int k = 8 + (int)floor(25.0 * orc_u01(kl, i));
        double sc = pow(10.0, -4.0 + 8.0 * orc_u01(ks, i));
        for (int e = 0; e < k; e++) {
            int j = (int)floor(orc_u01(kc, (uint64_t)i * 32 + e) * n);
            if (j >= n) j = n - 1;
            if (j == i) continue;
            double a = orc_normal01(kv, (uint64_t)i * 32 + e) * sc * 0.5;
            tr[nt].key = (long long)i * n + j; tr[nt].ord = ord++; tr[nt].v = a; nt++;
            tr[nt].key = (long long)j * n + i; tr[nt].ord = ord++; tr[nt].v = a; nt++;
        }
    }
    qsort(tr, nt, sizeof(orc_trip), orc_trip_cmp);
    size_t nk = 0;
    for (size_t q = 0; q < nt; q++) {
        if (nk > 0 && tr[nk - 1].key == tr[q].key) tr[nk - 1].v += tr[q].v;
        else tr[nk++] = tr[q];
    }
    double *rowabs = (double *)calloc((size_t)n, sizeof(double));
    for (size_t q = 0; q < nk; q++) rowabs[tr[q].key / n] += fabs(tr[q].v);
    int *rp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    int *ci = (int *)malloc(sizeof(int) * (nk + (size_t)n + 1));
    double *v = (double *)malloc(sizeof(double) * (nk + (size_t)n + 1));
    size_t q = 0, z = 0;
    rp[0] = 0;
    for (int i = 0; i < n; i++) {
        int diag_done = 0;
        while (q < nk && tr[q].key / n == i) {
            int j = (int)(tr[q].key % n);
            if (!diag_done && j > i) { ci[z] = i; v[z] = rowabs[i] + 1.0; z++; diag_done = 1; }
            ci[z] = j; v[z] = tr[q].v; z++;
            q++;
        }
        if (!diag_done) { ci[z] = i; v[z] = rowabs[i] + 1.0; z++; }
        rp[i + 1] = (int)z;
    }
    free(tr);
    free(rowabs);
    *nnz_out = (int)z;
    *rowptr = rp;
    *colidx = ci;
    *val = v;
    return n;
}

void orc_free(void *p) { free(p); }

/* ---- FP64 solvers (textbook order) --------------------------------------- */

void orc_csr_spmv(int n, const int *rp, const int *ci, const double *v, const double *x, double *y)
{
    for (int i = 0; i < n; i++) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) { double p = v[k] * x[ci[k]]; s = s + p; }
        y[i] = s;
    }
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0;
    for (int i = 0; i < n; i++) { double p = a[i] * b[i]; s = s + p; }
    return s;
}

double orc_true_relres(int n, const int *rp, const int *ci, const double *v, const double *b, const double *x)
{
    double *ax = (double *)malloc((size_t)n * sizeof(double));
    orc_csr_spmv(n, rp, ci, v, x, ax);
    double rr = 0, bb = 0;
    for (int i = 0; i < n; i++) { double d = b[i] - ax[i]; rr += d * d; bb += b[i] * b[i]; }
    free(ax);
    return bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
}

/* Unpreconditioned CG (the algorithm of src/Mille-feuille-cg.h:168-350),
 * x0 = 0, stopping when ||r||/||b|| <= tol (the reference's stopping test
 * is commented out at Mille-feuille-cg.h:232; tol = 0 runs maxiter).
 * Returns the iteration count; hist (optional) gets ||r_k||/||b||. */
int orc_cg(int n, const int *rp, const int *ci, const double *v, const double *b, double *x,
           int maxiter, double tol, double *relres_out, double *hist)
{
    double *r = (double *)malloc((size_t)n * sizeof(double));
    double *p = (double *)malloc((size_t)n * sizeof(double));
    double *q = (double *)malloc((size_t)n * sizeof(double));
    for (int i = 0; i < n; i++) { x[i] = 0; r[i] = b[i]; p[i] = b[i]; }
    double bb = dot(n, b, b), rho = bb;
    double nb = sqrt(bb) > 0 ? sqrt(bb) : 1.0;
    int it = 0;
    if (hist) hist[0] = sqrt(rho) / nb;
    while (it < maxiter && sqrt(rho) / nb > tol) {
        orc_csr_spmv(n, rp, ci, v, p, q);
        double pq = dot(n, p, q);
        double alpha = rho / pq;
        for (int i = 0; i < n; i++) { x[i] = x[i] + alpha * p[i]; r[i] = r[i] - alpha * q[i]; }
        double rho_new = dot(n, r, r);
        double beta = rho_new / rho;
        rho = rho_new;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
        it++;
        if (hist) hist[it] = sqrt(rho) / nb;
    }
    if (relres_out) *relres_out = sqrt(rho) / nb;
    free(r); free(p); free(q);
    return it;
}

/* Unpreconditioned BiCGSTAB (the algorithm of
 * src/Mille-feuille-bicg.h:202-474 with r_hat = r0), x0 = 0. */
int orc_bicgstab(int n, const int *rp, const int *ci, const double *v, const double *b, double *x,
                 int maxiter, double tol, double *relres_out)
{
    size_t sz = (size_t)n * sizeof(double);
    double *r = malloc(sz), *rh = malloc(sz), *p = malloc(sz), *vv = malloc(sz);
    double *s = malloc(sz), *t = malloc(sz);
    for (int i = 0; i < n; i++) { x[i] = 0; r[i] = b[i]; rh[i] = b[i]; p[i] = b[i]; }
    double nb = sqrt(dot(n, b, b)); if (nb == 0) nb = 1;
    double rho = dot(n, rh, r), rr = dot(n, r, r);
    int it = 0;
    while (it < maxiter && sqrt(rr) / nb > tol) {
        orc_csr_spmv(n, rp, ci, v, p, vv);
        double alpha = rho / dot(n, rh, vv);
        for (int i = 0; i < n; i++) s[i] = r[i] - alpha * vv[i];
        orc_csr_spmv(n, rp, ci, v, s, t);
        double tt = dot(n, t, t);
        double omega = tt != 0 ? dot(n, t, s) / tt : 0.0;
        for (int i = 0; i < n; i++) { x[i] = x[i] + alpha * p[i] + omega * s[i]; r[i] = s[i] - omega * t[i]; }
        double rho_new = dot(n, rh, r);
        double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * vv[i]);
        rr = dot(n, r, r);
        it++;
    }
    if (relres_out) *relres_out = sqrt(rr) / nb;
    free(r); free(rh); free(p); free(vv); free(s); free(t);
    return it;
}

/* ---- MLP policy oracle: 16 -> 32 -> 32 -> 4, ReLU, softmax cross-entropy.
 * Weights layout W1[32][16], b1[32], W2[32][32], b2[32], W3[4][32], b3[4]
 * (the learned policy of the library; no reference counterpart).  Returns
 * the mean loss over n samples and its gradient, in double precision. */
double orc_mlp_grad(const float *w, const float *X, const int *Y, int n, double *grad)
{
    enum { NF = 16, H1 = 32, H2 = 32, NO = 4 };
    const int OW1 = 0, OB1 = H1 * NF, OW2 = OB1 + H1, OB2 = OW2 + H2 * H1, OW3 = OB2 + H2, OB3 = OW3 + NO * H2;
    const int NP = OB3 + NO;
    for (int p = 0; p < NP; p++) grad[p] = 0;
    double loss = 0;
    for (int s = 0; s < n; s++) {
        const float *x = X + (size_t)s * NF;
        double h1[H1], h2[H2], o[NO], dl[NO], d2[H2], d1[H1];
        for (int j = 0; j < H1; j++) {
            double a = w[OB1 + j];
            for (int k = 0; k < NF; k++) a += (double)w[OW1 + j * NF + k] * x[k];
            h1[j] = a > 0 ? a : 0;
        }
        for (int j = 0; j < H2; j++) {
            double a = w[OB2 + j];
            for (int k = 0; k < H1; k++) a += (double)w[OW2 + j * H1 + k] * h1[k];
            h2[j] = a > 0 ? a : 0;
        }
        double mx = -1e300;
        for (int o_ = 0; o_ < NO; o_++) {
            double a = w[OB3 + o_];
            for (int k = 0; k < H2; k++) a += (double)w[OW3 + o_ * H2 + k] * h2[k];
            o[o_] = a;
            if (a > mx) mx = a;
        }
        double z = 0;
        for (int k = 0; k < NO; k++) z += exp(o[k] - mx);
        const int y = Y[s] & 3;
        loss += -(o[y] - mx - log(z));
        for (int k = 0; k < NO; k++) dl[k] = (exp(o[k] - mx) / z - (k == y ? 1.0 : 0.0)) / n;
        for (int j = 0; j < H2; j++) {
            double a = 0;
            for (int k = 0; k < NO; k++) a += (double)w[OW3 + k * H2 + j] * dl[k];
            d2[j] = h2[j] > 0 ? a : 0;
        }
        for (int j = 0; j < H1; j++) {
            double a = 0;
            for (int k = 0; k < H2; k++) a += (double)w[OW2 + k * H1 + j] * d2[k];
            d1[j] = h1[j] > 0 ? a : 0;
        }
        for (int j = 0; j < H1; j++) {
            for (int k = 0; k < NF; k++) grad[OW1 + j * NF + k] += d1[j] * x[k];
            grad[OB1 + j] += d1[j];
        }
        for (int j = 0; j < H2; j++) {
            for (int k = 0; k < H1; k++) grad[OW2 + j * H1 + k] += d2[j] * h1[k];
            grad[OB2 + j] += d2[j];
        }
        for (int o_ = 0; o_ < NO; o_++) {
            for (int k = 0; k < H2; k++) grad[OW3 + o_ * H2 + k] += dl[o_] * h2[k];
            grad[OB3 + o_] += dl[o_];
        }
    }
    return loss / n;
}
