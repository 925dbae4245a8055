// mtx_device.cu -- a Matrix Market file straight to a device-resident tiled
// matrix: the entries are parsed on the host threads (mtx_read_coo, the
// reference reader's semantics, src/biio2.0/src/mmio_highlevel.h:151-321),
// and the CSR is built on the GPU.
//
// The reference reader's CSR keeps each row's entries in file order, a
// symmetric file's mirrored entry (j, i) placed when (i, j) is read.  On the
// GPU: the entries become an event list in that order (entry k at
// k + mirrors before k, its mirror right after it), a stable radix sort of
// the events by row gives every row's events in event order, and the row
// pointers come from a histogram and an exclusive scan.  The result is the
// host reader's CSR bit for bit, handed to the tile build on the device.
#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include "mf_internal.h"

namespace mf {
mf_status mtx_read_coo(const char *path, long long &M, long long &N, long long &NZ, bool &sym, std::vector<int> &ri,
                       std::vector<int> &ci, std::vector<double> &vv);

namespace {

constexpr int MTX_NT = 256;

int mtx_grid(long long work)
{
    long long g = (work + MTX_NT - 1) / MTX_NT;
    return (int)(g < 1 ? 1 : g > 148 * 32 ? 148 * 32 : g);
}

// 1 for an entry that has a mirror (symmetric file, off the diagonal)
__global__ void k_mirror_flags(long long nz, int sym, const int *__restrict__ ri, const int *__restrict__ ci,
                               int *__restrict__ flag)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nz; k += (long long)gridDim.x * blockDim.x)
        flag[k] = (sym && ri[k] != ci[k]) ? 1 : 0;
}

// Event list: entry k at k + mirrors[k] (exclusive scan of the flags), its
// mirror at the next position; the key is the event's row, the payload its
// position.
__global__ void k_events(long long nz, const int *__restrict__ ri, const int *__restrict__ ci,
                         const int *__restrict__ flag, const int *__restrict__ before, int *__restrict__ key,
                         int *__restrict__ pos, int *__restrict__ row_count)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nz; k += (long long)gridDim.x * blockDim.x) {
        const long long e = k + before[k];
        key[e] = ri[k];
        pos[e] = (int)e;
        atomicAdd(&row_count[ri[k]], 1);
        if (flag[k]) {
            key[e + 1] = ci[k];
            pos[e + 1] = (int)(e + 1);
            atomicAdd(&row_count[ci[k]], 1);
        }
    }
}

// CSR entry o takes event pos[o]: an entry's column and value, or for a
// mirror the entry's row as the column.
__global__ void k_gather(long long ne, const int *__restrict__ ri, const int *__restrict__ ci,
                         const double *__restrict__ vv, const int *__restrict__ before,
                         const int *__restrict__ sorted_pos, const int *__restrict__ ev_entry,
                         int *__restrict__ col, double *__restrict__ val)
{
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < ne; o += (long long)gridDim.x * blockDim.x) {
        const int e = sorted_pos[o];
        const int k = ev_entry[e];
        const bool mirror = e != k + before[k];
        col[o] = mirror ? ri[k] : ci[k];
        val[o] = vv[k];
    }
}

// ev_entry[e]: the entry whose event e is (entry k owns events k + before[k]
// and, with a mirror, the next one)
__global__ void k_event_owner(long long nz, const int *__restrict__ flag, const int *__restrict__ before,
                              int *__restrict__ ev_entry)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nz; k += (long long)gridDim.x * blockDim.x) {
        const long long e = k + before[k];
        ev_entry[e] = (int)k;
        if (flag[k]) ev_entry[e + 1] = (int)k;
    }
}

int key_bits(long long rows)
{
    int b = 1;
    while (b < 31 && (1ll << b) < rows) b++;
    return b;
}

}  // namespace
}  // namespace mf

using namespace mf;

// Stream-ordered temporaries of one call, released on every return.
struct MtxBufs {
    cudaStream_t s;
    std::vector<void *> v;
    template <typename T>
    cudaError_t get(T **p, long long count)
    {
        void *q = nullptr;
        cudaError_t e = pool_malloc_async(&q, sizeof(T) * (size_t)(count + 1) + 16, s);
        if (e == cudaSuccess) v.push_back(q);
        *p = (T *)q;
        return e;
    }
    ~MtxBufs()
    {
        cudaStreamSynchronize(s);
        for (void *q : v) cudaFreeAsync(q, s);
    }
};

extern "C" mf_status mf_matrix_create_mtx(const char *path, void *stream, mf_matrix *out, int *is_symmetric)
{
    if (!path || !out) {
        set_last_error("mf_matrix_create_mtx: null argument");
        return MF_ERR_INVALID_ARG;
    }
    *out = nullptr;
    long long M, N, NZ;
    bool sym = false;
    std::vector<int> ri, ci;
    std::vector<double> vv;
    MF_TRY(mtx_read_coo(path, M, N, NZ, sym, ri, ci, vv));
    if (NZ > 0x3fffffff) {
        set_last_error("%s: more than 2^30 file entries", path);
        return MF_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MtxBufs B{s, {}};
    const long long nz = NZ;
    int *d_ri, *d_ci, *d_flag, *d_before;
    double *d_vv;
    MF_CUDA(B.get(&d_ri, nz));
    MF_CUDA(B.get(&d_ci, nz));
    MF_CUDA(B.get(&d_vv, nz));
    MF_CUDA(B.get(&d_flag, nz));
    MF_CUDA(B.get(&d_before, nz));
    if (nz > 0) {
        MF_CUDA(cudaMemcpyAsync(d_ri, ri.data(), sizeof(int) * nz, cudaMemcpyHostToDevice, s));
        MF_CUDA(cudaMemcpyAsync(d_ci, ci.data(), sizeof(int) * nz, cudaMemcpyHostToDevice, s));
        MF_CUDA(cudaMemcpyAsync(d_vv, vv.data(), sizeof(double) * nz, cudaMemcpyHostToDevice, s));
        k_mirror_flags<<<mtx_grid(nz), MTX_NT, 0, s>>>(nz, sym ? 1 : 0, d_ri, d_ci, d_flag);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    int mirrors = 0;
    MF_TRY(exclusive_scan_i32(d_flag, d_before, (int)nz, s, &mirrors));
    const long long ne = nz + mirrors;
    if (ne > 0x7fffffff) {
        set_last_error("%s: more than 2^31-1 entries", path);
        return MF_ERR_UNSUPPORTED;
    }
    int *d_key, *d_pos, *d_key2, *d_pos2, *d_owner, *d_cnt, *d_rp, *d_col;
    double *d_val;
    MF_CUDA(B.get(&d_key, ne));
    MF_CUDA(B.get(&d_pos, ne));
    MF_CUDA(B.get(&d_key2, ne));
    MF_CUDA(B.get(&d_pos2, ne));
    MF_CUDA(B.get(&d_owner, ne));
    MF_CUDA(B.get(&d_cnt, M));
    MF_CUDA(B.get(&d_rp, M));
    MF_CUDA(B.get(&d_col, ne));
    MF_CUDA(B.get(&d_val, ne));
    MF_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int) * (M + 1), s));
    if (nz > 0) {
        k_events<<<mtx_grid(nz), MTX_NT, 0, s>>>(nz, d_ri, d_ci, d_flag, d_before, d_key, d_pos, d_cnt);
        note_launch();
        MF_CUDA(cudaGetLastError());
        k_event_owner<<<mtx_grid(nz), MTX_NT, 0, s>>>(nz, d_flag, d_before, d_owner);
        note_launch();
        MF_CUDA(cudaGetLastError());
        // stable by row: the LSD radix sort keeps the event order within a row
        size_t tmp_bytes = 0;
        MF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_key, d_key2, d_pos, d_pos2, (int)ne, 0,
                                                key_bits(M), s));
        unsigned char *d_tmp;
        MF_CUDA(B.get(&d_tmp, (long long)tmp_bytes));
        MF_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_key, d_key2, d_pos, d_pos2, (int)ne, 0,
                                                key_bits(M), s));
        note_launch(4);
        k_gather<<<mtx_grid(ne), MTX_NT, 0, s>>>(ne, d_ri, d_ci, d_vv, d_before, d_pos2, d_owner, d_col, d_val);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    int total = 0;
    MF_TRY(exclusive_scan_i32(d_cnt, d_rp, (int)M + 1, s, &total));
    mf_matrix m = nullptr;
    MF_TRY(mf_matrix_create((int)M, (int)N, d_rp, d_col, d_val, nullptr, 1, stream, &m));
    *out = m;
    if (is_symmetric) *is_symmetric = sym ? 1 : 0;
    return MF_OK;
}
