// solver.h -- internal interface of the persistent solver kernels.
#pragma once
#include "mf_internal.h"

namespace mf {

// A chunk: up to CH_STRIPS consecutive strips of one CTA whose tiles,
// entries and bytes fit one shared-memory stage.  A strip too large for a
// stage on its own is a one-strip chunk with `direct` set (computed from
// global memory).
#ifndef MF_CHUNK_STRIPS
#define MF_CHUNK_STRIPS 16
#endif
constexpr int CH_STRIPS = MF_CHUNK_STRIPS;
constexpr int CH_TILES = 8 * CH_STRIPS;
constexpr int CH_ENTRIES = 128 * CH_STRIPS;
struct ChunkRec {
    int s0, s1;       // strips [s0, s1)
    int t0, t1;       // tiles [t0, t1)
    int e0, e1;       // entries [e0, e1)
    unsigned y0, y1;  // packed payload bytes [y0, y1) (mixed)
    int direct;
    int pad;
};

// A chunk of the row-slot layout: consecutive strips of one CTA whose slot
// words, values (or mixed payload) and tile columns fit one shared-memory
// stage.  `lanes` half-warps share each strip (1, 2, 4, 8 or 16; a chunk has
// 16 / lanes strips at most): each takes a contiguous part of the strip's
// slots, and the parts' sums are added in order.  A strip too large for a
// stage on its own is a one-strip chunk with `direct` set (16 half-warps,
// read from global memory).
//
// Staged chunks (the CG kernels' default when every chunk qualifies): the
// chunk's tile columns form at most SC_RUNS runs of consecutive tile
// columns holding SC_XCAP columns at most; the runs of the vectors the SpMV
// reads are copied into shared memory next to the slots, and the slot words
// are positions in that staged copy (spos), so no row reads a vector from
// global memory.
constexpr int SC_STRIPS = CH_STRIPS, SC_SLOTS = 8 * SC_STRIPS, SC_TILES = 16 * SC_STRIPS;
constexpr int SC_RUNS = 6, SC_XCAP = 1280;
struct SlotChunk {
    int s0, s1;            // strips [s0, s1)
    int k0, k1;            // slots [k0, k1)
    int t0, t1;            // tiles [t0, t1)
    int direct, lanes;
    long long y0, y1;      // mixed payload bytes [y0, y1)
    int fmt;               // mixed payload: 0 / 1 / 2 every slot fp32 / fp16 / int8, -1 otherwise
    int nrun;              // staged: column runs (-1: the chunk cannot be staged)
    int xlen;              // staged: columns staged (multiple of 16)
    int rg[SC_RUNS];                 // staged: first column of each run (multiple of 16)
    unsigned short rl[SC_RUNS];      // staged: columns of each run (multiple of 16)
    unsigned short rs[SC_RUNS];      // staged: position of each run in the staged vectors
};
static_assert(SC_XCAP < 65536, "staged run lengths and positions are 16-bit");

// Half-warps per strip for a strip of K slots: about 8 slots each.
__host__ __device__ __forceinline__ int slot_lanes(int K)
{
    return K <= 8 ? 1 : K <= 16 ? 2 : K <= 32 ? 4 : K <= 64 ? 8 : 16;
}

// Persistent solver state kept in device memory between launches.
enum : int { S_RHO = 0, S_BETA, S_NB, S_RMAX, S_ITERS, S_REFS, S_EXIT, S_RELRES, S_ALPHA, S_OMEGA, S_RZ, S_COUNT };
// Why a launch returned.
enum : int { EXIT_CONVERGED = 1, EXIT_MAXITER = 2, EXIT_BREAKDOWN = 3, EXIT_CHECKPOINT = 4 };

struct CgArgs {
    MfTiles A;
    const int *part;               // [G+1] strip range of each CTA
    const int *cta_chunk;          // [G+1] chunk range of each CTA
    const ChunkRec *chunks;
    const unsigned char *pay;      // mixed: packed per-tile payload bytes
    const unsigned *poff;          // mixed: [T+1] byte offset of each tile's payload
    const unsigned char *wcls;     // mixed: [T] working class of each tile
    const double *b;
    double *xhi;                   // solution (FP64)
    void *r, *p0, *p1, *q, *xlo;   // vectors (FP64, or FP32 when mixed)
    void *rhat, *v0, *v1, *t;      // BiCGSTAB: shadow residual, A p (double-buffered), A s
    double *partials;              // [8][G] per-CTA dot partials
    unsigned long long *bar;       // sharded grid barrier counters (9 lines, 0 at launch)
    int *status;                   // device status word (mf_status codes)
    double *state;                 // [S_COUNT]
    double *hist;                  // optional per-iteration ||r||/||b||
    int maxiter;
    double tol;
    int fixed;                     // 1: run exactly maxiter iterations
    double delta;                  // reliable-update trigger
    int exit_on_refine;            // 1: return after each reliable update
    int checkpoint_every;          // > 0: return every this many iterations
    unsigned long long budget_ns;  // bound of every grid-wide wait
    int start;                     // 1: initialise x, r, p and the state
    unsigned long long *timing;    // optional [G][8] per-CTA phase nanoseconds
    int last_tile_begin;           // first tile of the last strip
    int last_rowlen;               // rows of the last strip
    // row-slot layout (null when the kernel runs from tile chunks)
    const int *sslot;              // [tilem+1] first slot of each strip
    const uint16_t *smeta;         // [slots*16] tile-in-strip << 4 | in-tile column
    const double *sval;            // [slots*16] FP64 values
    const unsigned *shdr;          // mixed: [slots] payload offset (16 B) << 2 | format
    const unsigned char *spay;     // mixed: slot payload
    const int *scta_chunk;         // [G+1] slot-chunk range of each CTA
    const SlotChunk *schunks;
    int one_reduction;             // FP64: the single-reduction CG kernel (k_cg1)
    // staged slot chunks (null otherwise)
    const uint16_t *spos;          // [slots*16] position in the chunk's staged vectors (0xFFFF empty)
    const int2 *sdesc;             // [tilem] per strip: first slot within its chunk | slots << 16, and
                                   // the offset from a row to its own staged position (INT_MIN: none)
    double *xs;                    // padded FP64 copy of x that the refinement SpMV stages
    // Jacobi-preconditioned CG (null otherwise)
    void *z;                       // z = D^-1 r (solver's vector type)
    const double *dinv;            // [rows] 1 / diagonal (1 where the diagonal is 0)
};

struct SolverWork {
    void *r, *p0, *p1, *q, *xlo, *rhat, *v0, *v1, *t;
    double *ax, *partials, *rpart, *out, *state;
    unsigned long long *timing;
    unsigned long long *bar;
    int *status;
};

mf_status solver_resources(mf_matrix m, int G, SolverWork &w);

// Called at every checkpoint of a solve run with trace collection: the
// solver state (p of the last iteration in p_new, the previous p in p_old,
// q = A p_new, r) is in `w`.
struct TraceHook {
    int every;
    mf_status (*fn)(void *ctx, mf_matrix m, SolverWork &w, const void *p_new, const void *p_old, int it,
                    double relres, cudaStream_t s);
    void *ctx;
};
mf_status cg_solve_traced(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                          const TraceHook *hook, cudaStream_t s);
// chunks.cu: chunk table for the current partition; payload offsets refresh
mf_status build_chunks(mf_matrix m, cudaStream_t s);
mf_status refresh_chunk_payload(mf_matrix m, cudaStream_t s);
int solver_grid(mf_matrix m, bool mixed, int layout);  // layout: 0 tiles, 1 slots, 2 staged slots
mf_status launch_cg(bool mixed, CgArgs &a, int G, cudaStream_t s);
mf_status launch_bicgstab(bool mixed, CgArgs &a, int G, cudaStream_t s);
int bicgstab_grid(mf_matrix m, bool mixed, int layout);  // layout as solver_grid (2: mixed only)
// slots.cu: the row-slot layout (built once; state -1 = not describable)
mf_status build_slots(mf_matrix m, cudaStream_t s);
// multi.cu: k <= 16 right-hand sides, row-interleaved vectors
mf_status spmm_multi(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, cudaStream_t s);
mf_status cg_multi(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx, const mf_solve_opts &o,
                   mf_solve_report *reports, cudaStream_t s);
mf_status pack_slots(mf_matrix m, const unsigned char *d_wcls, cudaStream_t s);
// staged = true builds staged chunks and the positions; m->schunk_staged
// tells whether every chunk qualified (otherwise the chunks are plain)
mf_status build_slot_chunks(mf_matrix m, int G, bool staged, cudaStream_t s);
mf_status true_residual(mf_matrix m, const double *b, const double *x, SolverWork &w, double *relres, cudaStream_t s);
// Jacobi preconditioner: dinv[i] = 1 / a_ii (1 where the diagonal is 0)
mf_status jacobi_dinv(mf_matrix m, double *dinv, cudaStream_t s);
// payload.cu
mf_status pack_payload(mf_matrix m, const unsigned char *d_wcls, cudaStream_t s);
// STATIC classes; range16: MF_POLICY_STATIC_FP16's FP16 class for inexact tiles in binary16's normal range
mf_status static_working_classes(mf_matrix m, unsigned char *d_wcls, cudaStream_t s, bool range16 = false);
mf_status learned_working_classes(mf_matrix m, SolverWork &w, const void *p_new, const void *p_old,
                                  unsigned char *d_wcls, cudaStream_t s);
// RULE / RULE_SCALED classes for the FP32 directions p_new / p_old: the
// per-tile decision (may be null) and the working classes (may be null)
mf_status rule_classes(mf_matrix m, int policy, const void *p_new, const void *p_old, unsigned char *d_decision,
                       unsigned char *d_wcls, cudaStream_t s);

}  // namespace mf
