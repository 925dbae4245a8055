// solver.cu -- host orchestration of the persistent CG solves (policies,
// checkpoints, reports).
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "solver.h"

namespace mf {

static mf_status persistent_solve(bool bicg, mf_matrix m, const double *b, double *x, const mf_solve_opts &o,
                                  mf_solve_report &rep, double *history, cudaStream_t s,
                                  const TraceHook *hook = nullptr)
{
    const bool mixed = o.policy != MF_POLICY_FP64;
    // FP64 CG without checkpoints on small, short-row systems (latency-bound:
    // the grid-wide waits dominate): one reduction per iteration.  Larger or
    // long-row systems keep the two-reduction kernel, whose SpMV gathers two
    // vectors instead of three.  MF_CG_VARIANT=1 / 2 forces either.
    bool one_reduction;
    {
        const char *v = getenv("MF_CG_VARIANT");
        const bool small = m->v.rows <= (1 << 19) && (long long)m->v.nnz <= 16LL * m->v.rows;
        const int force = v ? atoi(v) : 0;
        const bool want = force == 1 || (force != 2 && small);
        one_reduction = !bicg && !mixed && !hook && want && !o.precond;
    }
    // execution layout: staged row slots for the mixed-precision
    // two-reduction CG kernel and the mixed BiCGSTAB kernel, plain row slots
    // otherwise or when a chunk cannot be staged, tile chunks when the slots
    // cannot describe the matrix.  (The FP64 CG kernel stages two FP64
    // vectors, which leaves room for two CTAs per SM only; its plain row
    // slots run faster.)  MF_SOLVER_LAYOUT=tiles / slots restricts the
    // choice, =staged also stages the FP64 CG kernel.
    const char *lay = getenv("MF_SOLVER_LAYOUT");
    const bool want_slots = !(lay && !strcmp(lay, "tiles"));
    if (want_slots) MF_TRY(build_slots(m, s));
    const bool slots = want_slots && m->slots_state == 1;
    const bool force_staged = lay && !strcmp(lay, "staged");
    bool staged = slots && !one_reduction && (bicg ? mixed : (mixed || force_staged)) &&
                  !(lay && !strcmp(lay, "slots")) && (long long)m->v.tilen <= (long long)m->v.tilem;
    auto layout_grid = [&](bool st) {
        const int l = st ? 2 : slots ? 1 : 0;
        return bicg ? bicgstab_grid(m, mixed, l) : solver_grid(m, mixed, l);
    };
    int G = layout_grid(staged);
    auto prepare = [&]() -> mf_status {
        if (m->part_ctas != G || (!slots && !m->d_chunks)) {
            MF_TRY(strip_partition(m, G, s));
            if (!slots) MF_TRY(build_chunks(m, s));
            m->packed_policy = -1;  // chunk payload offsets must be refreshed
        }
        if (slots) MF_TRY(build_slot_chunks(m, G, staged, s));
        return MF_OK;
    };
    MF_TRY(prepare());
    if (getenv("MF_LAYOUT_DEBUG"))
        fprintf(stderr, "mf: layout %s, grid %d, %d chunks, %d not stageable\n",
                staged ? "staged" : slots ? "slots" : "tiles", G, m->nschunks, m->schunk_unstaged);
    if (staged && !m->schunk_staged) {  // some chunk's columns do not fit: plain slots
        staged = false;
        G = layout_grid(false);
        MF_TRY(prepare());
    }
    SolverWork w;
    MF_TRY(solver_resources(m, G, w));
    const int T = m->v.tilenum;
    // repack the payload of the layout in use for the classes in d_wcls
    auto repack = [&](int policy) -> mf_status {
        MF_TRY(pack_payload(m, m->d_wcls, s));  // also counts the algorithmic payload bytes
        if (slots) {
            MF_TRY(pack_slots(m, m->d_wcls, s));
            m->slot_policy = policy;
        } else {
            MF_TRY(refresh_chunk_payload(m, s));
            m->packed_policy = policy;
        }
        return MF_OK;
    };
    // the classes a solve starts from: STATIC_FP16's, or STATIC's for every
    // other mixed policy
    const int base_policy = o.policy == MF_POLICY_STATIC_FP16 ? MF_POLICY_STATIC_FP16 : MF_POLICY_STATIC;
    if (mixed) {
        if (!m->d_wcls) MF_CUDA(cudaMalloc(&m->d_wcls, (size_t)T + 16));
        if ((slots ? m->slot_policy : m->packed_policy) != base_policy) {
            MF_TRY(static_working_classes(m, m->d_wcls, s, base_policy == MF_POLICY_STATIC_FP16));
            MF_TRY(repack(base_policy));
        }
    }
    if (o.policy == MF_POLICY_LEARNED) m->pol_have_prev = 0;  // no history from an earlier solve
    CgArgs a;
    memset(&a, 0, sizeof(a));
    a.A = m->v;
    a.part = m->d_part;
    a.cta_chunk = m->d_cta_chunk;
    a.chunks = (const ChunkRec *)m->d_chunks;
    a.last_tile_begin = m->last_tile_begin;
    a.last_rowlen = m->v.rows - (m->v.tilem - 1) * MF_TILE;
    if (slots) {
        a.sslot = m->d_sslot;
        a.smeta = m->d_smeta;
        a.sval = m->d_sval;
        a.shdr = m->d_shdr;
        a.spay = m->d_spay;
        a.scta_chunk = m->d_scta_chunk;
        a.schunks = (const SlotChunk *)m->d_schunks;
        if (staged) {
            a.spos = m->d_spos;
            a.sdesc = m->d_sdesc;
            // padded to whole strips (tile columns of a square tile grid); a
            // buffer the kernel does not otherwise use (BiCGSTAB uses t)
            a.xs = (double *)(bicg ? w.q : w.t);
        }
    }
    a.pay = m->d_pay;
    a.poff = m->d_poff;
    a.wcls = m->d_wcls;
    a.b = b;
    a.xhi = x;
    a.r = w.r;
    a.p0 = w.p0;
    a.p1 = w.p1;
    a.q = w.q;
    a.xlo = w.xlo;
    a.rhat = w.rhat;
    a.v0 = w.v0;
    a.v1 = w.v1;
    a.t = w.t;
    a.partials = w.partials;
    a.bar = w.bar;
    a.status = w.status;
    a.state = w.state;
    a.hist = (o.record_history && history) ? history : nullptr;
    a.maxiter = o.maxiter;
    a.tol = o.tol;
    a.fixed = o.tol < 0 ? 1 : 0;
    a.delta = o.refine_delta > 0 && o.refine_delta < 1 ? o.refine_delta : 0.1;
    // checkpoints (policy updates between launches) for CG's dynamic policies
    a.exit_on_refine = (!bicg && mixed && o.policy != MF_POLICY_STATIC && o.policy != MF_POLICY_STATIC_FP16) ? 1 : 0;
    a.checkpoint_every = (hook && !bicg) ? hook->every : 0;
    a.one_reduction = (one_reduction && a.checkpoint_every == 0) ? 1 : 0;
    if (!bicg && o.precond == 1) {
        // Jacobi: z in a vector CG does not otherwise use, D^-1 in another
        a.z = w.rhat;
        a.dinv = (const double *)w.v1;
        MF_TRY(jacobi_dinv(m, (double *)w.v1, s));
    }
    a.budget_ns = (unsigned long long)(o.wait_budget_s * 1e9);
    a.start = 1;
    a.timing = o.phase_times ? w.timing : nullptr;
    if (a.timing) MF_CUDA(cudaMemsetAsync(w.timing, 0, sizeof(unsigned long long) * 8 * G, s));
    MF_CUDA(cudaMemsetAsync(w.status, 0, sizeof(int), s));
    cudaEvent_t e0, e1;
    MF_CUDA(cudaEventCreate(&e0));
    MF_CUDA(cudaEventCreate(&e1));
    MF_CUDA(cudaEventRecord(e0, s));
    double st[S_COUNT];
    int h_status = 0, launches = 0;
    // stagnation guard of the dynamic policies: FP64 residual and
    // refinement count at the last reliable update
    double guard_relres = 1.0;
    int guard_refs = 0;
    for (;;) {
        MF_CUDA(cudaMemsetAsync(w.bar, 0, 9 * 128, s));
        if (bicg) MF_TRY(launch_bicgstab(mixed, a, G, s));
        else MF_TRY(launch_cg(mixed, a, G, s));
        launches++;
        if (!a.exit_on_refine && a.checkpoint_every == 0) break;
        MF_CUDA(cudaMemcpyAsync(st, w.state, sizeof(st), cudaMemcpyDeviceToHost, s));
        MF_CUDA(cudaMemcpyAsync(&h_status, w.status, sizeof(int), cudaMemcpyDeviceToHost, s));
        MF_CUDA(cudaStreamSynchronize(s));
        if (h_status != 0 || (int)st[S_EXIT] != EXIT_CHECKPOINT) break;
        // checkpoint: the policy picks new working classes, the payload is
        // repacked, and the solve resumes from the saved state
        const int it = (int)st[S_ITERS];
        const void *pnew = (it & 1) ? w.p1 : w.p0;  // written by the last iteration
        const void *pold = (it & 1) ? w.p0 : w.p1;
        if (hook) MF_TRY(hook->fn(hook->ctx, m, w, pnew, pold, it, st[S_RELRES], s));
        if (o.policy == MF_POLICY_FP64 || o.policy == MF_POLICY_STATIC || o.policy == MF_POLICY_STATIC_FP16 ||
            rep.fallback_iteration > 0) {
            a.start = 0;
            continue;
        }
        const bool rule = o.policy == MF_POLICY_RULE || o.policy == MF_POLICY_RULE_SCALED;
        if (rule && a.exit_on_refine && (int)st[S_REFS] > guard_refs) {
            // a whole refinement cycle under the rule's classes that did not
            // halve the FP64 residual (and did not end the solve): the static
            // classes take over for the rest of it (no further checkpoints)
            if (!(st[S_RELRES] <= 0.5 * guard_relres) && !(a.fixed == 0 && st[S_RELRES] <= o.tol)) {
                MF_TRY(static_working_classes(m, m->d_wcls, s));
                MF_TRY(repack(MF_POLICY_STATIC));
                a.exit_on_refine = 0;
                a.start = 0;
                rep.fallback_iteration = (int)st[S_ITERS];
                continue;
            }
            guard_relres = st[S_RELRES];
            guard_refs = (int)st[S_REFS];
        }
        if (o.policy == MF_POLICY_RULE || o.policy == MF_POLICY_RULE_SCALED) {
            MF_TRY(rule_classes(m, o.policy, pnew, pold, nullptr, m->d_wcls, s));
        } else {
            MF_TRY(learned_working_classes(m, w, pnew, pold, m->d_wcls, s));
        }
        MF_TRY(repack(o.policy));
        a.start = 0;
    }
    MF_CUDA(cudaEventRecord(e1, s));
    MF_CUDA(cudaMemcpyAsync(st, w.state, sizeof(st), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaMemcpyAsync(&h_status, w.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rep.iterations = (int)st[S_ITERS];
    rep.refinements = (int)st[S_REFS];
    rep.grid_ctas = G;
    rep.layout = staged ? 2 : slots ? 1 : 0;
    rep.kernel_ms = ms;
    rep.relres = st[S_RELRES];
    const long long n = m->v.rows, nnz = m->v.nnz;
    if (bicg) {
        // per iteration: two SpMVs plus 15 vector streams (FP64), or their
        // mixed-precision counterparts; reliable updates as for CG
        const long long spmv_fp64 = nnz * 9 + 24LL * T + 16 * n;
        const long long spmv_mixed = (long long)m->pay_used + nnz + 24LL * T + 8 * n;
        rep.bytes_moved = mixed ? (long long)rep.iterations * (2 * spmv_mixed + 60 * n) +
                                      (long long)rep.refinements * (spmv_fp64 + 32 * n)
                                : (long long)rep.iterations * (2 * spmv_fp64 + 120 * n);
    } else if (!mixed) {
        rep.bytes_moved = (long long)rep.iterations * (nnz * 9 + 24LL * T + 16 * n + 72 * n);
    } else {
        // per iteration: packed payload + column bytes + tile metadata + FP32
        // vectors (p, q gathered/written, x_lo, r: 9 streams of 4 bytes);
        // per reliable update: an FP64 SpMV plus 5 FP64/FP32 streams
        const long long spmv_mixed = (long long)m->pay_used + nnz + 24LL * T + 8 * n;
        const long long spmv_fp64 = nnz * 9 + 24LL * T + 16 * n;
        rep.bytes_moved = (long long)rep.iterations * (spmv_mixed + 36 * n) +
                          (long long)rep.refinements * (spmv_fp64 + 32 * n);
    }
    // Jacobi: D^-1 read (FP64) and z written (vector type) every iteration
    if (!bicg && o.precond) rep.bytes_moved += (long long)rep.iterations * (mixed ? 12 : 16) * n;
    (void)launches;
    if (a.timing) {
        std::vector<unsigned long long> t((size_t)G * 8);
        MF_CUDA(cudaMemcpy(t.data(), w.timing, sizeof(unsigned long long) * 8 * G, cudaMemcpyDeviceToHost));
        double mx = 0;
        for (int k = 0; k < 9; k++) rep.phase_us[k] = 0;
        for (int g = 0; g < G; g++) {
            for (int k = 0; k < 5; k++) rep.phase_us[k] += t[(size_t)g * 8 + k] * 1e-3 / G;
            for (int k = 5; k < 8; k++) rep.phase_us[k + 1] += t[(size_t)g * 8 + k] * 1e-3 / G;
            mx = std::max(mx, t[(size_t)g * 8] * 1e-3);
        }
        rep.phase_us[5] = mx;
    }
    MF_TRY(true_residual(m, b, x, w, &rep.relres_true, s));
    if (h_status != 0) {
        rep.status = h_status;
        set_last_error(h_status == MF_ERR_TIMEOUT ? "grid-wide wait exceeded its budget"
                                                  : (bicg ? "BiCGSTAB breakdown" : "CG breakdown"));
        return (mf_status)h_status;
    }
    if (!a.fixed && !(rep.relres_true <= o.tol * (1.0 + 1e-6) || rep.relres <= o.tol)) {
        rep.status = MF_ERR_NOT_CONVERGED;
        return MF_ERR_NOT_CONVERGED;
    }
    if (!a.fixed && (int)st[S_EXIT] == EXIT_MAXITER) {
        rep.status = MF_ERR_NOT_CONVERGED;
        return MF_ERR_NOT_CONVERGED;
    }
    rep.status = MF_OK;
    return MF_OK;
}

mf_status cg_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                   double *history, cudaStream_t s)
{
    return persistent_solve(false, m, b, x, o, rep, history, s);
}

mf_status cg_solve_traced(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                          const TraceHook *hook, cudaStream_t s)
{
    return persistent_solve(false, m, b, x, o, rep, nullptr, s, hook);
}

mf_status bicgstab_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                         double *history, cudaStream_t s)
{
    mf_solve_opts oo = o;
    // BiCGSTAB has no checkpoint policies: dynamic policies run with the
    // value-range (static) classes
    if (oo.policy == MF_POLICY_RULE || oo.policy == MF_POLICY_RULE_SCALED || oo.policy == MF_POLICY_LEARNED)
        oo.policy = MF_POLICY_STATIC;
    return persistent_solve(true, m, b, x, oo, rep, history, s);
}

}  // namespace mf
