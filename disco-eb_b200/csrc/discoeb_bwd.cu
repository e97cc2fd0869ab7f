// Discrete adjoint on sm_100a: the recording forward solve, the reverse sweep and the contraction
// of the cotangents with parameter tangents; C ABI (include/discoeb.h).
//
// Layout: the recording forward is the forward solve (one warp per k-mode) whose accept hook
// writes each accepted step's end time (8 bytes) and every checkpoint_every-th start state into
// the caller's record buffer.  The reverse sweep runs one block of five warps per mode (replay of
// the segments from their checkpoints, recomputation of each step, the chain of the cotangents of
// y[1:], the a-component's scalar chain, the parameter and table seeds; bwd_split_kernel), with
// the cosmology, two recomputed steps, the critical warp's workspace and two steps' functional
// records in shared memory (~108 KB at n = 143) and two segment buffers per mode in the caller's
// workspace.
// Table-knot cotangents are summed over the modes of a cosmology with double-precision atomics
// (the order of those additions is not fixed, so they agree between runs to rounding, not bit
// for bit).
#include <cuda_runtime.h>

#include <cstdint>

#include "adjoint.cuh"
#include "discoeb.h"

using namespace dscb;

namespace {

constexpr int kCosmoDoublesB = (sizeof(DiscoebCosmo) + 7) / 8;

__device__ __forceinline__ void copy_cosmo_warp(const WarpTeam& tm, const DiscoebCosmo* src, DiscoebCosmo* dst)
{
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = tm.lane; i < (int)(sizeof(DiscoebCosmo) / 4); i += 32) d[i] = s[i];
    tm.sync();
}

// output fields of one output time: RSA projection (scratch: n doubles of shared memory) then
// convert_to_output_variables
__device__ void record_emit(const WarpTeam& tm, const DiscoebCosmo& P, const Dims& D, double k, double tau,
                            const double* y, double* y20, double* scratch)
{
    const int n = D.n;
    double fld[4];
    const bool rsa = rsa_projection<double>(P, nullptr, D, tau, k, y, nullptr, fld);
    for (int i = tm.lane; i < n; i += 32) {
        double v = y[i];
        if (rsa) {
            const int s = rsa_slot(D, i);
            if (s >= 0) v = fld[s];
            else if (s == -1) v = 0.0;
        }
        scratch[i] = v;
    }
    tm.sync();
    if (tm.leader()) {
        double o[20];
        output_vars<double>(P, nullptr, D, k, scratch, nullptr, o);
        for (int q = 0; q < 20; ++q) y20[q] = o[q];
    }
    tm.sync();
}

__global__ void __launch_bounds__(128) fwd_record_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, DiscoebControl ctrl,
    int n_modes, const double* __restrict__ kmodes, const double* __restrict__ tau_start, const double* __restrict__ y0,
    const double* __restrict__ sw, int n_out, const double* __restrict__ tau_out, int mem_doubles, int cap, int every,
    long long rec_doubles, double* records, int32_t* n_acc, double* y_out20, int32_t* status, int32_t* nsteps)
{
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5;
    const WarpTeam tm{(int)(threadIdx.x & 31)};
    const int wpb = blockDim.x >> 5;
    double* base = smem + (size_t)warp * (kCosmoDoublesB + mem_doubles);
    DiscoebCosmo* P = reinterpret_cast<DiscoebCosmo*>(base);
    double* wmem = base + kCosmoDoublesB;
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    auto fill_nan = [&](int mode, int from) {
        if (y_out20)
            for (int j = from; j < n_out; ++j)
                for (int i = tm.lane; i < 20; i += 32) y_out20[((size_t)mode * n_out + j) * 20 + i] = qnan;
    };
    int cur = -1;
    for (int mode = blockIdx.x * wpb + warp; mode < n_modes; mode += gridDim.x * wpb) {
        const int ci = mode_cosmo ? mode_cosmo[mode] : 0;
        bool bad = ci < 0 || ci >= n_cosmo;
        if (!bad && ci != cur) {
            copy_cosmo_warp(tm, cosmos + ci, P);
            cur = ci;
        }
        const Dims D = make_dims(*P);
        if (!bad && mode_mem_doubles(D) != mem_doubles) bad = true;
        if (bad) {
            fill_nan(mode, 0);
            if (tm.leader()) {
                status[mode] = DISCOEB_BAD_INDEX;
                nsteps[mode] = 0;
                n_acc[mode] = 0;
            }
            continue;
        }
        const int n = D.n;
        ModeMem M = carve(wmem, D);
        const double k = kmodes[mode];
        for (int i = tm.lane; i < n; i += 32) M.y[i] = y0[(size_t)mode * n + i];
        double swm[3] = {sw[3 * mode], sw[3 * mode + 1], sw[3 * mode + 2]};
        tm.sync();
        double* rec = records + (size_t)mode * rec_doubles;
        Recorder<WarpTeam> R{&tm, &M, rec, rec + cap, cap, every, n, 0};
        const double* tout = tau_out + (size_t)ci * n_out;
        auto emit = [&](int j, const double* y, int) {
            if (y_out20) record_emit(tm, *P, D, k, tout[j], y, y_out20 + ((size_t)mode * n_out + j) * 20, M.f);
        };
        const SolveResult res = solve_mode(tm, *P, D, ctrl, k, tau_start[mode], swm, n_out, tout, M, emit,
                                           (const DiscoebTangent*)nullptr, (const TanMem*)nullptr, (double*)nullptr, 0,
                                           &R);
        fill_nan(mode, res.outputs);
        if (tm.leader()) {
            status[mode] = (res.status == DISCOEB_ABORTED && R.count >= cap) ? DISCOEB_RECORD_FULL : res.status;
            nsteps[mode] = res.steps;
            n_acc[mode] = R.count;
        }
        tm.sync();
    }
}

// ---- the reverse sweep, split over five cooperating warps per mode ----
// Warp roles (one mode per block, steps taken apart last to first, "job" j = step nacc - 1 - j):
//   0 critical:   the chain of the cotangents of y[1:] (adjoint_step) and the output layer;
//   1 recompute:  each step's stages, factorisation, U columns and Zt into one of two shared
//                 step slots, from the step's start state;
//   2 replay:     each segment of `every` steps re-run from its checkpoint into one of two
//                 global segment buffers (the start states the recompute warp reads);
//   3 a-chain:    the a-component of every step (achain_step), then the parameter and table
//                 seeds of the step's W-term records 8..15;
//   4 deferred:   the parameter and table seeds of the stage records 0..7 and the column-0
//                 record 16 (after warp 3 has filled in their lambda_0).
// Records and step scalars live in one of two shared buffers per job parity.  Hand-over by
// counters in shared memory, every wait bounded (a wait that runs out sets the block's abort
// flag, every warp leaves its loop, the mode reports DISCOEB_ABORTED with NaN results and the
// launch ends normally).
constexpr long long kMaxPollsB = 1LL << 24;  // ~2 s with the back-off below; a step takes < 1 ms
enum { F_REC = 0, F_CRIT = 1, F_ACHAIN = 2, F_DEF1 = 3, F_DEF2 = 4, F_SEG = 5, F_SEGUSED = 6, F_ABORT = 7,
       kNFlags = 8 };
constexpr int kBwdWarps = 5;

__device__ bool wait_flag(const WarpTeam& tm, volatile int* flags, int which, int target)
{
    int ok = 0;
    if (tm.leader()) {
        long long polls = 0;
        while (true) {
            if (flags[which] >= target) { ok = 1; break; }
            if (flags[F_ABORT]) break;
            if (++polls > kMaxPollsB) { flags[F_ABORT] = 1; break; }
            __nanosleep(100);
        }
        __threadfence_block();
    }
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ void post_flag(const WarpTeam& tm, volatile int* flags, int which, int value)
{
    tm.sync();
    if (tm.leader()) {
        __threadfence_block();
        flags[which] = value;
    }
    tm.sync();
}

// a step slot: the recomputed step (ModeMem), U columns, Zt, 4 scalars, the 8 stage backgrounds
DHD int slot_doubles(const Dims& D) { return mode_mem_doubles(D) + 6 * D.n + 4 + 8 * bg_image_doubles(); }
DHD long long bwd_ws_doubles_per_mode(const Dims& D, int every)
{
    return 2LL * every * D.n + mode_mem_doubles(D);
}
// one job parity's records and step scalars
DHD int job_buf_doubles(const Dims& D) { return kRecPerStep * drec_doubles(D) + kAScalars; }
// shared memory of bwd_split_kernel, in doubles after the cosmology and the flags: the critical
// warp's workspace, two step slots, two job buffers, the a-chain warp's scratch and staging, the
// deferred warp's staging, two accumulator sets (16 parameter doubles + kNTabSeeds two-double
// accumulators each) and the a-chain's final value
DHD int bwd_smem_doubles(const Dims& D)
{
    return adj_mem_doubles(D, false) + 2 * slot_doubles(D) + 2 * job_buf_doubles(D) + kAScratch +
           2 * 8 * kDeferredSeeds + 2 * (16 + 2 * kNTabSeeds) + 2;
}

__global__ void __launch_bounds__(32 * kBwdWarps, 1) bwd_split_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, int n_modes,
    const double* __restrict__ kmodes, const double* __restrict__ tau_start, const double* __restrict__ sw, int n_out,
    const double* __restrict__ tau_out, int cap, int every, long long rec_doubles, const double* __restrict__ records,
    const int32_t* __restrict__ n_acc, const int32_t* __restrict__ fwd_status, double* ws,
    const double* __restrict__ ybar20, int mem_doubles, double* y0_bar, double* tau_out_bar, double* par_bar,
    double* table_bar, int tstride, int table_per_mode, int32_t* status)
{
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5;
    const WarpTeam tm{(int)(threadIdx.x & 31)};
    const int mode = blockIdx.x;
    if (mode >= n_modes) return;
    DiscoebCosmo* P = reinterpret_cast<DiscoebCosmo*>(smem);
    int* flags = reinterpret_cast<int*>(smem + kCosmoDoublesB);
    volatile int* vf = flags;
    double* wmem = smem + kCosmoDoublesB + kNFlags / 2;
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    const int ci = mode_cosmo ? mode_cosmo[mode] : 0;
    int st = fwd_status[mode];
    if (ci < 0 || ci >= n_cosmo) st = DISCOEB_BAD_INDEX;
    if (st == DISCOEB_OK) {
        const int* src = reinterpret_cast<const int*>(cosmos + ci);
        int* dst = reinterpret_cast<int*>(P);
        for (int i = threadIdx.x; i < (int)(sizeof(DiscoebCosmo) / 4); i += blockDim.x) dst[i] = src[i];
    }
    if (threadIdx.x < kNFlags) flags[threadIdx.x] = 0;
    __syncthreads();
    if (st == DISCOEB_OK && mode_mem_doubles(make_dims(*P)) != mem_doubles) st = DISCOEB_BAD_INDEX;
    const int n = (mem_doubles - 4 * kMaxSlots - 32) / 23;  // state size of the launch (mode_mem_doubles)
    if (st != DISCOEB_OK) {  // no forward to take apart: report, write NaN (the whole block returns)
        for (int i = threadIdx.x; i < n; i += blockDim.x) y0_bar[(size_t)mode * n + i] = qnan;
        for (int j = threadIdx.x; j < n_out; j += blockDim.x) tau_out_bar[(size_t)mode * n_out + j] = qnan;
        for (int q = threadIdx.x; q < 8; q += blockDim.x) par_bar[(size_t)mode * 8 + q] = qnan;
        if (threadIdx.x == 0) status[mode] = st;
        return;
    }
    const Dims D = make_dims(*P);
    const double k = kmodes[mode];
    const double t0 = tau_start[mode];
    const double* swm = sw + 3 * mode;
    const double* tout = tau_out + (size_t)ci * n_out;
    const double* rec = records + (size_t)mode * rec_doubles;
    const double* tlog = rec;
    const double* ckpt = rec + cap;
    const int nacc = n_acc[mode];
    double* tbar = table_bar + (size_t)(table_per_mode ? mode : ci) * 8 * tstride;
    // shared (bwd_smem_doubles): critical warp's workspace, two step slots, two job buffers (records
    // + step scalars), the a-chain warp's scratch, staging of both seed warps, their accumulators
    AdjMem A = carve_adj(wmem, D, false);
    double* slots = wmem + adj_mem_doubles(D, false);
    const int sd = slot_doubles(D);
    double* jobbuf = slots + 2 * sd;
    const int jb = job_buf_doubles(D);
    const int recs_len = kRecPerStep * drec_doubles(D);
    double* ascr = jobbuf + 2 * jb;
    double* g1 = ascr + kAScratch;
    double* g2 = g1 + 8 * kDeferredSeeds;
    double* pb1 = g2 + 8 * kDeferredSeeds;
    TabAcc* tab1 = reinterpret_cast<TabAcc*>(pb1 + 16);
    double* pb2 = pb1 + 16 + 2 * kNTabSeeds;
    TabAcc* tab2 = reinterpret_cast<TabAcc*>(pb2 + 16);
    double* lam0_final = pb2 + 16 + 2 * kNTabSeeds;
    auto job_recs = [&](int j) { return jobbuf + (size_t)(j & 1) * jb; };
    auto job_sc = [&](int j) { return jobbuf + (size_t)(j & 1) * jb + recs_len; };
    auto slot_mem = [&](int j, ModeMem& M, double*& Uk, double*& Zt, double*& meta) {
        double* b = slots + (size_t)(j & 1) * sd;
        M = carve(b, D);
        Uk = b + mem_doubles;
        Zt = Uk + 3 * n;
        meta = Zt + 3 * n;
    };
    // global: two segment buffers and the replay warp's step workspace
    double* mws = ws + (size_t)mode * bwd_ws_doubles_per_mode(D, every);
    double* segbuf = mws;
    const int last_sg = nacc > 0 ? (nacc - 1) / every : -1;
    int hint = P->xe_loga.n_knots / 2;

    if (warp == 0) {
        // ---- critical ----
        for (int i = tm.lane; i < n; i += 32) A.lam[i] = 0.0;
        for (int q = tm.lane; q < 16; q += 32) A.pb[q] = 0.0;
        for (int q = tm.lane; q < kNTabSeeds; q += 32) {
            A.tab[q].cur = -1;
            A.tab[q].w = 0.0;
        }
        tm.sync();
        int jout = n_out - 1;
        const double* ob = ybar20 + (size_t)mode * n_out * 20;
        for (int j = 0; j < nacc; ++j) {
            if (!wait_flag(tm, vf, F_REC, j + 1)) break;
            // the job buffer of parity j was last read by job j - 2's seed warps
            if (!wait_flag(tm, vf, F_DEF1, j - 1) || !wait_flag(tm, vf, F_DEF2, j - 1)) break;
            ModeMem M;
            double *Uk, *Zt, *meta;
            slot_mem(j, M, Uk, Zt, meta);
            const double tm0 = meta[0], h = meta[1];
            const int regime = (int)meta[2];
            double lam0_out = 0.0;  // the output layer's a-cotangent at this step's end (warp 3's chain)
            while (jout >= 0 && tout[jout] > tm0) {  // outputs emitted at the end of this step
                for (int i = tm.lane; i < n; i += 32) {
                    A.us[i] = M.u[i] + M.K[7 * n + i];
                    A.ub[i] = 0.0;
                }
                tm.sync();
                output_adjoint(tm, *P, D, tout[jout], k, A.us, ob + (size_t)jout * 20, A, A.ub, tbar, tstride);
                Bg<double> bo;
                bg_eval_team(tm, *P, A.us[0], tout[jout], k, regime, bo, hint);
                rhs_team(tm, *P, D, bo, k, tout[jout], A.us, A.yb, (double*)nullptr);
                tm.sync();
                double acc = 0.0;
                for (int i = tm.lane; i < n; i += 32) {
                    acc += A.ub[i] * A.yb[i];
                    if (i > 0) A.lam[i] += A.ub[i];
                }
                const double tb = tm.sum(acc);
                if (tm.leader()) tau_out_bar[(size_t)mode * n_out + jout] = tb;
                lam0_out += A.ub[0];
                tm.sync();
                --jout;
            }
            adjoint_step(tm, *P, D, k, tm0, h, regime, M, A, Uk, Zt, job_recs(j), job_sc(j), lam0_out, hint, meta + 4);
            post_flag(tm, vf, F_CRIT, j + 1);
        }
        if (tm.leader())
            for (; jout >= 0; --jout) tau_out_bar[(size_t)mode * n_out + jout] = 0.0;
        tm.sync();
    } else if (warp == 1) {
        // ---- recompute ----
        for (int j = 0; j < nacc; ++j) {
            const int m = nacc - 1 - j;
            const int sg = m / every, q = last_sg - sg, n0 = sg * every;
            if (!wait_flag(tm, vf, F_SEG, q + 1)) break;
            if (!wait_flag(tm, vf, F_CRIT, j - 1)) break;
            ModeMem M;
            double *Uk, *Zt, *meta;
            slot_mem(j, M, Uk, Zt, meta);
            const double* ym = (m == n0) ? ckpt + (size_t)sg * n : segbuf + ((size_t)(q & 1) * every + (m - n0)) * n;
            for (int i = tm.lane; i < n; i += 32) M.y[i] = ym[i];
            tm.sync();
            const double tm0 = m == 0 ? t0 : tlog[m - 1], h = tlog[m] - tm0;
            const int regime = regime_at(*P, tm0, swm);
            rodas5_step(tm, *P, D, k, tm0, h, regime, M, hint, (const DiscoebTangent*)nullptr, (const TanMem*)nullptr,
                        Uk);
            make_Zt(tm, D, M, h, Zt);
            stage_backgrounds(tm, *P, D, k, tm0, h, regime, M, meta + 4, hint);
            if (tm.leader()) {
                meta[0] = tm0;
                meta[1] = h;
                meta[2] = (double)regime;
            }
            post_flag(tm, vf, F_REC, j + 1);
            if (m == n0) post_flag(tm, vf, F_SEGUSED, q + 1);
        }
    } else if (warp == 2) {
        // ---- replay ----
        ModeMem M = carve(mws + 2LL * every * n, D);
        for (int q = 0; q <= last_sg; ++q) {
            const int sg = last_sg - q, n0 = sg * every, n1 = nacc < n0 + every ? nacc : n0 + every;
            if (!wait_flag(tm, vf, F_SEGUSED, q - 1)) break;
            double* buf = segbuf + (size_t)(q & 1) * every * n;
            const double* ck = ckpt + (size_t)sg * n;
            for (int i = tm.lane; i < n; i += 32) M.y[i] = ck[i];
            tm.sync();
            double t = n0 == 0 ? t0 : tlog[n0 - 1];
            for (int m = n0; m < n1 - 1; ++m) {
                const double tn = tlog[m];
                rodas5_step(tm, *P, D, k, t, tn - t, regime_at(*P, t, swm), M, hint);
                for (int i = tm.lane; i < n; i += 32) {
                    const double y1 = M.u[i] + M.K[7 * n + i];
                    M.y[i] = y1;
                    buf[(size_t)(m + 1 - n0) * n + i] = y1;
                }
                tm.sync();
                t = tn;
                if (__shfl_sync(0xffffffffu, vf[F_ABORT], 0)) break;  // warp-uniform
            }
            post_flag(tm, vf, F_SEG, q + 1);
        }
    } else {
        // ---- seed warps: 3 (the a-chain, then records 8..15) and 4 (records 0..7 and 16) ----
        const bool achain = warp == 3;
        double* pbw = achain ? pb1 : pb2;
        TabAcc* tabw = achain ? tab1 : tab2;
        double* gw = achain ? g1 : g2;
        for (int q = tm.lane; q < 16; q += 32) pbw[q] = 0.0;
        for (int q = tm.lane; q < kNTabSeeds; q += 32) {
            tabw[q].cur = -1;
            tabw[q].w = 0.0;
        }
        tm.sync();
        double lam0 = 0.0;  // warp 3: the a-component of the running cotangent
        for (int j = 0; j < nacc; ++j) {
            if (!wait_flag(tm, vf, F_CRIT, j + 1)) break;
            double* recs = job_recs(j);
            if (achain) {
                achain_step(tm, *P, D, k, recs, job_sc(j), lam0, ascr);
                post_flag(tm, vf, F_ACHAIN, j + 1);
                deferred_records(tm, *P, D, k, recs, 8, 16, gw, DefAcc{pbw, tabw}, tbar, tstride);
                post_flag(tm, vf, F_DEF1, j + 1);
            } else {
                if (!wait_flag(tm, vf, F_ACHAIN, j + 1)) break;
                deferred_records(tm, *P, D, k, recs, 0, 8, gw, DefAcc{pbw, tabw}, tbar, tstride);
                deferred_records(tm, *P, D, k, recs, 16, 17, gw, DefAcc{pbw, tabw}, tbar, tstride);
                post_flag(tm, vf, F_DEF2, j + 1);
            }
        }
        if (achain && tm.leader()) *lam0_final = lam0;
        tm.sync();
    }
    __syncthreads();
    const bool aborted = vf[F_ABORT] != 0;
    if (warp == 0) {
        for (int i = tm.lane; i < n; i += 32)
            y0_bar[(size_t)mode * n + i] = aborted ? qnan : (i == 0 ? *lam0_final : A.lam[i]);
        for (int q = tm.lane; q < 8; q += 32)
            par_bar[(size_t)mode * 8 + q] = aborted ? qnan : A.pb[X_GRHOM + q] + pb1[X_GRHOM + q] + pb2[X_GRHOM + q];
        if (aborted)
            for (int j = tm.lane; j < n_out; j += 32) tau_out_bar[(size_t)mode * n_out + j] = qnan;
        for (int xs = X_KNOT0 + tm.lane; xs < X_KNOT0 + kNTabSeeds; xs += 32) {
            if (aborted) break;
            tab_flush(A.tab[xs - X_KNOT0], xs, tbar, tstride);
            tab_flush(tab1[xs - X_KNOT0], xs, tbar, tstride);
            tab_flush(tab2[xs - X_KNOT0], xs, tbar, tstride);
        }
        if (tm.leader()) status[mode] = aborted ? DISCOEB_ABORTED : DISCOEB_OK;
    }
}

// theta_bar[c, d] = sum over the modes of cosmology c of ybar0 . y0_dot + taubar . tau_out_dot +
// pbar . (scalar tangents), plus the table cotangents against the table tangents: one block per
// (cosmology, direction)
__global__ void __launch_bounds__(256) contract_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, int n_modes, int n,
    int n_out, const DiscoebTangent* __restrict__ tangents, int n_dir, const double* __restrict__ y0_dot,
    const double* __restrict__ tau_out_dot, const double* __restrict__ y0_bar, const double* __restrict__ tau_out_bar,
    const double* __restrict__ par_bar, const double* __restrict__ table_bar, int tstride, double* theta_bar)
{
    const int c = blockIdx.x / n_dir, d = blockIdx.x - c * n_dir;
    const DiscoebTangent& tn = tangents[(size_t)c * n_dir + d];
    const double sc[8] = {tn.grhom, tn.Omegam, tn.Omegab, tn.OmegaDE, tn.amnu, tn.w0, tn.wa, tn.H0};
    double acc = 0.0;
    for (int m = threadIdx.x; m < n_modes; m += blockDim.x) {
        if ((mode_cosmo ? mode_cosmo[m] : 0) != c) continue;
        const double* yb = y0_bar + (size_t)m * n;
        const double* yd = y0_dot + ((size_t)d * n_modes + m) * n;
        for (int i = 0; i < n; ++i) acc += yb[i] * yd[i];
        const double* tb = tau_out_bar + (size_t)m * n_out;
        const double* td = tau_out_dot + ((size_t)c * n_dir + d) * n_out;
        for (int j = 0; j < n_out; ++j) acc += tb[j] * td[j];
        for (int q = 0; q < 8; ++q) acc += par_bar[(size_t)m * 8 + q] * sc[q];
    }
    const DiscoebCosmo& P = cosmos[c];
    const double* rows[8] = {tn.xe_y, tn.xe_S, tn.cs2a_y, tn.cs2a_S, tn.logrhonu_y, tn.logrhonu_S, tn.logpnu_y,
                             tn.logpnu_S};
    const int nk[4] = {P.xe_loga.n_knots, P.cs2a_loga.n_knots, P.logrhonu_loga.n_knots, P.logpnu_loga.n_knots};
    for (int r = 0; r < 8; ++r) {
        if (!rows[r]) continue;
        const int m = nk[r >> 1] < tstride ? nk[r >> 1] : tstride;
        const double* tb = table_bar + ((size_t)c * 8 + r) * tstride;
        for (int i = threadIdx.x; i < m; i += blockDim.x) acc += tb[i] * rows[r][i];
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) theta_bar[blockIdx.x] = red[0];
}

// theta_bar[m, d] for each mode on its own (its table cotangents in rows [m, 8, tstride]): one
// warp per (mode, direction)
__global__ void __launch_bounds__(128) contract_mode_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, int n_modes, int n,
    int n_out, const DiscoebTangent* __restrict__ tangents, int n_dir, const double* __restrict__ y0_dot,
    const double* __restrict__ tau_out_dot, const double* __restrict__ y0_bar, const double* __restrict__ tau_out_bar,
    const double* __restrict__ par_bar, const double* __restrict__ table_bar, int tstride, double* theta_bar)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long long)n_modes * n_dir) return;
    const int m = (int)(w / n_dir), d = (int)(w - (long long)m * n_dir);
    const int c = mode_cosmo ? mode_cosmo[m] : 0;
    if (c < 0 || c >= n_cosmo) {
        if (lane == 0) theta_bar[w] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const DiscoebTangent& tn = tangents[(size_t)c * n_dir + d];
    double acc = 0.0;
    const double* yb = y0_bar + (size_t)m * n;
    const double* yd = y0_dot + ((size_t)d * n_modes + m) * n;
    for (int i = lane; i < n; i += 32) acc += yb[i] * yd[i];
    const double* td = tau_out_dot + ((size_t)c * n_dir + d) * n_out;
    for (int j = lane; j < n_out; j += 32) acc += tau_out_bar[(size_t)m * n_out + j] * td[j];
    const double sc[8] = {tn.grhom, tn.Omegam, tn.Omegab, tn.OmegaDE, tn.amnu, tn.w0, tn.wa, tn.H0};
    if (lane < 8) acc += par_bar[(size_t)m * 8 + lane] * sc[lane];
    const DiscoebCosmo& P = cosmos[c];
    const double* rows[8] = {tn.xe_y, tn.xe_S, tn.cs2a_y, tn.cs2a_S, tn.logrhonu_y, tn.logrhonu_S, tn.logpnu_y,
                             tn.logpnu_S};
    const int nk[4] = {P.xe_loga.n_knots, P.cs2a_loga.n_knots, P.logrhonu_loga.n_knots, P.logpnu_loga.n_knots};
    for (int r = 0; r < 8; ++r) {
        if (!rows[r]) continue;
        const int kk = nk[r >> 1] < tstride ? nk[r >> 1] : tstride;
        const double* tb = table_bar + ((size_t)m * 8 + r) * tstride;
        for (int i = lane; i < kk; i += 32) acc += tb[i] * rows[r][i];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) theta_bar[w] = acc;
}

int validate_cosmo_b(const DiscoebCosmo* c)
{
    if (!c) return DISCOEB_EINVAL;
    if (c->nqmax < 0 || c->nqmax > DISCOEB_MAX_NQ) return DISCOEB_EINVAL;
    if (c->lmaxg < 3 || c->lmaxgp < 3 || c->lmaxr < 3 || c->lmaxnu < 3) return DISCOEB_EINVAL;
    if (c->use_tca) return DISCOEB_EUNSUPPORTED;
    return DISCOEB_SUCCESS;
}

}  // namespace

extern "C" {

int64_t discoeb_step_record_doubles(int32_t nvar, int32_t step_capacity, int32_t checkpoint_every)
{
    if (nvar < 1 || step_capacity < 1 || checkpoint_every < 1) return DISCOEB_EINVAL;
    return (int64_t)record_doubles(nvar, step_capacity, checkpoint_every);
}

int32_t discoeb_fwd_record(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                           const DiscoebControl* ctrl, int32_t n_modes, const int32_t* mode_cosmo, const double* kmodes,
                           const double* tau_start, const double* y0, const double* switch_tau, int32_t n_out,
                           const double* tau_out, double* y_out20, int32_t* status, int32_t* nsteps,
                           int32_t step_capacity, int32_t checkpoint_every, double* records, int32_t* n_accepted,
                           void* stream)
{
    int rc = validate_cosmo_b(cosmo0_host);
    if (rc) return rc;
    if (!cosmos_dev || !ctrl || n_cosmo < 1 || n_modes < 0 || n_out < 1 || step_capacity < 1 || checkpoint_every < 1)
        return DISCOEB_EINVAL;
    if (n_modes == 0) return DISCOEB_SUCCESS;
    if (!kmodes || !tau_start || !y0 || !switch_tau || !tau_out || !status || !nsteps || !records || !n_accepted)
        return DISCOEB_EINVAL;
    if (ctrl->method != DISCOEB_METHOD_RODAS5_STRUCTURED) return DISCOEB_EUNSUPPORTED;
    if (!(ctrl->rtol > 0.0) || !(ctrl->atol >= 0.0) || ctrl->max_steps < 1) return DISCOEB_EINVAL;
    const Dims D = make_dims(*cosmo0_host);
    const int mem = mode_mem_doubles(D);
    const int wpb = 4;
    const size_t smem = (size_t)wpb * (kCosmoDoublesB + mem) * sizeof(double);
    int dev = 0, max_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DISCOEB_ECUDA;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > (size_t)max_optin) return DISCOEB_EUNSUPPORTED;
    if (cudaFuncSetAttribute(fwd_record_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DISCOEB_ECUDA;
    const long long rec = record_doubles(D.n, step_capacity, checkpoint_every);
    const int blocks = (n_modes + wpb - 1) / wpb;
    fwd_record_kernel<<<blocks, 32 * wpb, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        cosmos_dev, n_cosmo, mode_cosmo, *ctrl, n_modes, kmodes, tau_start, y0, switch_tau, n_out, tau_out, mem,
        step_capacity, checkpoint_every, rec, records, n_accepted, y_out20, status, nsteps);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int64_t discoeb_bwd_workspace_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_modes, int32_t checkpoint_every)
{
    if (!cosmo0_host || n_modes < 0 || checkpoint_every < 1) return DISCOEB_EINVAL;
    return (int64_t)n_modes * bwd_ws_doubles_per_mode(make_dims(*cosmo0_host), checkpoint_every) *
           (int64_t)sizeof(double);
}

int32_t discoeb_bwd(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const int32_t* mode_cosmo, int32_t n_modes, const double* kmodes, const double* tau_start,
                    const double* switch_tau, int32_t n_out, const double* tau_out, int32_t step_capacity,
                    int32_t checkpoint_every, const double* records, const int32_t* n_accepted,
                    const int32_t* fwd_status, const double* y_out20_bar, double* y0_bar, double* tau_out_bar,
                    double* par_bar, double* table_bar, int32_t table_stride, int32_t table_per_mode, void* workspace,
                    int64_t workspace_bytes, int32_t* status, void* stream)
{
    int rc = validate_cosmo_b(cosmo0_host);
    if (rc) return rc;
    if (!cosmos_dev || n_cosmo < 1 || n_modes < 0 || n_out < 1 || step_capacity < 1 || checkpoint_every < 1)
        return DISCOEB_EINVAL;
    if (n_modes == 0) return DISCOEB_SUCCESS;
    if (!kmodes || !tau_start || !switch_tau || !tau_out || !records || !n_accepted || !fwd_status || !y_out20_bar ||
        !y0_bar || !tau_out_bar || !par_bar || !table_bar || !workspace || !status)
        return DISCOEB_EINVAL;
    const Dims D = make_dims(*cosmo0_host);
    const int kmax = cosmo0_host->xe_loga.n_knots > cosmo0_host->cs2a_loga.n_knots ? cosmo0_host->xe_loga.n_knots
                                                                                   : cosmo0_host->cs2a_loga.n_knots;
    if (table_stride < kmax || table_stride < cosmo0_host->logrhonu_loga.n_knots ||
        table_stride < cosmo0_host->logpnu_loga.n_knots)
        return DISCOEB_EINVAL;
    if (workspace_bytes < discoeb_bwd_workspace_bytes(cosmo0_host, n_modes, checkpoint_every)) return DISCOEB_EINVAL;
    const int mem = mode_mem_doubles(D);
    const size_t smem = (size_t)(kCosmoDoublesB + kNFlags / 2 + bwd_smem_doubles(D)) * sizeof(double);
    int dev = 0, max_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DISCOEB_ECUDA;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > (size_t)max_optin) return DISCOEB_EUNSUPPORTED;
    if (cudaFuncSetAttribute(bwd_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DISCOEB_ECUDA;
    const long long rec = record_doubles(D.n, step_capacity, checkpoint_every);
    bwd_split_kernel<<<n_modes, 32 * kBwdWarps, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        cosmos_dev, n_cosmo, mode_cosmo, n_modes, kmodes, tau_start, switch_tau, n_out, tau_out, step_capacity,
        checkpoint_every, rec, records, n_accepted, fwd_status, static_cast<double*>(workspace), y_out20_bar, mem,
        y0_bar, tau_out_bar, par_bar, table_bar, table_stride, table_per_mode ? 1 : 0, status);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int32_t discoeb_bwd_contract(const DiscoebCosmo* cosmos_dev, int32_t n_cosmo, const int32_t* mode_cosmo,
                             int32_t n_modes, int32_t nvar, int32_t n_out, const DiscoebTangent* tangents_dev,
                             int32_t n_dir, const double* y0_dot, const double* tau_out_dot, const double* y0_bar,
                             const double* tau_out_bar, const double* par_bar, const double* table_bar,
                             int32_t table_stride, int32_t per_mode, double* theta_bar, void* stream)
{
    if (!cosmos_dev || n_cosmo < 1 || n_modes < 0 || nvar < 1 || n_out < 1 || !tangents_dev || n_dir < 1 || !y0_dot ||
        !tau_out_dot || !y0_bar || !tau_out_bar || !par_bar || !table_bar || table_stride < 1 || !theta_bar)
        return DISCOEB_EINVAL;
    if ((long long)n_cosmo * n_dir > 0x7fffffffLL) return DISCOEB_EINVAL;
    if (per_mode) {
        const long long threads = (long long)n_modes * n_dir * 32;
        if (threads / 128 >= 0x7fffffffLL) return DISCOEB_EINVAL;
        if (n_modes == 0) return DISCOEB_SUCCESS;
        contract_mode_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            cosmos_dev, n_cosmo, mode_cosmo, n_modes, nvar, n_out, tangents_dev, n_dir, y0_dot, tau_out_dot, y0_bar,
            tau_out_bar, par_bar, table_bar, table_stride, theta_bar);
        return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
    }
    contract_kernel<<<n_cosmo * n_dir, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        cosmos_dev, n_cosmo, mode_cosmo, n_modes, nvar, n_out, tangents_dev, n_dir, y0_dot, tau_out_dot, y0_bar,
        tau_out_bar, par_bar, table_bar, table_stride, theta_bar);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

}  // extern "C"
