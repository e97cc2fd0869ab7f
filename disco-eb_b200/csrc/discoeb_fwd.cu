// Forward perturbation solve on sm_100a: kernels and the C ABI (include/discoeb.h).
//
// Layout: one warp owns one k-mode.  Its whole working set (state, eight Rodas5 stage
// vectors, the banded chain factors and the Woodbury blocks, 27 n doubles) lives in
// shared memory; the four background tables are read through the read-only cache.
// All modes of all cosmologies run in one launch; each warp takes modes from a
// grid-stride schedule ordered by the caller (longest first).  HBM traffic is only the
// initial states and the outputs, so the kernel is bound by FP64 latency, not bandwidth.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "discoeb.h"
#include "stepper.cuh"

using namespace dscb;

namespace {

constexpr int kCosmoDoubles = (sizeof(DiscoebCosmo) + 7) / 8;

__device__ __forceinline__ void copy_cosmo(const WarpTeam& tm, const DiscoebCosmo* src, DiscoebCosmo* dst)
{
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = tm.lane; i < (int)(sizeof(DiscoebCosmo) / 4); i += 32) d[i] = s[i];
    tm.sync();
}

// write state / projected state / output fields of one output time (team-parallel)
__device__ void emit_output(const WarpTeam& tm, const DiscoebCosmo& P, const Dims& D, double k, double tau,
                            const double* y, double* yfull, double* y20, double* scratch20)
{
    const int n = D.n;
    double fld[4];
    const bool rsa = rsa_projection<double>(P, nullptr, D, tau, k, y, nullptr, fld);  // all lanes, identical
    // projected state into scratch (shared) then outputs
    double* yp = scratch20;  // n doubles of shared scratch
    for (int i = tm.lane; i < n; i += 32) {
        double v = y[i];
        if (rsa) {
            const int s = rsa_slot(D, i);
            if (s >= 0) v = fld[s];
            else if (s == -1) v = 0.0;
        }
        yp[i] = v;
        if (yfull) yfull[i] = v;
    }
    tm.sync();
    if (y20 && tm.leader()) {
        double o[20];
        output_vars<double>(P, nullptr, D, k, yp, nullptr, o);
        for (int q = 0; q < 20; ++q) y20[q] = o[q];
    }
    tm.sync();
}

// TM: WarpTeam (FP64) or WarpTeamMixed (FP32 chain factors, mix_doubles more per warp)
template <class TM>
__global__ void __launch_bounds__(256) fwd_structured_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, DiscoebControl ctrl,
    int n_modes,
    const double* __restrict__ kmodes, const double* __restrict__ tau_start, const double* __restrict__ y0,
    const double* __restrict__ sw, int n_out, const double* __restrict__ tau_out, int mem_doubles, int mix_doubles,
    double* y_full, double* y_out20, int32_t* status, int32_t* nsteps)
{
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5;
    const TM tm{(int)(threadIdx.x & 31)};
    const int wpb = blockDim.x >> 5;
    double* base = smem + (size_t)warp * (kCosmoDoubles + mem_doubles + mix_doubles);
    DiscoebCosmo* P = reinterpret_cast<DiscoebCosmo*>(base);
    double* wmem = base + kCosmoDoubles;
    const int total_warps = gridDim.x * wpb;
    const int n0 = (mem_doubles - 4 * kMaxSlots - 32) / 23;  // state size of the launch (mode_mem_doubles)
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    // outputs never reached are filled with NaN so that they cannot pass for data
    auto fill_nan = [&](int mode, int from) {
        for (int j = from; j < n_out; ++j) {
            const size_t o = (size_t)mode * n_out + j;
            if (y_full) for (int i = tm.lane; i < n0; i += 32) y_full[o * n0 + i] = qnan;
            if (y_out20) for (int i = tm.lane; i < 20; i += 32) y_out20[o * 20 + i] = qnan;
        }
    };
    int cur_cosmo = -1;
    for (int mode = blockIdx.x * wpb + warp; mode < n_modes; mode += total_warps) {
        const int ci = mode_cosmo ? mode_cosmo[mode] : 0;
        if (ci < 0 || ci >= n_cosmo) {  // invalid cosmology index: report, solve nothing
            fill_nan(mode, 0);
            if (tm.leader()) {
                status[mode] = DISCOEB_BAD_INDEX;
                nsteps[mode] = 0;
            }
            continue;
        }
        if (ci != cur_cosmo) {
            copy_cosmo(tm, cosmos + ci, P);
            cur_cosmo = ci;
        }
        const Dims D = make_dims(*P);
        const int n = D.n;
        if (mode_mem_doubles(D) != mem_doubles || (TM::mixed && mixed_mem_doubles(D) != mix_doubles)) {
            // every cosmology must have the sizes of the first
            fill_nan(mode, 0);
            if (tm.leader()) {
                status[mode] = DISCOEB_BAD_INDEX;
                nsteps[mode] = 0;
            }
            continue;
        }
        ModeMem M = carve(wmem, D);
        if constexpr (TM::mixed) carve_mixed(wmem + mem_doubles, D, M);
        const double k = kmodes[mode];
        for (int i = tm.lane; i < n; i += 32) M.y[i] = y0[(size_t)mode * n + i];
        double swm[3] = {sw[3 * mode], sw[3 * mode + 1], sw[3 * mode + 2]};
        tm.sync();
        const size_t obase = (size_t)mode * n_out;
        const double* tout = tau_out + (size_t)ci * n_out;  // this cosmology's output times
        auto emit = [&](int j, const double* y, int) {
            const size_t o = obase + j;
            emit_output(tm, *P, D, k, tout[j], y, y_full ? y_full + o * n : nullptr,
                        y_out20 ? y_out20 + o * 20 : nullptr, M.f);
        };
        const SolveResult R = solve_mode(tm, *P, D, ctrl, k, tau_start[mode], swm, n_out, tout, M, emit);
        const int st = R.status, steps = R.steps;
        fill_nan(mode, R.outputs);
        if (tm.leader()) {
            status[mode] = st;
            nsteps[mode] = steps;
        }
        tm.sync();
    }
}

constexpr int kTanDoubles = (sizeof(DiscoebTangent) + 7) / 8;
constexpr int kMaxDirsPerBlock = 6;

// Output fields and their tangents at output time j of one (mode, direction): the tangent of
// the state at the moving output time is y' + f tau_out', then the RSA projection and the
// output conversion in dual numbers.  y: the forward state at tau_out[j]; pf: n doubles of
// scratch; TT.fd / TT.jk are used as scratch.  Full: the RSA-projected state and its tangent
// (n values per output) are written instead of the 20 output fields.  Kept out of line: it runs
// at output times only, and inlined into the tangent loop it lengthens the hot code the seven
// warps of a block fetch (measured: the gradient kernel 2% slower inlined).
template <bool Full>
__device__ __noinline__ void emit_tangent_output(const WarpTeam& tm, const DiscoebCosmo& P, const DiscoebTangent* TN, const Dims& D,
                                    double k, int mode, int dir, int n_modes, int n_out, int j, const double* tau_out,
                                    const double* tau_out_dot, const double* y, int regime, const TanMem& TT,
                                    double* pf, double* y_out20, double* y_out20_dot)
{
    const int n = D.n;
    // f at the output time (left limit of the last step's regime), for the moving output time
    int hint = P.xe_loga.n_knots / 2;
    Bg<double> b;
    bg_eval_team(tm, P, y[0], tau_out[j], k, regime, b, hint);
    rhs_team(tm, P, D, b, k, tau_out[j], y, TT.fd, (double*)nullptr);
    tm.sync();
    const double td = tau_out_dot[(size_t)dir * n_out + j];
    for (int i = tm.lane; i < n; i += 32) TT.jk[i] = TT.yd[i] + TT.fd[i] * td;
    tm.sync();
    Dual fld[4];
    const bool rsa = rsa_projection<Dual>(P, TN, D, tau_out[j], k, y, TT.jk, fld);
    for (int i = tm.lane; i < n; i += 32) {
        double v = y[i], vd = TT.jk[i];
        if (rsa) {
            const int sl = rsa_slot(D, i);
            if (sl >= 0) { v = fld[sl].v; vd = fld[sl].d; }
            else if (sl == -1) { v = 0.0; vd = 0.0; }
        }
        if constexpr (Full) {
            const size_t oo = (size_t)mode * n_out + j;
            y_out20_dot[((size_t)dir * n_modes * n_out + oo) * n + i] = vd;
            if (dir == 0 && y_out20) y_out20[oo * n + i] = v;
        } else {
            pf[i] = v;
            TT.fd[i] = vd;
        }
    }
    tm.sync();
    if constexpr (Full) return;
    if (tm.leader()) {
        Dual o[20];
        output_vars<Dual>(P, TN, D, k, pf, TT.fd, o);
        const size_t oo = (size_t)mode * n_out + j;
        for (int q = 0; q < 20; ++q) y_out20_dot[((size_t)dir * n_modes * n_out + oo) * 20 + q] = o[q].d;
        if (dir == 0 && y_out20)
            for (int q = 0; q < 20; ++q) y_out20[oo * 20 + q] = o[q].v;
    }
    tm.sync();
}

// Bounded wait of one warp on a shared-memory counter: lane 0 polls until *flag >= target (or
// the block's abort flag is set, or the poll budget runs out, after which it sets the abort
// flag itself); returns true when the target was reached.  No wait can last forever.
constexpr long long kMaxPolls = 1LL << 24;  // ~2 s with the back-off below; a step takes < 1 ms
__device__ long long poll_budget(const DiscoebControl& c) { return c.max_polls > 0 ? (long long)c.max_polls : kMaxPolls; }
__device__ bool wait_at_least(const WarpTeam& tm, volatile int* flag, int target, volatile int* abort_flag,
                              long long max_polls)
{
    int ok = 0;
    if (tm.leader()) {
        long long polls = 0;
        while (true) {
            if (*flag >= target) { ok = 1; break; }
            if (*abort_flag) break;
            if (++polls > max_polls) { *abort_flag = 1; break; }
            __nanosleep(100);
        }
        __threadfence_block();
    }
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// discoeb_jvp: one block per (mode, group of directions).  Warp 0 runs the adaptive forward
// solve and publishes every accepted step (start state, the 8 stages and the factorisation of
// W) into one of two shared-memory record slots; warps 1..nd each carry the tangent of one
// direction through the published steps (tangent_step) and write its outputs.  The forward
// is solved once per block instead of once per direction, and it runs ahead of the tangents
// by up to two steps.  Steps are handed over with counters in shared memory (published /
// consumed), every wait bounded (wait_at_least); if a wait gives up, the whole block stops and
// reports DISCOEB_ABORTED.  The step sequence is the forward's only, so the tangent is the
// derivative of the discrete solution with the accepted steps held fixed.
template <bool Full, bool Split>
__global__ void __launch_bounds__(32 * (1 + kMaxDirsPerBlock)) jvp_block_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo,
    const DiscoebTangent* __restrict__ tangents, int n_dir, int dpb,
    DiscoebControl ctrl, int n_modes, const double* __restrict__ kmodes, const double* __restrict__ tau_start,
    const double* __restrict__ y0, const double* __restrict__ y0_dot, const double* __restrict__ sw, int n_out,
    const double* __restrict__ tau_out, const double* __restrict__ tau_out_dot, int mem_doubles, int tan_doubles,
    double* rec_glob, double* y_out20, double* y_out20_dot, int32_t* status, int32_t* nsteps)
{
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5;
    WarpTeamSeq tm;
    tm.lane = (int)(threadIdx.x & 31);
    const int groups = (n_dir + dpb - 1) / dpb;
    const int mode = blockIdx.x / groups, grp = blockIdx.x - mode * groups;
    const int d0 = grp * dpb, nd = min(dpb, n_dir - d0);
    const int ci = mode_cosmo ? mode_cosmo[mode] : 0;
    if (ci < 0 || ci >= n_cosmo) {  // invalid cosmology index: report, solve nothing
        const double qn = __longlong_as_double(0x7ff8000000000000LL);
        if (threadIdx.x == 0 && grp == 0) {
            status[mode] = DISCOEB_BAD_INDEX;
            nsteps[mode] = 0;
        }
        // outputs of width 20 (fields) or, for Full, the state size of the first cosmology
        const int W = Full ? make_dims(cosmos[0]).n : 20;
        for (int dd = 0; dd < nd; ++dd)
            for (int i = threadIdx.x; i < n_out * W; i += blockDim.x) {
                y_out20_dot[((size_t)(d0 + dd) * n_modes + mode) * n_out * W + i] = qn;
                if (d0 + dd == 0 && y_out20) y_out20[(size_t)mode * n_out * W + i] = qn;
            }
        return;
    }
    const DiscoebCosmo* cosmo = cosmos + ci;
    tangents += (size_t)ci * n_dir;
    tau_out += (size_t)ci * n_out;
    tau_out_dot += (size_t)ci * n_dir * n_out;
    // shared layout: cosmology, tangents, forward workspace, two step records (+4 scalars
    // each: t, h, t_next, regime), per tangent warp its workspace + 3 n doubles, flags.  With
    // rec_glob (for states whose records would leave room for fewer tangent warps) there is one
    // record, split: its first 13 n doubles (state, stage vectors) in the block's own part of that
    // global array, the factorisation of W (10 n + 224 doubles, re-read by every stage's solve)
    // and the scalars in shared memory; the forward runs one step ahead instead of two
    DiscoebCosmo* P = reinterpret_cast<DiscoebCosmo*>(smem);
    DiscoebTangent* TNs = reinterpret_cast<DiscoebTangent*>(smem + kCosmoDoubles);
    double* fmem = smem + kCosmoDoubles + dpb * kTanDoubles;
    const int rec = mem_doubles + 4;
    const int n0 = (mem_doubles - 4 * kMaxSlots - 32) / 23;  // state size (mode_mem_doubles)
    constexpr int ns = Split ? 1 : 2;            // record slots
    const int gpart = Split ? 13 * n0 : 0;       // doubles of a record in global memory
    const int spart = rec - gpart;               // doubles of a record in shared memory
    double* gslot = Split ? rec_glob + (size_t)blockIdx.x * gpart : nullptr;
    double* slot0 = fmem + mem_doubles;
    const int per_tan = tan_doubles + 3 * n0;
    double* twork = slot0 + ns * spart;
    int* flags = reinterpret_cast<int*>(twork + (size_t)dpb * per_tan);
    // flags: [0,1] published count per slot (step m + 1), [2,3] consumptions per slot,
    //        [4] forward finished, [5] published steps in total, [6] abort
    volatile int* vf = flags;
    {
        const int* s = reinterpret_cast<const int*>(cosmo);
        int* d = reinterpret_cast<int*>(P);
        for (int i = threadIdx.x; i < (int)(sizeof(DiscoebCosmo) / 4); i += blockDim.x) d[i] = s[i];
        for (int dd = 0; dd < nd; ++dd) {
            const int* ts = reinterpret_cast<const int*>(tangents + d0 + dd);
            int* td = reinterpret_cast<int*>(TNs + dd);
            for (int i = threadIdx.x; i < (int)(sizeof(DiscoebTangent) / 4); i += blockDim.x) td[i] = ts[i];
        }
        if (threadIdx.x < 8) flags[threadIdx.x] = 0;
    }
    __syncthreads();
    if (warp > nd) return;  // surplus warps of the last group
    const Dims D = make_dims(*P);
    const int n = D.n;
    if (mode_mem_doubles(D) != mem_doubles) {  // every cosmology must have the sizes of the first
        const double qn = __longlong_as_double(0x7ff8000000000000LL);
        if (warp == 0) {
            if (tm.leader() && grp == 0) {
                status[mode] = DISCOEB_BAD_INDEX;
                nsteps[mode] = 0;
            }
        } else {
            const int dir = d0 + warp - 1;
            const int W = Full ? make_dims(cosmos[0]).n : 20;
            for (int i = tm.lane; i < n_out * W; i += 32) {
                y_out20_dot[((size_t)dir * n_modes + mode) * n_out * W + i] = qn;
                if (dir == 0 && y_out20) y_out20[(size_t)mode * n_out * W + i] = qn;
            }
        }
        return;
    }
    const double k = kmodes[mode];
    const double* tout = tau_out;
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);

    if (warp == 0) {
        // ---- forward: solve, publish every accepted step ----
        ModeMem M = carve(fmem, D);
        for (int i = tm.lane; i < n; i += 32) M.y[i] = y0[(size_t)mode * n + i];
        double swm[3] = {sw[3 * mode], sw[3 * mode + 1], sw[3 * mode + 2]};
        tm.sync();
        int m = 0;
        auto accept = [&](double t, double h, double tnext, int regime) -> bool {
            const int sl = m % ns;
            if (m >= ns && !wait_at_least(tm, vf + 2 + sl, nd * (m / ns), vf + 6, poll_budget(ctrl))) return false;
            double* dst = slot0 + sl * spart;
            if (Split)
                for (int i = tm.lane; i < gpart; i += 32) gslot[i] = fmem[i];
            for (int i = tm.lane; i < mem_doubles - gpart; i += 32) dst[i] = fmem[gpart + i];
            if (tm.leader()) {
                dst[spart - 4] = t;
                dst[spart - 3] = h;
                dst[spart - 2] = tnext;
                dst[spart - 1] = (double)regime;
            }
            tm.sync();
            if (tm.leader()) {
                __threadfence_block();
                vf[sl] = m + 1;
            }
            tm.sync();
            ++m;
            return true;
        };
        auto no_emit = [&](int, const double*, int) {};
        const SolveResult R = solve_mode(tm, *P, D, ctrl, k, tau_start[mode], swm, n_out, tout, M, no_emit,
                                         (const DiscoebTangent*)nullptr, (const TanMem*)nullptr, (double*)nullptr, 0,
                                         &accept);
        if (tm.leader()) {
            vf[5] = m;
            __threadfence_block();
            vf[4] = 1;
            if (grp == 0) {
                status[mode] = R.status;
                nsteps[mode] = R.steps;
            }
        }
        return;
    }

    // ---- tangent of direction d0 + warp - 1 ----
    const int dl = warp - 1, dir = d0 + dl;
    const DiscoebTangent* TN = TNs + dl;
    double* mine = twork + (size_t)dl * per_tan;
    const TanMem TT = carve_tan(mine, D);
    double* ubuf = mine + tan_doubles;
    double* yend = ubuf + n;
    double* pf = yend + n;
    for (int i = tm.lane; i < n; i += 32) TT.yd[i] = y0_dot[((size_t)dir * n_modes + mode) * n + i];
    tm.sync();
    int hint = P->xe_loga.n_knots / 2, iout = 0;
    const long long budget = poll_budget(ctrl);
    for (int m = 0;; ++m) {
        const int sl = m % ns;
        // the next step, unless the forward has finished with fewer steps
        int have = 0;
        if (tm.leader()) {
            long long polls = 0;
            while (true) {
                if (vf[sl] == m + 1) { have = 1; break; }
                if (vf[4] && vf[5] <= m) break;
                if (vf[6]) break;
                if (++polls > budget) { vf[6] = 1; break; }
                __nanosleep(100);
            }
            __threadfence_block();
        }
        if (!__shfl_sync(0xffffffffu, have, 0)) break;
        const double* r = slot0 + sl * spart;
        ModeMem Mr = Split ? carve_split(gslot, const_cast<double*>(r), D) : carve(const_cast<double*>(r), D);
        Mr.u = ubuf;
        const double t = r[spart - 4], h = r[spart - 3], tnext = r[spart - 2];
        const int regime = (int)r[spart - 1];
        tangent_step(tm, *P, D, k, t, h, regime, Mr, TT, TN, hint);
        for (int i = tm.lane; i < n; i += 32) yend[i] = ubuf[i] + Mr.K[7 * n + i];
        tm.sync();
        if (tm.leader()) {
            __threadfence_block();
            atomicAdd(flags + 2 + sl, 1);  // the record may be overwritten from here on
        }
        tm.sync();
        while (iout < n_out && tout[iout] <= tnext) {
            emit_tangent_output<Full>(tm, *P, TN, D, k, mode, dir, n_modes, n_out, iout, tout, tau_out_dot, yend,
                                      regime, TT, pf, y_out20, y_out20_dot);
            ++iout;
        }
    }
    constexpr int W20 = 20;
    const int W = Full ? n : W20;
    for (int j = iout; j < n_out; ++j) {
        const size_t oo = (size_t)mode * n_out + j;
        for (int i = tm.lane; i < W; i += 32) {
            y_out20_dot[((size_t)dir * n_modes * n_out + oo) * W + i] = qnan;
            if (dir == 0 && y_out20) y_out20[oo * W + i] = qnan;
        }
    }
    tm.sync();
}

__global__ void rhs_kernel(const DiscoebCosmo* __restrict__ cosmo, int n_points, const double* __restrict__ tau,
                           const double* __restrict__ kmodes, const double* __restrict__ y, int regime, double* f)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= n_points) return;
    const WarpTeam tm{(int)(threadIdx.x & 31)};
    const DiscoebCosmo& P = *cosmo;
    const Dims D = make_dims(P);
    const double* yy = y + (size_t)warp * D.n;
    Bg<double> b;
    bg_eval(P, yy[0], tau[warp], kmodes[warp], regime, b);
    rhs_team(tm, P, D, b, kmodes[warp], tau[warp], yy, f + (size_t)warp * D.n, (double*)nullptr);
}

int validate_cosmo(const DiscoebCosmo* c)
{
    if (!c) return DISCOEB_EINVAL;
    if (c->nqmax < 0 || c->nqmax > DISCOEB_MAX_NQ) return DISCOEB_EINVAL;
    if (c->lmaxg < 3 || c->lmaxgp < 3 || c->lmaxr < 3 || c->lmaxnu < 3) return DISCOEB_EINVAL;
    if (c->use_tca) return DISCOEB_EUNSUPPORTED;
    return DISCOEB_SUCCESS;
}

// Directions per block of discoeb_jvp: as many as fit in shared memory (at most
// kMaxDirsPerBlock; the forward is solved once per block).  With the two step records in shared
// memory (dpb, smem), or in a global workspace (dpb_glob, smem_glob), which is worth its
// records_bytes only when it lets more directions share a block (larger states, e.g. l_max 50).
struct JvpPlan {
    int dpb, dpb_glob, mem, tmem;
    size_t smem, smem_glob;
    int64_t records_bytes;  // recommended: the split form's workspace where it adds directions, else 0
    int64_t split_bytes;    // the split form's workspace (a caller may ask for it anyway)
};

JvpPlan jvp_plan(const DiscoebCosmo& c0, int n_dir, int n_modes)
{
    JvpPlan p{};
    const Dims D = make_dims(c0);
    p.mem = mode_mem_doubles(D);
    p.tmem = tan_mem_doubles(D);
    int dev = 0, max_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        p.dpb = -1;
        return p;
    }
    // shared doubles: cosmology, tangents, forward workspace, the records' shared parts (two
    // whole records, or one record's factorisation and scalars), the tangent warps' workspaces
    auto bytes = [&](int d, bool glob) {
        const size_t recs = glob ? (size_t)(p.mem + 4 - 13 * D.n) : 2 * (size_t)(p.mem + 4);
        return (size_t)(kCosmoDoubles + d * kTanDoubles + p.mem + recs + d * (p.tmem + 3 * D.n)) * sizeof(double) +
               8 * sizeof(int);
    };
    const int want = n_dir < kMaxDirsPerBlock ? n_dir : kMaxDirsPerBlock;
    auto fit = [&](bool glob) {
        int d = want;
        while (d > 1 && bytes(d, glob) > (size_t)max_optin) --d;
        return bytes(d, glob) <= (size_t)max_optin ? d : 0;
    };
    p.dpb = fit(false);
    p.dpb_glob = fit(true);
    p.smem = bytes(p.dpb > 0 ? p.dpb : 1, false);
    p.smem_glob = bytes(p.dpb_glob > 0 ? p.dpb_glob : 1, true);
    if (p.dpb_glob > 0) {
        const long long blocks = (long long)n_modes * ((n_dir + p.dpb_glob - 1) / p.dpb_glob);
        p.split_bytes = blocks * 13LL * D.n * (int64_t)sizeof(double);
    }
    if (p.dpb_glob > p.dpb) p.records_bytes = p.split_bytes;
    return p;
}

template <bool Full>
int32_t launch_jvp(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                   const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                   const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                   const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                   const double* tau_out, const double* tau_out_dot, double* y_out, double* y_out_dot,
                   int32_t* status, int32_t* nsteps, double* records, int64_t records_bytes, void* stream)
{
    int rc = validate_cosmo(cosmo0_host);
    if (rc) return rc;
    if (!cosmos_dev || !ctrl || !tangents_dev || n_cosmo < 1 || n_dir < 1 || n_modes < 0 || n_out < 1)
        return DISCOEB_EINVAL;
    if (n_modes == 0) return DISCOEB_SUCCESS;
    if (!kmodes || !tau_start || !y0 || !y0_dot || !switch_tau || !tau_out || !tau_out_dot || !y_out_dot ||
        !status || !nsteps)
        return DISCOEB_EINVAL;
    if (ctrl->method != DISCOEB_METHOD_RODAS5_STRUCTURED) return DISCOEB_EUNSUPPORTED;
    if (!(ctrl->rtol > 0.0) || !(ctrl->atol >= 0.0) || ctrl->max_steps < 1) return DISCOEB_EINVAL;
    const JvpPlan plan = jvp_plan(*cosmo0_host, n_dir, n_modes);
    if (plan.dpb < 0) return DISCOEB_ECUDA;
    // the split record is used when the caller passes room for it (discoeb_jvp_records_bytes
    // recommends it where it lets more directions share a block; a caller may pass it anyway)
    const bool glob = plan.dpb_glob >= plan.dpb && plan.split_bytes > 0 && records && records_bytes >= plan.split_bytes;
    if (!glob && plan.dpb == 0) return DISCOEB_EUNSUPPORTED;
    const int dpb = glob ? plan.dpb_glob : plan.dpb;
    const size_t smem = glob ? plan.smem_glob : plan.smem;
    const int mem = plan.mem, tmem = plan.tmem;
    auto kernel = glob ? jvp_block_kernel<Full, true> : jvp_block_kernel<Full, false>;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DISCOEB_ECUDA;
    const long long blocks = (long long)n_modes * ((n_dir + dpb - 1) / dpb);
    if (blocks > 0x7fffffffLL) return DISCOEB_EINVAL;
    kernel<<<(unsigned)blocks, 32 * (1 + dpb), smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        cosmos_dev, n_cosmo, mode_cosmo, tangents_dev, n_dir, dpb, *ctrl, n_modes, kmodes, tau_start, y0, y0_dot,
        switch_tau, n_out, tau_out, tau_out_dot, mem, tmem, glob ? records : nullptr, y_out, y_out_dot, status,
        nsteps);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

}  // namespace

extern "C" {

int32_t discoeb_abi_version(void) { return DISCOEB_ABI_VERSION; }

int32_t discoeb_nvar(const DiscoebCosmo* cosmo)
{
    if (!cosmo) return DISCOEB_EINVAL;
    return make_dims(*cosmo).n;
}

int32_t discoeb_fwd(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const DiscoebControl* ctrl, int32_t n_modes, const int32_t* mode_cosmo, const double* kmodes,
                    const double* tau_start, const double* y0, const double* switch_tau, int32_t n_out,
                    const double* tau_out, double* y_full, double* y_out20, int32_t* status, int32_t* nsteps,
                    void* stream)
{
    int rc = validate_cosmo(cosmo0_host);
    if (rc) return rc;
    if (!cosmos_dev || !ctrl || n_cosmo < 1 || n_modes < 0 || n_out < 1) return DISCOEB_EINVAL;
    if (n_modes == 0) return DISCOEB_SUCCESS;
    if (!kmodes || !tau_start || !y0 || !switch_tau || !tau_out || !status || !nsteps) return DISCOEB_EINVAL;
    if (!y_full && !y_out20) return DISCOEB_EINVAL;
    const bool mixed = ctrl->method == DISCOEB_METHOD_RODAS5_STRUCTURED_MIXED;
    if (ctrl->method != DISCOEB_METHOD_RODAS5_STRUCTURED && !mixed) return DISCOEB_EUNSUPPORTED;
    if (!(ctrl->rtol > 0.0) || !(ctrl->atol >= 0.0) || ctrl->max_steps < 1) return DISCOEB_EINVAL;
    const Dims D = make_dims(*cosmo0_host);
    const int mem = mode_mem_doubles(D), mix = mixed ? mixed_mem_doubles(D) : 0;
    const size_t per_warp = (size_t)(kCosmoDoubles + mem + mix) * sizeof(double);
    const auto kernel = mixed ? fwd_structured_kernel<WarpTeamMixed> : fwd_structured_kernel<WarpTeam>;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DISCOEB_ECUDA;
    int max_optin = 0, n_sm = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    int wpb = ctrl->warps_per_block > 0 ? ctrl->warps_per_block : 1;  // one mode per block: the most resident warps
    if (wpb > 8) wpb = 8;
    while (wpb > 1 && per_warp * wpb > (size_t)max_optin) --wpb;
    if (per_warp > (size_t)max_optin) return DISCOEB_EUNSUPPORTED;
    const size_t smem = per_warp * wpb;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DISCOEB_ECUDA;
    int blocks = (n_modes + wpb - 1) / wpb;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    kernel<<<blocks, 32 * wpb, smem, s>>>(cosmos_dev, n_cosmo, mode_cosmo, *ctrl, n_modes, kmodes, tau_start, y0,
                                          switch_tau, n_out, tau_out, mem, mix, y_full, y_out20, status, nsteps);
    (void)n_sm;
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int32_t discoeb_jvp(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev,
                    int32_t n_dir, const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes,
                    const double* tau_start, const double* y0, const double* y0_dot, const double* switch_tau,
                    int32_t n_out, const double* tau_out, const double* tau_out_dot, double* y_out20,
                    double* y_out20_dot, int32_t* status, int32_t* nsteps, void* stream)
{
    return launch_jvp<false>(cosmos_dev, cosmo0_host, n_cosmo, mode_cosmo, tangents_dev, n_dir, ctrl, n_modes, kmodes,
                             tau_start, y0, y0_dot, switch_tau, n_out, tau_out, tau_out_dot, y_out20, y_out20_dot,
                             status, nsteps, nullptr, 0, stream);
}

int32_t discoeb_jvp_full(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                         const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                         const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                         const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                         const double* tau_out, const double* tau_out_dot, double* y_full, double* y_full_dot,
                         int32_t* status, int32_t* nsteps, void* stream)
{
    return launch_jvp<true>(cosmos_dev, cosmo0_host, n_cosmo, mode_cosmo, tangents_dev, n_dir, ctrl, n_modes, kmodes,
                            tau_start, y0, y0_dot, switch_tau, n_out, tau_out, tau_out_dot, y_full, y_full_dot,
                            status, nsteps, nullptr, 0, stream);
}

int64_t discoeb_jvp_records_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_dir, int32_t n_modes)
{
    if (validate_cosmo(cosmo0_host) || n_dir < 1 || n_modes < 0) return DISCOEB_EINVAL;
    const JvpPlan plan = jvp_plan(*cosmo0_host, n_dir, n_modes);
    return plan.dpb < 0 ? (int64_t)DISCOEB_ECUDA : plan.records_bytes;
}

int64_t discoeb_jvp_split_records_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_dir, int32_t n_modes)
{
    if (validate_cosmo(cosmo0_host) || n_dir < 1 || n_modes < 0) return DISCOEB_EINVAL;
    const JvpPlan plan = jvp_plan(*cosmo0_host, n_dir, n_modes);
    return plan.dpb < 0 ? (int64_t)DISCOEB_ECUDA : plan.split_bytes;
}

int32_t discoeb_jvp_records(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                            const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                            const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                            const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                            const double* tau_out, const double* tau_out_dot, double* y_out, double* y_out_dot,
                            int32_t* status, int32_t* nsteps, int32_t full, void* records, int64_t records_bytes,
                            void* stream)
{
    if (full != 0 && full != 1) return DISCOEB_EINVAL;
    double* rec = static_cast<double*>(records);
    if (full)
        return launch_jvp<true>(cosmos_dev, cosmo0_host, n_cosmo, mode_cosmo, tangents_dev, n_dir, ctrl, n_modes,
                                kmodes, tau_start, y0, y0_dot, switch_tau, n_out, tau_out, tau_out_dot, y_out,
                                y_out_dot, status, nsteps, rec, records_bytes, stream);
    return launch_jvp<false>(cosmos_dev, cosmo0_host, n_cosmo, mode_cosmo, tangents_dev, n_dir, ctrl, n_modes, kmodes,
                             tau_start, y0, y0_dot, switch_tau, n_out, tau_out, tau_out_dot, y_out, y_out_dot, status,
                             nsteps, rec, records_bytes, stream);
}

int32_t discoeb_rhs(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host, int32_t n_points,
                    const double* tau, const double* kmodes, const double* y, int32_t regime, double* f, void* stream)
{
    int rc = validate_cosmo(cosmo_host);
    if (rc) return rc;
    if (!cosmo_dev || n_points < 0) return DISCOEB_EINVAL;
    if (n_points == 0) return DISCOEB_SUCCESS;
    if (!tau || !kmodes || !y || !f) return DISCOEB_EINVAL;
    const int threads = 128;
    const long long blocks = ((long long)n_points * 32 + threads - 1) / threads;
    rhs_kernel<<<(unsigned)blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(cosmo_dev, n_points, tau,
                                                                                          kmodes, y, regime, f);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

}  // extern "C"
