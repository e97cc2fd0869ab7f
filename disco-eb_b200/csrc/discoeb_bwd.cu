// Discrete adjoint on sm_100a: the recording forward solve, the reverse sweep and the contraction
// of the cotangents with parameter tangents; C ABI (include/discoeb.h).
//
// Layout: one warp per k-mode.  The recording forward is the forward solve whose accept hook
// writes each accepted step's end time (8 bytes) and every checkpoint_every-th start state into
// the caller's record buffer.  The reverse sweep holds its cosmology, the recomputed step (state,
// stages, factorisation) and the adjoint workspace in shared memory (42 n doubles: one warp per
// block, four blocks per SM at n = 143), recomputes each segment of checkpoint_every steps from
// its checkpoint into the caller's workspace, and takes it apart step by step.  Table-knot
// cotangents are summed over the modes of a cosmology with double-precision atomics (the order of
// those additions is not fixed, so they agree between runs to rounding, not bit for bit).
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

__global__ void __launch_bounds__(32) bwd_kernel(
    const DiscoebCosmo* __restrict__ cosmos, int n_cosmo, const int32_t* __restrict__ mode_cosmo, int n_modes,
    const double* __restrict__ kmodes, const double* __restrict__ tau_start, const double* __restrict__ sw, int n_out,
    const double* __restrict__ tau_out, int cap, int every, long long rec_doubles, const double* __restrict__ records,
    const int32_t* __restrict__ n_acc, const int32_t* __restrict__ fwd_status, double* seg,
    const double* __restrict__ ybar20, int mem_doubles, int adj_doubles, double* y0_bar, double* tau_out_bar,
    double* par_bar, double* table_bar, int tstride, int table_per_mode, int32_t* status)
{
    extern __shared__ double smem[];
    const WarpTeam tm{(int)(threadIdx.x & 31)};
    const int mode = blockIdx.x;
    if (mode >= n_modes) return;
    DiscoebCosmo* P = reinterpret_cast<DiscoebCosmo*>(smem);
    double* wmem = smem + kCosmoDoublesB;
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    const int ci = mode_cosmo ? mode_cosmo[mode] : 0;
    int st = fwd_status[mode];
    if (ci < 0 || ci >= n_cosmo) st = DISCOEB_BAD_INDEX;
    if (st == DISCOEB_OK) {
        copy_cosmo_warp(tm, cosmos + ci, P);
        if (mode_mem_doubles(make_dims(*P)) != mem_doubles || adj_mem_doubles(make_dims(*P)) != adj_doubles)
            st = DISCOEB_BAD_INDEX;
    }
    const int n = (mem_doubles - 4 * kMaxSlots - 32) / 23;  // state size of the launch (mode_mem_doubles)
    if (st != DISCOEB_OK) {  // no forward to take apart: report, write NaN
        for (int i = tm.lane; i < n; i += 32) y0_bar[(size_t)mode * n + i] = qnan;
        for (int j = tm.lane; j < n_out; j += 32) tau_out_bar[(size_t)mode * n_out + j] = qnan;
        for (int q = tm.lane; q < 8; q += 32) par_bar[(size_t)mode * 8 + q] = qnan;
        if (tm.leader()) status[mode] = st;
        return;
    }
    const Dims D = make_dims(*P);
    ModeMem M = carve(wmem, D);
    AdjMem A = carve_adj(wmem + mem_doubles, D);
    const double* rec = records + (size_t)mode * rec_doubles;
    bwd_mode(tm, *P, D, kmodes[mode], tau_start[mode], sw + 3 * mode, n_out, tau_out + (size_t)ci * n_out, rec,
             rec + cap, every, n_acc[mode], seg + (size_t)mode * every * n, ybar20 + (size_t)mode * n_out * 20, M, A,
             y0_bar + (size_t)mode * n, tau_out_bar + (size_t)mode * n_out,
             table_bar + (size_t)(table_per_mode ? mode : ci) * 8 * tstride, tstride);
    for (int q = tm.lane; q < 8; q += 32) par_bar[(size_t)mode * 8 + q] = A.pb[X_GRHOM + q];
    if (tm.leader()) status[mode] = DISCOEB_OK;
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
    return (int64_t)n_modes * checkpoint_every * make_dims(*cosmo0_host).n * (int64_t)sizeof(double);
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
    const int mem = mode_mem_doubles(D), adj = adj_mem_doubles(D);
    const size_t smem = (size_t)(kCosmoDoublesB + mem + adj) * sizeof(double);
    int dev = 0, max_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DISCOEB_ECUDA;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > (size_t)max_optin) return DISCOEB_EUNSUPPORTED;
    if (cudaFuncSetAttribute(bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DISCOEB_ECUDA;
    const long long rec = record_doubles(D.n, step_capacity, checkpoint_every);
    bwd_kernel<<<n_modes, 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        cosmos_dev, n_cosmo, mode_cosmo, n_modes, kmodes, tau_start, switch_tau, n_out, tau_out, step_capacity,
        checkpoint_every, rec, records, n_accepted, fwd_status, static_cast<double*>(workspace), y_out20_bar, mem, adj,
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
