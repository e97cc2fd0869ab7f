// Test harness: compiles the device model and stepper sources for one host thread so that
// their algebra can be compared with the oracle on a CPU.  Test infrastructure only; the
// library that ships is the CUDA build of the same headers.
#include <cstring>
#include <vector>

#include "stepper.cuh"

using namespace dscb;

template <class Team>
static int wsolve_impl(const DiscoebCosmo* P, double tau, const double* y, double k, int regime, double h,
                       const double* r, double* x)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    std::vector<double> mem(mode_mem_doubles(D) + mixed_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    if (Team::mixed) carve_mixed(mem.data() + mode_mem_doubles(D), D, M);
    Team tm;
    std::memcpy(M.y, y, sizeof(double) * n);
    Bg<Dual> bd;
    bg_eval(*P, Dual(y[0], 1.0), tau, k, regime, bd);
    rhs_team(tm, *P, D, bd, k, tau, M.y, M.f, M.col0);
    Bg<double> b;
    bg_eval(*P, y[0], tau, k, regime, b);
    bool ok = factor_W(tm, *P, D, b, k, tau, h, M);
    std::memcpy(x, r, sizeof(double) * n);
    solve_W(tm, D, M, h, x);
    return ok ? 0 : 1;
}

template <class Team>
static int solve_mode_impl(const DiscoebCosmo* P, const DiscoebControl* C, double k, double t0, const double* y0,
                           const double* sw, int nout, const double* tout, double* yout, int* stats)
{
    const Dims D = make_dims(*P);
    std::vector<double> mem(mode_mem_doubles(D) + mixed_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    if (Team::mixed) carve_mixed(mem.data() + mode_mem_doubles(D), D, M);
    std::memcpy(M.y, y0, sizeof(double) * D.n);
    Team tm;
    const int n = D.n;
    auto emit = [&](int j, const double* y, int) { std::memcpy(yout + (size_t)j * n, y, sizeof(double) * n); };
    SolveResult R = solve_mode(tm, *P, D, *C, k, t0, sw, nout, tout, M, emit);
    stats[0] = R.status;
    stats[1] = R.steps;
    stats[2] = R.accepted;
    return R.status;
}

extern "C" {

int shim_nvar(const DiscoebCosmo* P) { return make_dims(*P).n; }

void shim_rhs(const DiscoebCosmo* P, double tau, const double* y, double k, int regime, double* f, double* col0)
{
    const Dims D = make_dims(*P);
    HostTeam tm;
    Bg<Dual> b;
    bg_eval(*P, Dual(y[0], 1.0), tau, k, regime, b);
    rhs_team(tm, *P, D, b, k, tau, y, f, col0);
}

// dense expansion of the structured Jacobian J = [[j00,0],[c0, S + U G]] (+ row 1) and dT
void shim_jacobian(const DiscoebCosmo* P, double tau, const double* y, double k, int regime, double* J, double* dT)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    std::vector<double> f(n), col0(n);
    shim_rhs(P, tau, y, k, regime, f.data(), col0.data());
    Bg<double> b;
    bg_eval(*P, y[0], tau, k, regime, b);
    std::vector<double> G(3 * n);
    for (int j = 0; j < n; ++j) {
        double g[3];
        gcol(*P, D, b, k, j, g);
        for (int r = 0; r < 3; ++r) G[r * n + j] = g[r];
    }
    std::memset(J, 0, sizeof(double) * n * n);
    for (int i = 0; i < n; ++i) J[i * n] = col0[i];
    double fu[3];
    f1u(*P, b, k, fu);
    for (int j = 2; j < n; ++j) J[n + j] = f1col(*P, D, b, k, j) + fu[0] * G[j] + fu[1] * G[n + j] + fu[2] * G[2 * n + j];
    for (int i = 2; i < n; ++i) {
        double band[7], etac, u[3];
        rowc(*P, D, b, k, tau, i, band, etac, u);
        const int s = row_stride(D, i);
        for (int m = -3; m <= 3; ++m) {
            int jj = i + m * s;
            if (jj >= 0 && jj < n) J[i * n + jj] += band[m + 3];
        }
        J[i * n + 2] += etac;
        for (int j = 1; j < n; ++j) J[i * n + j] += u[0] * G[j] + u[1] * G[n + j] + u[2] * G[2 * n + j];
    }
    for (int i = 0; i < n; ++i) dT[i] = dtau_row(D, b, tau, i, y);
}

// x = W^{-1} r with W = I/(gamma h) - J(t, y), through the structured factorisation
int shim_wsolve(const DiscoebCosmo* P, double tau, const double* y, double k, int regime, double h, const double* r,
                double* x)
{
    return wsolve_impl<HostTeam>(P, tau, y, k, regime, h, r, x);
}

// the same with FP32 chain factors and one FP64 refinement per chain solve
int shim_wsolve_mixed(const DiscoebCosmo* P, double tau, const double* y, double k, int regime, double h,
                      const double* r, double* x)
{
    return wsolve_impl<HostTeamMixed>(P, tau, y, k, regime, h, r, x);
}

// forward + tangent solve: raw state and its tangent at the output times (fixed output times)
int shim_solve_mode_tangent(const DiscoebCosmo* P, const DiscoebTangent* tn, const DiscoebControl* C, double k,
                            double t0, const double* y0, const double* yd0, const double* sw, int nout,
                            const double* tout, double* yout, double* ydout, int* stats, double* tlog, int tlog_cap)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    std::vector<double> mem(mode_mem_doubles(D)), tmem(tan_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    TanMem TT = carve_tan(tmem.data(), D);
    std::memcpy(M.y, y0, sizeof(double) * n);
    std::memcpy(TT.yd, yd0, sizeof(double) * n);
    HostTeam tm;
    auto emit = [&](int j, const double* y, int) {
        std::memcpy(yout + (size_t)j * n, y, sizeof(double) * n);
        std::memcpy(ydout + (size_t)j * n, TT.yd, sizeof(double) * n);
    };
    SolveResult R = solve_mode(tm, *P, D, *C, k, t0, sw, nout, tout, M, emit, tn, &TT, tlog, tlog_cap);
    stats[0] = R.status;
    stats[1] = R.steps;
    stats[2] = R.accepted;
    return R.status;
}

// forward solve replaying a given sequence of step end times (no error control)
int shim_replay(const DiscoebCosmo* P, double k, double t0, const double* y0, const double* sw, int nsteps,
                const double* tsteps, double* yend)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    std::vector<double> mem(mode_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    std::memcpy(M.y, y0, sizeof(double) * n);
    HostTeam tm;
    int hint = P->xe_loga.n_knots / 2;
    double t = t0;
    for (int s = 0; s < nsteps; ++s) {
        const double h = tsteps[s] - t;
        const int regime = regime_at(*P, t, sw);
        rodas5_step(tm, *P, D, k, t, h, regime, M, hint);
        for (int i = 0; i < n; ++i) M.y[i] = M.u[i] + M.K[7 * n + i];
        t = tsteps[s];
    }
    std::memcpy(yend, M.y, sizeof(double) * n);
    return 0;
}

int shim_solve_mode(const DiscoebCosmo* P, const DiscoebControl* C, double k, double t0, const double* y0,
                    const double* sw, int nout, const double* tout, double* yout, int* stats)
{
    return solve_mode_impl<HostTeam>(P, C, k, t0, y0, sw, nout, tout, yout, stats);
}

int shim_solve_mode_mixed(const DiscoebCosmo* P, const DiscoebControl* C, double k, double t0, const double* y0,
                          const double* sw, int nout, const double* tout, double* yout, int* stats)
{
    return solve_mode_impl<HostTeamMixed>(P, C, k, t0, y0, sw, nout, tout, yout, stats);
}

// the 20 output fields and their tangents (output_vars with dual numbers), and the RSA
// projection fields; tn may be null (state tangent only)
void shim_output_tangent(const DiscoebCosmo* P, const DiscoebTangent* tn, double k, double tau, const double* y,
                         const double* yd, double* o, double* od, double* rsa, double* rsad)
{
    const Dims D = make_dims(*P);
    Dual out[20], f[4];
    output_vars<Dual>(*P, tn, D, k, y, yd, out);
    for (int q = 0; q < 20; ++q) { o[q] = out[q].v; od[q] = out[q].d; }
    rsa_projection<Dual>(*P, tn, D, tau, k, y, yd, f);
    for (int q = 0; q < 4; ++q) { rsa[q] = f[q].v; rsad[q] = f[q].d; }
}

// forward solve that records every accepted step, then the tangent replayed from the records
// (the arithmetic of the per-mode block kernel of discoeb_jvp); tangents at the output times
int shim_solve_mode_tangent_records(const DiscoebCosmo* P, const DiscoebTangent* tn, const DiscoebControl* C, double k,
                                    double t0, const double* y0, const double* yd0, const double* sw, int nout,
                                    const double* tout, double* ydout, int* stats)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    std::vector<double> mem(mode_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    std::memcpy(M.y, y0, sizeof(double) * n);
    HostTeam tm;
    const int mem_n = mode_mem_doubles(D);
    std::vector<std::vector<double>> recs;
    std::vector<double> rt, rh, rtn;
    std::vector<int> rr;
    auto accept = [&](double t, double h, double tnext, int regime) {
        recs.emplace_back(mem.begin(), mem.begin() + mem_n);
        rt.push_back(t);
        rh.push_back(h);
        rtn.push_back(tnext);
        rr.push_back(regime);
        return true;
    };
    auto emit = [&](int, const double*, int) {};
    SolveResult R = solve_mode(tm, *P, D, *C, k, t0, sw, nout, tout, M, emit, (const DiscoebTangent*)nullptr,
                               (const TanMem*)nullptr, (double*)nullptr, 0, &accept);
    stats[0] = R.status;
    stats[1] = R.steps;
    stats[2] = R.accepted;
    std::vector<double> tmem(tan_mem_doubles(D));
    TanMem TT = carve_tan(tmem.data(), D);
    std::memcpy(TT.yd, yd0, sizeof(double) * n);
    int hint = P->xe_loga.n_knots / 2, iout = 0;
    for (size_t m = 0; m < recs.size(); ++m) {
        ModeMem Mr = carve(recs[m].data(), D);
        tangent_step(tm, *P, D, k, rt[m], rh[m], rr[m], Mr, TT, tn, hint);
        const double tnew = rtn[m];
        while (iout < nout && tout[iout] <= tnew) {
            std::memcpy(ydout + (size_t)iout * n, TT.yd, sizeof(double) * n);
            ++iout;
        }
    }
    return R.status;
}
}

// the 20 output fields at an output time and their tangents, after the RSA projection (the
// arithmetic of the output stage of the forward and tangent kernels): state y with tangent yd
// (the tangent at the moving output time), parameter tangent tn (may be null)
extern "C" void shim_projected_output_tangent(const DiscoebCosmo* P, const DiscoebTangent* tn, double k, double tau,
                                              const double* y, const double* yd, double* o, double* od)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    Dual fld[4];
    const bool rsa = rsa_projection<Dual>(*P, tn, D, tau, k, y, yd, fld);
    std::vector<double> yp(n), ypd(n);
    for (int i = 0; i < n; ++i) {
        double v = y[i], vd = yd[i];
        if (rsa) {
            const int s = rsa_slot(D, i);
            if (s >= 0) { v = fld[s].v; vd = fld[s].d; }
            else if (s == -1) { v = 0.0; vd = 0.0; }
        }
        yp[i] = v;
        ypd[i] = vd;
    }
    Dual out[20];
    output_vars<Dual>(*P, tn, D, k, yp.data(), ypd.data(), out);
    for (int q = 0; q < 20; ++q) { o[q] = out[q].v; od[q] = out[q].d; }
}
