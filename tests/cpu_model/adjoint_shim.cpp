// Test harness: the discrete adjoint (adjoint.cuh) compiled for one host thread, next to the
// forward-mode tangent of the same steps, so that the two can be checked against each other on a
// CPU.  Test infrastructure only; the library that ships is the CUDA build of the same headers.
#include <cstring>
#include <vector>

#include "adjoint.cuh"

using namespace dscb;

extern "C" {

// One Rodas5 step from (t, y) with size h in a fixed regime: the tangent yd1 of the step's result
// along (yd, tn), and the reverse of the same step, lam1 (cotangent of the result) -> lam0 (of y),
// pbar [16] (parameters, by seed index) and tbar [8][tstride] (table knots, accumulated).
int shim_adjoint_step(const DiscoebCosmo* P, const DiscoebTangent* tn, double k, double t, double h, int regime,
                      const double* y, const double* yd, const double* lam1, double* y1, double* yd1, double* lam0,
                      double* pbar, double* tbar, int tstride)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    HostTeam tm;
    int hint = P->xe_loga.n_knots / 2;
    std::vector<double> mem(mode_mem_doubles(D)), tmem(tan_mem_doubles(D)), amem(adj_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    TanMem TT = carve_tan(tmem.data(), D);
    AdjMem A = carve_adj(amem.data(), D);
    std::memcpy(M.y, y, sizeof(double) * n);
    std::memcpy(TT.yd, yd, sizeof(double) * n);
    const bool ok = rodas5_step(tm, *P, D, k, t, h, regime, M, hint, tn, &TT);
    for (int i = 0; i < n; ++i) {
        y1[i] = M.u[i] + M.K[7 * n + i];
        yd1[i] = TT.ud[i] + TT.Kd[7 * n + i];
    }
    // the reverse: recompute the step keeping U, then one adjoint step
    std::memcpy(M.y, y, sizeof(double) * n);
    rodas5_step(tm, *P, D, k, t, h, regime, M, hint, (const DiscoebTangent*)nullptr, (const TanMem*)nullptr, A.Uk);
    make_Zt(tm, D, M, h, A.Zt);
    std::memcpy(A.lam, lam1, sizeof(double) * n);
    for (int q = 0; q < 16; ++q) A.pb[q] = 0.0;
    for (int q = 0; q < kNTabSeeds; ++q) {
        A.tab[q].cur = -1;
        A.tab[q].w = 0.0;
    }
    double l0 = lam1[0];
    adjoint_step(tm, *P, D, k, t, h, regime, M, A, A.Uk, A.Zt, A.rec, A.as, 0.0, hint);
    achain_step(tm, *P, D, k, A.rec, A.as, l0, A.scr);
    deferred_records(tm, *P, D, k, A.rec, 0, kRecPerStep, A.g, DefAcc{A.pb, A.tab}, tbar, tstride);
    A.lam[0] = l0;
    for (int xs = X_KNOT0; xs < X_KNOT0 + kNTabSeeds; ++xs) tab_flush(A.tab[xs - X_KNOT0], xs, tbar, tstride);
    std::memcpy(lam0, A.lam, sizeof(double) * n);
    for (int q = 0; q < 16; ++q) pbar[q] = A.pb[q];
    return ok ? 0 : 1;
}

// Forward solve recording its accepted steps (end times tlog [cap], every-th start states ckpt),
// with the 20 output fields at the output times; stats = (status, step attempts, accepted)
int shim_fwd_record(const DiscoebCosmo* P, const DiscoebControl* C, double k, double t0, const double* y0,
                    const double* sw, int nout, const double* tout, int cap, int every, double* tlog, double* ckpt,
                    double* y20, int* stats)
{
    const Dims D = make_dims(*P);
    const int n = D.n;
    HostTeam tm;
    std::vector<double> mem(mode_mem_doubles(D));
    ModeMem M = carve(mem.data(), D);
    std::memcpy(M.y, y0, sizeof(double) * n);
    Recorder<HostTeam> rec{&tm, &M, tlog, ckpt, cap, every, n, 0};
    std::vector<double> yp(n);
    auto emit = [&](int j, const double* y, int) {
        double fld[4];
        const bool rsa = rsa_projection<double>(*P, nullptr, D, tout[j], k, y, nullptr, fld);
        for (int i = 0; i < n; ++i) {
            double v = y[i];
            if (rsa) {
                const int s = rsa_slot(D, i);
                if (s >= 0) v = fld[s];
                else if (s == -1) v = 0.0;
            }
            yp[i] = v;
        }
        output_vars<double>(*P, nullptr, D, k, yp.data(), nullptr, y20 + (size_t)j * 20);
    };
    SolveResult R = solve_mode(tm, *P, D, *C, k, t0, sw, nout, tout, M, emit, (const DiscoebTangent*)nullptr,
                               (const TanMem*)nullptr, (double*)nullptr, 0, &rec);
    stats[0] = R.status;
    stats[1] = R.steps;
    stats[2] = rec.count;
    return R.status;
}

// Reverse sweep of one recorded mode: ob [nout][20] -> y0bar [n], toutbar [nout], pbar [8]
// (DiscoebTangent's scalar order), tbar [8][tstride] (accumulated)
int shim_bwd_mode(const DiscoebCosmo* P, double k, double t0, const double* sw, int nout, const double* tout,
                  const double* tlog, const double* ckpt, int every, int nacc, const double* ob, double* y0bar,
                  double* toutbar, double* pbar, double* tbar, int tstride)
{
    const Dims D = make_dims(*P);
    HostTeam tm;
    std::vector<double> mem(mode_mem_doubles(D)), amem(adj_mem_doubles(D)), seg((size_t)every * D.n);
    ModeMem M = carve(mem.data(), D);
    AdjMem A = carve_adj(amem.data(), D);
    bwd_mode(tm, *P, D, k, t0, sw, nout, tout, tlog, ckpt, every, nacc, seg.data(), ob, M, A, y0bar, toutbar, tbar,
             tstride);
    for (int q = 0; q < 8; ++q) pbar[q] = A.pb[X_GRHOM + q];
    return 0;
}

}  // extern "C"
