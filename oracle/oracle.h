/*
 * CPU oracle for the per-k-mode linear perturbation solve: TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C float64 restatement of the reference's algorithm, used by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the checker.
 * Nothing in the shipped library links or calls it.
 *
 * Restated reference functions (paths relative to the reference project):
 *   model_synchronous           src/discoeb/perturbations.py:88-525
 *   nu_perturb                  src/discoeb/perturbations.py:29-57
 *   convert_to_output_variables src/discoeb/perturbations.py:528-677
 *   adiabatic_ics_one_mode      src/discoeb/perturbations.py:680-781
 *   determine_starting_time     src/discoeb/perturbations.py:784-835, util.py:249-280
 *   rms_norm_filtered(_batched) src/discoeb/perturbations.py:844-878
 *   approximations             src/discoeb/approximations.py:9-176
 *   get_aprimeoa                src/discoeb/background.py:101-123
 *   spline evaluate/derivative  src/discoeb/spline_interpolation.py:132-228
 *   Rodas5Transformed.step      src/discoeb/ode_integrators_stiff.py:680-892
 *   Rodas5Batched.step          src/discoeb/ode_integrators_stiff.py:904-1059
 * and diffrax's PIDController / SaveAt(ts) / LocalLinearInterpolation (third-party,
 * not part of the reference tree) from their documented behaviour.
 */
#ifndef DISCOEB_ORACLE_H
#define DISCOEB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_NQ 64

typedef struct {
    int n;           /* number of knots */
    int uniform;     /* 1: O(1) index from (x - x0)/dx */
    const double* x;
    const double* y;
    const double* S; /* second derivatives at the knots */
} OracleSpline;

typedef struct {
    int n, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax;
    int use_tca, use_rsa, use_ufa;
    double tca_tau_c_over_tau_h, tca_tau_c_over_tau_k;
    double rsa_tau_c_over_tau, rsa_tau_over_tau_k, ufa_tau_over_tau_k;
    double grhom, grhog, grhor, Omegam, Omegab, OmegaDE, Omegak, Neff, Nmnu, amnu;
    double w0, wa, cs2_DE, YHe, H0, taumin;
    double de_guard_eps; /* 0: literal reference (NaN at w=-1); >0 freeze DE when |1+w|<eps */
    double q[ORACLE_MAX_NQ], w[ORACLE_MAX_NQ];
    OracleSpline xe_loga, cs2a_loga, logrhonu_loga, logpnu_loga;
    OracleSpline a_of_tau, xe_of_tau, tau_of_a;
} OracleProblem;

typedef struct {
    double rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin;
    int max_steps;
    int linear_interp;   /* 1: diffrax SaveAt(ts)+LocalLinearInterpolation, no clipping */
    int literal_regime;  /* 1: approximation switches evaluated per RHS call */
} OracleControl;

typedef struct {
    int steps, accepted, rejected, status; /* status 0 ok, 1 max_steps, 2 nonfinite */
} OracleStats;

int oracle_nvar(const OracleProblem* P);
/* f = RHS(tau, y); regime < 0: literal switches, else bitmask 1=RSA 2=UFA 4=TCA */
void oracle_rhs(const OracleProblem* P, double tau, const double* y, double k, double* f, int regime);
/* dense Jacobian J[n*n] (row-major) and explicit time derivative dT[n] */
void oracle_jacobian(const OracleProblem* P, double tau, const double* y, double k, double* J, double* dT,
                     int regime);
double oracle_start_time(const OracleProblem* P, double k);
void oracle_ics(const OracleProblem* P, double tau, double k, double* y);
void oracle_rsa_project(const OracleProblem* P, double tau, double k, const double* y, double* out);
void oracle_output_vars(const OracleProblem* P, double k, const double* y, double* out20);
int oracle_regime(const OracleProblem* P, double tau, const double* sw);
/* switch times sw[3] = {tau_rsa, tau_ufa, tau_tca_end} (inf when absent) */
void oracle_switch_times(const OracleProblem* P, double k, double* sw);

/* Integrate nb modes from t0 (shared) to max(tout).  nb > 1 shares the step size and
 * the error norm across the batch as the reference's Rodas5Batched path does.
 * y0[nb*n]; yout[nb*nout*n] (raw state, no projection); sw[nb*3] switch times
 * (used when !literal_regime).  Returns 0 ok, else status. */
int oracle_solve(const OracleProblem* P, const OracleControl* C, int nb, const double* k, double t0,
                 const double* y0, int nout, const double* tout, const double* sw, double* yout,
                 OracleStats* st);

#ifdef __cplusplus
}
#endif
#endif
