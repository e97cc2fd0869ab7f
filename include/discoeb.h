/*
 * discoeb_b200 C ABI: the drop-in boundary of the per-k-mode linear perturbation solve.
 *
 * Plain C types only.  All array pointers passed to discoeb_fwd / discoeb_los are DEVICE
 * pointers owned by the caller (torch tensors, XLA FFI buffers, cudaMalloc'd memory);
 * `stream` is a cudaStream_t passed as void*.  Calls are stream-ordered and re-entrant;
 * the library keeps no per-call state.
 *
 * Interfaces replaced (paths relative to the reference project, lawrenceberry/DISCO-EB):
 *   discoeb_fwd    -> evolve_one_mode / evolve_perturbations / evolve_perturbations_batched
 *                     (src/discoeb/perturbations.py:882-949, :1124-1226, :1229-1337):
 *                     the diffrax solve with Rodas5 + PIDController + SaveAt(ts),
 *                     the RSA output projection (src/discoeb/approximations.py:84-176)
 *                     and convert_to_output_variables (src/discoeb/perturbations.py:528-677).
 *                     Start times and adiabatic initial conditions
 *                     (perturbations.py:680-835) stay in the caller's host code so that
 *                     automatic differentiation can flow through them.
 *   discoeb_rhs    -> model_synchronous (src/discoeb/perturbations.py:88-525) evaluated at
 *                     given states, i.e. compute_time_derivatives (perturbations.py:1339-1406).
 *   discoeb_background -> evolve_background (src/discoeb/background.py:191-345) with
 *                     thermo_module='RECFAST' (src/discoeb/thermodynamics_recfast.py:124-492),
 *                     and its parameter derivatives: host memory, host code (the producer of
 *                     the solve's tables, not a device entry point).
 */
#ifndef DISCOEB_B200_H
#define DISCOEB_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DISCOEB_MAX_NQ 16
#define DISCOEB_ABI_VERSION 1

/* Natural cubic spline table (x, y, S = y'' at the knots), the format of the reference's
 * spline_interpolation (src/discoeb/spline_interpolation.py:6-116).  Device pointers. */
typedef struct {
    int32_t n_knots;
    int32_t uniform; /* 1: knots equally spaced, index = floor((x - x0)/dx) */
    const double* x;
    const double* y;
    const double* S;
} DiscoebSpline;

/* One cosmology: scalar parameters of the param dict (background.py:141-189), the
 * neutrino momentum quadrature (background.py:14-45) and the four tables the RHS reads. */
typedef struct {
    int32_t lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax;
    int32_t use_tca, use_rsa, use_ufa;
    double tca_tau_c_over_tau_h, tca_tau_c_over_tau_k;
    double rsa_tau_c_over_tau, rsa_tau_over_tau_k, ufa_tau_over_tau_k;
    double grhom, grhog, grhor, Omegam, Omegab, OmegaDE, Omegak, Neff, Nmnu, amnu;
    double w0, wa, cs2_DE, YHe, H0;
    /* 0: reference equations (NaN at w = -1 exactly); > 0: dark-energy perturbations are
     * held constant where |1 + w(a)| < de_guard_eps (the cosmological-constant limit). */
    double de_guard_eps;
    double q[DISCOEB_MAX_NQ], wq[DISCOEB_MAX_NQ];
    DiscoebSpline xe_loga, cs2a_loga, logrhonu_loga, logpnu_loga;
} DiscoebCosmo;

/* Tangent of one cosmology along one parameter direction: the derivatives of the scalar
 * parameters the solve reads and of the (y, S) arrays of the four spline tables (the knots do
 * not depend on the parameters).  Device pointers; NULL arrays mean zero. */
typedef struct {
    double grhom, Omegam, Omegab, OmegaDE, amnu, w0, wa, H0;
    const double *xe_y, *xe_S, *cs2a_y, *cs2a_S, *logrhonu_y, *logrhonu_S, *logpnu_y, *logpnu_S;
} DiscoebTangent;

/* Step control: diffrax PIDController fields (perturbations.py:913-914, :1124-1128). */
typedef struct {
    double rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin;
    int32_t max_steps;
    int32_t method;       /* DISCOEB_METHOD_* */
    int32_t warps_per_block;
    /* Poll budget of every wait between cooperating warps of one mode (discoeb_jvp): a warp that
     * polls a hand-over counter this many times without progress stops the mode with
     * DISCOEB_ABORTED instead of waiting on.  <= 0: the library default, 2^24 polls of ~100 ns
     * (about 2 s; one step takes well under a millisecond). */
    int32_t max_polls;
} DiscoebControl;

#define DISCOEB_METHOD_RODAS5_STRUCTURED 0 /* default: banded-chain + rank-3 LU, FP64 */
#define DISCOEB_METHOD_RODAS5_DENSE 1      /* dense partial-pivot LU per mode, FP64 */
#define DISCOEB_METHOD_RODAS5_DENSE_MIXED 2/* dense FP32 LU + FP64 residual refinement */
/* the structured form with the chain factors in FP32 and one FP64 residual refinement of every
 * chain solve (discoeb_fwd only; the gradient and adjoint entries answer DISCOEB_EUNSUPPORTED) */
#define DISCOEB_METHOD_RODAS5_STRUCTURED_MIXED 3

/* per-mode status codes */
#define DISCOEB_OK 0
#define DISCOEB_MAX_STEPS 1
#define DISCOEB_NONFINITE 2 /* the state or the Jacobian at a step start is not finite (a NaN or an
                             * infinity in an input table, say): no step size can help */
#define DISCOEB_DT_UNDERFLOW 3
#define DISCOEB_SINGULAR 4
#define DISCOEB_BAD_INDEX 5 /* mode_cosmo[mode] outside [0, n_cosmo), or that cosmology's l_max / nq
                              * differ from cosmos[0]'s: the mode was not solved */
#define DISCOEB_ABORTED 6   /* the solve stopped because a cooperating warp of the same mode gave up */
#define DISCOEB_RECORD_FULL 7 /* discoeb_fwd_record: the mode took more accepted steps than its record holds */

/* return codes of the entry points */
#define DISCOEB_SUCCESS 0
#define DISCOEB_EINVAL -1
#define DISCOEB_ECUDA -2
#define DISCOEB_EUNSUPPORTED -3

int32_t discoeb_abi_version(void);

/* Number of state variables per mode: 7 + (lmaxg+1) + (lmaxgp+1) + (lmaxr+1)
 * + nqmax*(lmaxnu+1) + 2 (perturbations.py:893). */
int32_t discoeb_nvar(const DiscoebCosmo* cosmo);

/* Forward solve of n_modes k-modes.
 *   cosmos[n_cosmo]        device array of DiscoebCosmo (tables inside are device pointers); all
 *                          with the l_max / nqmax of cosmo0_host (a host copy of cosmos[0])
 *   mode_cosmo[n_modes]    cosmology index per mode (NULL: all 0)
 *   kmodes, tau_start      [n_modes]
 *   y0                     [n_modes, nvar]   initial states (adiabatic ICs)
 *   switch_tau             [n_modes, 3]      times where RSA starts, UFA starts, TCA ends
 *                                            (+inf when never); steps end exactly there
 *   tau_out                [n_cosmo, n_out] increasing output times of each cosmology (a row per
 *                          cosmology: the same scale factors map to different times)
 *   y_full                 [n_modes, n_out, nvar] state at tau_out after the RSA projection
 *                          (may be NULL)
 *   y_out20                [n_modes, n_out, 20] output fields (may be NULL)
 *   status, nsteps         [n_modes] per-mode status code and number of step attempts
 * All modes of all cosmologies run in one launch (jax.vmap over cosmologies of the reference's
 * evolve_perturbations maps onto n_cosmo / mode_cosmo). */
int32_t discoeb_fwd(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const DiscoebControl* ctrl, int32_t n_modes, const int32_t* mode_cosmo,
                    const double* kmodes, const double* tau_start, const double* y0,
                    const double* switch_tau, int32_t n_out, const double* tau_out,
                    double* y_full, double* y_out20, int32_t* status, int32_t* nsteps, void* stream);

/* Forward solve plus tangents along n_dir parameter directions, for gradients with respect to
 * cosmological parameters (replaces jax.jacfwd through diffeqsolve with DirectAdjoint,
 * perturbations.py:904-925, as used in the reference's gradient notebooks).  The tangent is the
 * exact derivative of the discrete Rodas5 solution with the accepted step sequence held fixed.
 *   cosmos[n_cosmo], mode_cosmo[n_modes]   as in discoeb_fwd (mode_cosmo may be NULL: all 0)
 *   tangents [n_cosmo, n_dir]        device array: d(parameters, tables)/d(theta_d) per cosmology
 *   y0_dot [n_dir, n_modes, nvar]    d(initial state)/d(theta_d) at fixed start times
 *   tau_out [n_cosmo, n_out]         output times of each cosmology
 *   tau_out_dot [n_cosmo, n_dir, n_out]  d(output times)/d(theta_d)
 *   y_out20 [n_modes, n_out, 20]     output fields (may be NULL)
 *   y_out20_dot [n_dir, n_modes, n_out, 20]  their derivatives
 * One block per mode (and group of up to 6 directions): one warp solves the forward once, the
 * others carry the tangents through its published steps; one launch. */
int32_t discoeb_jvp(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                    const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                    const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                    const double* tau_out, const double* tau_out_dot, double* y_out20, double* y_out20_dot,
                    int32_t* status, int32_t* nsteps, void* stream);

/* discoeb_jvp with whole states out instead of the 20 output fields: the RSA-projected state at
 * every output time and its derivative along each direction (the inputs of the CMB source
 * functions, whose gradients jax.jacfwd through the reference's
 * compute_Cell_spectrum_from_cosmo_params, cmb.py:931-1090, pushes through the solve):
 *   y_full [n_modes, n_out, nvar]             states (may be NULL)
 *   y_full_dot [n_dir, n_modes, n_out, nvar]  d(state at the moving output time)/d(theta_d)
 * Other arguments, launch and status codes as discoeb_jvp. */
int32_t discoeb_jvp_full(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                         const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                         const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                         const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                         const double* tau_out, const double* tau_out_dot, double* y_full, double* y_full_dot,
                         int32_t* status, int32_t* nsteps, void* stream);

/* discoeb_jvp (full = 0) or discoeb_jvp_full (full = 1) with a caller workspace for the step
 * records that the forward warp of a block hands to its tangent warps.  The plain entries keep
 * two whole records in shared memory, which for large states (l_max 50: n = 219) leaves room for
 * only three tangent warps per block, so the forward runs twice per mode and an SM holds three
 * tangent warps.  Here one record is kept, its state and stage vectors (13 n doubles per block) in
 * the workspace and the factorisation of W in shared memory, and all six directions share a block
 * (same results bit for bit).
 * discoeb_jvp_records_bytes: the workspace size (0: the records fit with every direction in one
 * block, nothing to gain; < 0: error).  records: >= that many bytes of device memory, 16-byte
 * aligned, or NULL / too small for the shared-memory form.  Other arguments as discoeb_jvp. */
int64_t discoeb_jvp_records_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_dir, int32_t n_modes);
/* The split form's workspace whether or not it adds directions per block (a caller that passes
 * this much gets the split form also where the records would fit in shared memory). */
int64_t discoeb_jvp_split_records_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_dir, int32_t n_modes);
int32_t discoeb_jvp_records(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                            const int32_t* mode_cosmo, const DiscoebTangent* tangents_dev, int32_t n_dir,
                            const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                            const double* y0, const double* y0_dot, const double* switch_tau, int32_t n_out,
                            const double* tau_out, const double* tau_out_dot, double* y_out, double* y_out_dot,
                            int32_t* status, int32_t* nsteps, int32_t full, void* records, int64_t records_bytes,
                            void* stream);

/* ---- Discrete adjoint (reverse mode) ----
 * Replaces reverse-mode differentiation (jax.grad / jax.vjp) through diffeqsolve(...,
 * adjoint=DirectAdjoint()) (src/discoeb/perturbations.py:904-925, :1059-1083): the exact
 * vector-Jacobian product of the discrete Rodas5 solution with its accepted step sequence held
 * fixed (the transpose of what discoeb_jvp computes), in one reverse sweep per mode whatever the
 * number of parameters.  Two launches: discoeb_fwd_record solves forward and records the accepted
 * steps (their end times, and the start state of every checkpoint_every-th step); discoeb_bwd
 * runs the reverse sweep from the cotangent of the output fields, recomputing each segment of
 * checkpoint_every steps from its checkpoint.  Start times and approximation switch times are
 * held fixed, as forward-mode AD through the reference leaves them.
 *
 * Doubles of one mode's record: step_capacity step end times plus
 * ceil(step_capacity / checkpoint_every) checkpoint states of nvar doubles. */
int64_t discoeb_step_record_doubles(int32_t nvar, int32_t step_capacity, int32_t checkpoint_every);

/* discoeb_fwd (same arguments; y_out20 may be NULL, whole states are not written) that also writes
 * records [n_modes, discoeb_step_record_doubles(...)] and n_accepted [n_modes] (device).  A mode
 * that takes more than step_capacity accepted steps stops with status DISCOEB_RECORD_FULL. */
int32_t discoeb_fwd_record(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                           const DiscoebControl* ctrl, int32_t n_modes, const int32_t* mode_cosmo,
                           const double* kmodes, const double* tau_start, const double* y0,
                           const double* switch_tau, int32_t n_out, const double* tau_out, double* y_out20,
                           int32_t* status, int32_t* nsteps, int32_t step_capacity, int32_t checkpoint_every,
                           double* records, int32_t* n_accepted, void* stream);

/* Device workspace of discoeb_bwd: one segment of checkpoint_every states per mode. */
int64_t discoeb_bwd_workspace_bytes(const DiscoebCosmo* cosmo0_host, int32_t n_modes, int32_t checkpoint_every);

/* Reverse sweep of a recorded solve (the same cosmos, modes, start and switch times, output times,
 * records, n_accepted and the forward's status; device arrays):
 *   y_out20_bar [n_modes, n_out, 20]  cotangent of the output fields
 *   y0_bar [n_modes, nvar]            cotangent of the initial states
 *   tau_out_bar [n_modes, n_out]      cotangent of the output times (through y' = f at each one)
 *   par_bar [n_modes, 8]              cotangents of grhom, Omegam, Omegab, OmegaDE, amnu, w0, wa, H0
 *                                     (DiscoebTangent's scalar order)
 *   table_bar [n_cosmo, 8, table_stride]  ADDED to (the caller zeroes it): cotangents of the knot
 *                                     values xe_y, xe_S, cs2a_y, cs2a_S, logrhonu_y, logrhonu_S,
 *                                     logpnu_y, logpnu_S (DiscoebTangent's table order), summed
 *                                     over each cosmology's modes (atomically: equal to rounding
 *                                     between runs); table_stride >= every table's knot count
 *   table_per_mode                    nonzero: table_bar is [n_modes, 8, table_stride], one block
 *                                     of rows per mode (the per-mode gradients of a Jacobian row) 
 *   workspace                         >= discoeb_bwd_workspace_bytes(...) bytes
 *   status [n_modes]                  DISCOEB_OK, or the forward's status (NaN outputs) */
int32_t discoeb_bwd(const DiscoebCosmo* cosmos_dev, const DiscoebCosmo* cosmo0_host, int32_t n_cosmo,
                    const int32_t* mode_cosmo, int32_t n_modes, const double* kmodes, const double* tau_start,
                    const double* switch_tau, int32_t n_out, const double* tau_out, int32_t step_capacity,
                    int32_t checkpoint_every, const double* records, const int32_t* n_accepted,
                    const int32_t* fwd_status, const double* y_out20_bar, double* y0_bar, double* tau_out_bar,
                    double* par_bar, double* table_bar, int32_t table_stride, int32_t table_per_mode, void* workspace,
                    int64_t workspace_bytes, int32_t* status, void* stream);

/* theta_bar [n_cosmo, n_dir] = the cotangents of discoeb_bwd contracted with n_dir parameter
 * tangents (tangents_dev [n_cosmo, n_dir], y0_dot [n_dir, n_modes, nvar], tau_out_dot
 * [n_cosmo, n_dir, n_out], the arrays discoeb_jvp takes): the gradient of a scalar loss with
 * respect to those parameters, summed over each cosmology's modes (device arrays).  per_mode
 * nonzero (table_bar per mode, as discoeb_bwd's table_per_mode): theta_bar [n_modes, n_dir], each
 * mode's own gradient (a row of dP(k)/dtheta when the cotangent is that mode's output). */
int32_t discoeb_bwd_contract(const DiscoebCosmo* cosmos_dev, int32_t n_cosmo, const int32_t* mode_cosmo,
                             int32_t n_modes, int32_t nvar, int32_t n_out, const DiscoebTangent* tangents_dev,
                             int32_t n_dir, const double* y0_dot, const double* tau_out_dot, const double* y0_bar,
                             const double* tau_out_bar, const double* par_bar, const double* table_bar,
                             int32_t table_stride, int32_t per_mode, double* theta_bar, void* stream);

/* RHS f(tau_i, y_i; k_i) of n_points states (compute_time_derivatives):
 *   y, f [n_points, nvar]; tau, kmodes [n_points]; regime < 0: approximation switches
 *   evaluated from (tau, a) as the reference does, else bitmask 1=RSA 2=UFA 4=TCA. */
int32_t discoeb_rhs(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host, int32_t n_points,
                    const double* tau, const double* kmodes, const double* y, int32_t regime, double* f,
                    void* stream);

/* ---- CMB sources and line-of-sight integral (src/discoeb/cmb.py) ---- */

/* Per-output-time background table bgtab[DISCOEB_BG_NFIELDS, n_tau] (row f = field f):
 * a(tau_out), a'/a (get_aprimeoa), rho_nu, rho_Q, w_Q (compute_background_quantities,
 * background.py:348-406), and the visibility functions of compute_visibility_functions
 * (cmb.py:95-163): opacity, its tau derivative, g, g', g'', optical depth. */
#define DISCOEB_BG_A 0
#define DISCOEB_BG_APRIMEOA 1
#define DISCOEB_BG_RHONU 2
#define DISCOEB_BG_RHO_Q 3
#define DISCOEB_BG_W_Q 4
#define DISCOEB_BG_OPAC 5
#define DISCOEB_BG_OPACPRIME 6
#define DISCOEB_BG_GVIS 7
#define DISCOEB_BG_GVISPRIME 8
#define DISCOEB_BG_GVISPPRIME 9
#define DISCOEB_BG_OPTICAL_DEPTH 10
#define DISCOEB_BG_NFIELDS 11

/* Output fields of discoeb_sources, fields[DISCOEB_SRC_NFIELDS, n_modes, n_tau]. */
#define DISCOEB_SRC_S 0             /* S = S1 + S2 + S3 + S4 (compute_source_function) */
#define DISCOEB_SRC_S1 1            /* ISW, compute_source_term_isw */
#define DISCOEB_SRC_S2 2            /* Sachs-Wolfe */
#define DISCOEB_SRC_S3 3            /* Doppler */
#define DISCOEB_SRC_S4 4            /* polarisation */
#define DISCOEB_SRC_POTENTIAL 5     /* eta + alpha' (differentiated for S1) */
#define DISCOEB_SRC_ALPHA 6         /* compute_metric_perturbations: alpha, alpha', alpha'', h', eta', (a'/a)' */
#define DISCOEB_SRC_ALPHAPRIME 7
#define DISCOEB_SRC_ALPHAPPRIME 8
#define DISCOEB_SRC_HPRIME 9
#define DISCOEB_SRC_ETAPRIME 10
#define DISCOEB_SRC_APRIMEOAPRIME 11
#define DISCOEB_SRC_POL 12          /* compute_polarization_terms: Pi, Pi', Pi'' */
#define DISCOEB_SRC_POLPRIME 13
#define DISCOEB_SRC_POLPPRIME 14
#define DISCOEB_SRC_DRHONU 15       /* compute_neutrino_perturbations */
#define DISCOEB_SRC_DPNU 16
#define DISCOEB_SRC_FNU 17
#define DISCOEB_SRC_SHEARNU 18
#define DISCOEB_SRC_RHONUPRIME 19
#define DISCOEB_SRC_SHEARNUPRIME 20
#define DISCOEB_SRC_THETABPRIME 21  /* theta_b' of compute_time_derivatives */
#define DISCOEB_SRC_E 22            /* E-mode polarisation source (3/16) g Pi (no counterpart in the
                                     * reference, which computes temperature only) */
#define DISCOEB_SRC_NFIELDS 23

/* CMB source function at the output times of a full solve: replaces
 * compute_time_derivatives + extract_perturbations + compute_neutrino_perturbations +
 * compute_metric_perturbations + compute_polarization_terms + compute_source_term_* +
 * compute_source_function (perturbations.py:1339-1406, cmb.py:17-633).
 *   y_full [n_modes, n_tau, nvar]  RSA-projected states (discoeb_fwd's y_full), device
 *   tau [n_tau] increasing, kmodes [n_modes], bgtab [DISCOEB_BG_NFIELDS, n_tau], device
 *   fields [DISCOEB_SRC_NFIELDS, n_modes, n_tau] out; scratch [n_modes, n_tau] doubles. */
int32_t discoeb_sources(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host, int32_t n_modes,
                        const double* kmodes, int32_t n_tau, const double* tau, const double* bgtab,
                        const double* y_full, double* fields, double* scratch, void* stream);

/* The forward solve of one cosmology's modes with the source assembly done in its output stage:
 * discoeb_fwd (its arguments for n_cosmo = 1, the output times being the source times tau) and
 * discoeb_sources in one pass, replacing evolve_perturbations(return_full=True) +
 * compute_time_derivatives + the source assembly of cmb.py:17-633 without the full states
 * making the round trip through device memory.  Each mode's warp projects the state at every
 * output time, re-evaluates y' there and assembles the sources; the ISW term follows as in
 * discoeb_sources.  y_full [n_modes, n_tau, nvar] (may be NULL) still receives the projected
 * states; fields, scratch, bgtab as discoeb_sources; status / nsteps per mode as discoeb_fwd
 * (fields of a failed mode's unreached times are NaN).  The results equal discoeb_fwd followed
 * by discoeb_sources.  Structured FP64 method only. */
int32_t discoeb_fwd_sources(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host,
                            const DiscoebControl* ctrl, int32_t n_modes, const double* kmodes, const double* tau_start,
                            const double* y0, const double* switch_tau, int32_t n_tau, const double* tau,
                            const double* bgtab, double* y_full, double* fields, double* scratch, int32_t* status,
                            int32_t* nsteps, void* stream);

/* discoeb_sources for callers that cannot allocate device memory: code running where another
 * framework owns the GPU's memory (XLA preallocates most of it, so an FFI handler that was given
 * no workspace buffer has nothing to pass as scratch and must not cudaMalloc behind the
 * framework's back), or a real-time host loop where allocation is not allowed.  It takes the
 * arguments of discoeb_sources without `scratch` and allocates nothing: its scratch is a
 * file-scope device array of 2^20 doubles (8 MiB) that the library holds on every GPU that loads
 * it, until the process exits.  Limit: n_modes * n_tau <= 1048576, else DISCOEB_EINVAL and no
 * work.  The first call on a device looks up the array's device address (cudaGetSymbolAddress,
 * with that device current) and keeps it until the process exits; make that first call before any
 * stream capture, and do not use this entry after resetting a device it has run on
 * (cudaDeviceReset unloads the array, and the kept address would be stale).  Every call shares
 * the array, so calls that overlap on the GPU (two streams, two host threads) race: serialise
 * them.  Nothing in the array has to start at zero (it is written before it is read).  No
 * counterpart in the reference. */
int32_t discoeb_sources_noalloc(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host, int32_t n_modes,
                                const double* kmodes, int32_t n_tau, const double* tau, const double* bgtab,
                                const double* y_full, double* fields, void* stream);

/* Forward-mode sources: the derivative of S (fields row DISCOEB_SRC_S) along n_dir parameter
 * directions, from the derivatives of the states at the (moving) output times, of the output
 * times, of the background rows and of the tables and scalars (the C_l gradient's sources:
 * jax.jacfwd through compute_source_function, cmb.py:17-633).
 *   tangents_dev [n_dir]                   d(parameters, tables)/d(theta_d), as for discoeb_jvp
 *   tau_dot [n_dir, n_tau], bgtab_dot [n_dir, DISCOEB_BG_NFIELDS, n_tau]
 *   y_full_dot [n_dir, n_modes, n_tau, nvar]  (discoeb_jvp_full's state tangents)
 *   fields: discoeb_sources' output at the base point (its potential row is read)
 *   S_dot [n_dir, n_modes, n_tau] out; scratch: 8 n_dir n_modes n_tau doubles
 *   SE_dot [n_dir, n_modes, n_tau] out, may be NULL: the derivative of the E-mode source
 *   (DISCOEB_SRC_E; no counterpart in the reference).  Device arrays.
 * One warp per (mode, time) evaluates the base point's y' once and every direction after it, so
 * one call with all directions costs less than one call per direction (same results bit for
 * bit). */
int32_t discoeb_sources_jvp(const DiscoebCosmo* cosmo_dev, const DiscoebCosmo* cosmo_host,
                            const DiscoebTangent* tangents_dev, int32_t n_dir, int32_t n_modes, const double* kmodes,
                            int32_t n_tau, const double* tau, const double* tau_dot, const double* bgtab,
                            const double* bgtab_dot, const double* y_full, const double* y_full_dot,
                            const double* fields, double* S_dot, double* scratch, double* SE_dot, void* stream);

/* Workspace bytes of discoeb_los for these sizes (< 0: invalid sizes or a cuFFT error). */
int64_t discoeb_los_workspace_bytes(int32_t n_modes, int32_t n_tau, int32_t ellmax, int32_t n_fftlog,
                                    int32_t n_k_dense);

/* Line-of-sight multipoles Theta_l(k) = int S(k, tau) j_l(k (tau0 - tau)) dtau by the
 * reference's FFTLog method: replaces compute_theta_ell (cmb.py:680-835).
 *   S [n_modes, n_tau] device; kmodes [n_modes] increasing; tau [n_tau] increasing.
 *   n_k_dense > 0: S is first spline-resampled onto n_k_dense log-spaced modes.
 *   theta [K', ellmax + 1] and kmodes_out [K'] out, K' = n_k_dense or n_modes.
 *   workspace: >= discoeb_los_workspace_bytes(...) bytes of device memory, 256-byte aligned
 *   (the FFT buffer, the coefficient table and the cuFFT / cuBLAS work areas live there). */
int32_t discoeb_los(int32_t n_modes, const double* kmodes, int32_t n_tau, const double* tau, const double* S,
                    double tau0, int32_t ellmax, int32_t n_fftlog, int32_t n_k_dense, void* workspace,
                    int64_t workspace_bytes, double* theta, double* kmodes_out, void* stream);

/* How discoeb_los, discoeb_los_e and discoeb_los_cell_jvp contract the frequency sum
 * theta[k, l] = sum_q c_q(k) M_l(p_q) (cmb.py:809-834, two real einsums there):
 * DISCOEB_LOS_INT8 (default, slices 7): discoeb_dgemm_i8 below, about 1e-13 of each row's largest
 * |theta_l(k)| from the FP64 sum; DISCOEB_LOS_FP64: a cuBLAS DGEMM.  A library-wide setting, read
 * once by each call (and by the *_workspace_bytes queries, whose result depends on it). */
#define DISCOEB_LOS_FP64 0
#define DISCOEB_LOS_INT8 1
int32_t discoeb_set_los_contraction(int32_t kind, int32_t slices);
int32_t discoeb_get_los_contraction(int32_t* kind, int32_t* slices);

/* FP64 product C = A B^T on the int8 tensor cores (tcgen05.mma kind::i8): the line of sight's
 * frequency sum (cmb.py:809-834, two real einsums there) without an FP64 GEMM.  Each row of A and
 * of B is split over one power-of-two scale into `slices` (1..8) signed 8-bit digit planes
 * (d_0 in [-127, 127], then 7 bits each); the digit products of equal total weight accumulate
 * exactly in int32 and the slices levels are summed in FP64.  Error per element about
 * 2^(1 - 7 slices) (max_k |A_ik| sum_k |B_jk| + sum_k |A_ik| max_k |B_jk|) on top of FP64
 * rounding; a row holding a non-finite value gives NaN products.
 *   C [m, ldc >= n] row-major; op(A)[i, q] = A[i * lda + q] (trans_a = 0, A [m, lda >= k]) or
 *   A[q * lda + i] (trans_a = 1, A [k, lda >= m]); B likewise with n: C = op(A) op(B)^T.
 *   Device arrays.  split: K ranges per output tile (<= 0: chosen from the SM count).
 *   workspace: >= discoeb_dgemm_i8_workspace_bytes(m, n, k, slices, split) bytes, 256-byte
 *   aligned (digit planes, scales, level sums).  A kernel whose bounded waits run out (never in a
 *   correct launch) writes NaN into C. */
int64_t discoeb_dgemm_i8_workspace_bytes(int32_t m, int32_t n, int32_t k, int32_t slices, int32_t split);
int32_t discoeb_dgemm_i8(int32_t m, int32_t n, int32_t k, const double* A, int64_t lda, int32_t trans_a,
                         const double* B, int64_t ldb, int32_t trans_b, double* C, int64_t ldc, int32_t slices,
                         int32_t split, void* workspace, int64_t workspace_bytes, void* stream);

/* C_l = trapezoid over ln k of (k/k_p)^(n_s-1) Theta_l(k)^2: replaces compute_Cell
 * (cmb.py:838-873).  theta [n_modes, n_ell], cell [n_ell], device. */
int32_t discoeb_cell(int32_t n_modes, const double* kmodes, int32_t n_ell, const double* theta, double n_s,
                     double k_p, double* cell, void* stream);

/* E-mode polarisation (no counterpart in the reference, which computes C_l^TT only): the
 * multipoles Theta_E,l(k) = sqrt((l+2)!/(l-2)!) int S_E(k, tau) j_l(x) / x^2 dtau, x = k(tau0 - tau)
 * (Zaldarriaga & Seljak 1997), of the source row DISCOEB_SRC_E, by the FFTLog method of
 * discoeb_los: for l < 8 applied to S_E / chi^2 (chi held >= 1 Mpc), for l >= 8 applied to S_E at
 * l - 2, l, l + 2 and combined by the spherical Bessel recurrence (j_l / x^2 as a sum of j_(l-2),
 * j_l, j_(l+2)), which keeps the FFTLog's error from being multiplied by l^2.  Arguments as
 * discoeb_los; workspace: discoeb_los_e_workspace_bytes(...) bytes, 256-byte aligned.  theta_l = 0
 * for l < 2. */
int64_t discoeb_los_e_workspace_bytes(int32_t n_modes, int32_t n_tau, int32_t ellmax, int32_t n_fftlog,
                                      int32_t n_k_dense);
int32_t discoeb_los_e(int32_t n_modes, const double* kmodes, int32_t n_tau, const double* tau, const double* S_E,
                      double tau0, int32_t ellmax, int32_t n_fftlog, int32_t n_k_dense, void* workspace,
                      int64_t workspace_bytes, double* theta, double* kmodes_out, void* stream);

/* Cross spectrum C_l^AB = trapezoid over ln k of (k/k_p)^(n_s-1) Theta^A_l(k) Theta^B_l(k) (C_l^TE
 * from the temperature and E-mode multipoles on the same k grid); as discoeb_cell otherwise. */
int32_t discoeb_cell_cross(int32_t n_modes, const double* kmodes, int32_t n_ell, const double* theta_a,
                           const double* theta_b, double n_s, double k_p, double* cell, void* stream);

/* C_l of the line of sight (discoeb_los then discoeb_cell, same arguments) and its derivative
 * along n_dir directions of the inputs, in forward mode through the resampling, the FFT
 * coefficients and the table M_l(p) (the grid moves with tau0 - tau; the interval indices of the
 * resampling are the base point's): the C_l part of jax.jacfwd through compute_theta_ell and
 * compute_Cell (cmb.py:680-873).
 *   tau_dot [n_dir, n_tau], S_dot [n_dir, n_modes, n_tau]   device
 *   tau0_dot [n_dir]                                         host
 *   cell [ellmax + 1], cell_dot [n_dir, ellmax + 1]          device
 *   cell_dns [ellmax + 1]  d C_l / d n_s (the primordial weight's derivative), device, may be NULL
 *   workspace: >= discoeb_los_cell_jvp_workspace_bytes(...) bytes, 256-byte aligned
 * One GEMM for the base point, one shared, one per direction (each the size of discoeb_los's). */
int64_t discoeb_los_cell_jvp_workspace_bytes(int32_t n_modes, int32_t n_tau, int32_t ellmax, int32_t n_fftlog,
                                             int32_t n_k_dense);
int32_t discoeb_los_cell_jvp(int32_t n_modes, const double* kmodes, int32_t n_tau, const double* tau, const double* S,
                             double tau0, int32_t n_dir, const double* tau_dot, const double* S_dot,
                             const double* tau0_dot, int32_t ellmax, int32_t n_fftlog, int32_t n_k_dense, double n_s,
                             double k_p, void* workspace, int64_t workspace_bytes, double* cell, double* cell_dot,
                             double* cell_dns, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Observables of the linear power spectrum (device arrays, stream-ordered).
 *
 * squared = 0: amp[i] = sqrt(2 pi^2 A_s (k_i/k_p)^(n_s-1) k_i^-3) y[i * y_stride + idx], the field
 * amplitudes that power_Kaiser and power_multipoles build from the output fields
 * (perturbations.py:1515-1516, :1555-1556); squared = 1: the power spectrum of get_power
 * (perturbations.py:1445-1468). */
int32_t discoeb_power_amplitudes(int32_t n_k, const double* kmodes, const double* y, int32_t y_stride, int32_t idx,
                                 double A_s, double n_s, double k_p, int32_t squared, double* amp, void* stream);

/* Savitzky-Golay smoothing of log P as get_power_smoothed (perturbations.py:1471-1493, with
 * savgol_filter of util.py:291-327): out = exp(convolve(log P, coeffs, 'same')), except the first
 * window_length/2 and the last (window_length+1)/2 entries, which keep P.  coeffs
 * [window_length] (odd) are the filter coefficients (a small least-squares solve the caller does). */
int32_t discoeb_savgol_log_power(int32_t n_k, const double* P, int32_t window_length, const double* coeffs,
                                 double* out, void* stream);

/* Kaiser redshift-space spectrum P(k_i, mu_j) = (bias delta_i - mu_j^2 theta_i)^2 into pkmu
 * [n_k, n_mu] (power_Kaiser, perturbations.py:1495-1524). */
int32_t discoeb_power_kaiser(int32_t n_k, const double* delta, const double* theta, double bias, int32_t n_mu,
                             const double* mu, double* pkmu, void* stream);

/* Its multipoles l = 0, 2, 4 (power_multipoles, perturbations.py:1528-1564). */
int32_t discoeb_power_multipoles(int32_t n_k, const double* delta, const double* theta, double b, double* P0,
                                 double* P2, double* P4, void* stream);

/* Correlation function multipole xi_l(r) from P(k) on log-spaced k by FFTLog (get_xi_from_P,
 * perturbations.py:1409-1442): xi, r [n_k] in increasing r = 2 pi / k.  n_k even (the reference's
 * inverse real FFT returns n_k - 1 points for odd n_k and fails).  workspace: at least
 * discoeb_xi_workspace_bytes(n_k) bytes of 256-byte-aligned device memory. */
int64_t discoeb_xi_workspace_bytes(int32_t n_k);
int32_t discoeb_xi_from_power(int32_t n_k, const double* kmodes, const double* Pk, int32_t ell, void* workspace,
                              int64_t workspace_bytes, double* xi, double* r, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Background and thermal history (host code): replaces evolve_background with RECFAST
 * (background.py:141-345, thermodynamics_recfast.py:124-492) and, with tangents, jax.jacfwd
 * through it.  The cosmological parameters of the reference's param dict; the first six carry
 * derivatives. */
typedef struct {
    double H0, Omegab, Omegam, mnu, w_DE_0, w_DE_a;
    double Tcmb, YHe, Neff, Nmnu, cs2_DE, Omegak;
} DiscoebCosmoParams;

/* Output layout: DISCOEB_BGS_COUNT scalars, then DISCOEB_BGN_COUNT arrays of DISCOEB_NU_KNOTS
 * doubles (massive-neutrino tables on the log-a grid), then DISCOEB_BGT_COUNT arrays of
 * num_thermo doubles (the Recfast a-grid tables); total discoeb_background_size(num_thermo). */
#define DISCOEB_NU_KNOTS 512
enum {
    DISCOEB_BGS_AMIN, DISCOEB_BGS_AMAX, DISCOEB_BGS_GRHOM, DISCOEB_BGS_GRHOG, DISCOEB_BGS_GRHOR,
    DISCOEB_BGS_ADOTRAD, DISCOEB_BGS_AMNU, DISCOEB_BGS_OMEGAMNU, DISCOEB_BGS_OMEGADE, DISCOEB_BGS_TAUMIN,
    DISCOEB_BGS_TAUMAX, DISCOEB_BGS_FHE, DISCOEB_BGS_TAU0, DISCOEB_BGS_TAU_MAXVIS, DISCOEB_BGS_H0,
    DISCOEB_BGS_OMEGAB, DISCOEB_BGS_OMEGAM, DISCOEB_BGS_MNU, DISCOEB_BGS_W0, DISCOEB_BGS_WA,
    DISCOEB_BGS_COUNT
};
enum {
    DISCOEB_BGN_A, DISCOEB_BGN_LOGA, DISCOEB_BGN_LOGRHONU_Y, DISCOEB_BGN_LOGRHONU_S, DISCOEB_BGN_LOGPNU_Y,
    DISCOEB_BGN_LOGPNU_S, DISCOEB_BGN_LOGPPNU_Y, DISCOEB_BGN_LOGPPNU_S, DISCOEB_BGN_COUNT
};
/* *_S: second derivatives of the natural spline whose knots and values are the named arrays
 * (tau_of_a: x = AEXP, y = TAU; a_of_tau: TAU, AEXP; xe_of_tau: TAU, XE; cs2a_of_tau: TAU, CS2A;
 * tempba_of_tau: TAU, TEMPBA; xe_of_loga: LOGA, XE; cs2a_of_loga: LOGA, CS2A; opac: TAU, OPAC).
 * REC_CASE: Recfast branch of each interval (1 early, 2 He Saha, 3 H Saha, 4 full ODE);
 * REC_STEPS: accepted GRK4A steps of each interval (zero in the tangents). */
enum {
    DISCOEB_BGT_AEXP, DISCOEB_BGT_LOGA, DISCOEB_BGT_TAU, DISCOEB_BGT_XE, DISCOEB_BGT_XEHI, DISCOEB_BGT_XEHEI,
    DISCOEB_BGT_XEHEII, DISCOEB_BGT_CS2, DISCOEB_BGT_TM, DISCOEB_BGT_MU, DISCOEB_BGT_XEPRIME_RECF,
    DISCOEB_BGT_CS2A, DISCOEB_BGT_TEMPBA, DISCOEB_BGT_TAU_OF_A_S, DISCOEB_BGT_A_OF_TAU_S,
    DISCOEB_BGT_XE_OF_TAU_S, DISCOEB_BGT_CS2A_OF_TAU_S, DISCOEB_BGT_TEMPBA_OF_TAU_S, DISCOEB_BGT_XE_OF_LOGA_S,
    DISCOEB_BGT_CS2A_OF_LOGA_S, DISCOEB_BGT_OPAC, DISCOEB_BGT_OPAC_S, DISCOEB_BGT_OPTICAL_DEPTH,
    DISCOEB_BGT_GVIS, DISCOEB_BGT_GVISPRIME, DISCOEB_BGT_GVISPPRIME, DISCOEB_BGT_XEPRIME,
    DISCOEB_BGT_REC_CASE, DISCOEB_BGT_REC_STEPS, DISCOEB_BGT_COUNT
};

/* Number of doubles of one background output (values or one tangent). */
int64_t discoeb_background_size(int32_t num_thermo);

/* Background, Recfast history and visibility tables of one cosmology, and optionally their
 * derivatives along n_dir parameter directions (the exact derivative of the discrete result with
 * the Recfast branches and GRK4A step sequence held fixed, as forward-mode AD through the
 * reference's loops gives).
 *   par                     parameters
 *   par_dot [n_dir]         d(par)/d(theta_d) (only the first six fields are read; may be NULL
 *                           when n_dir = 0)
 *   num_thermo              Recfast a-grid size (>= 32; the reference's default is 256)
 *   out [size]              values (host memory)
 *   out_dot [n_dir, size]   tangents (host memory; NULL when n_dir = 0)
 *   n_threads               host threads for the directions (<= 0: one per direction)
 * Host code: touches no device and allocates only host scratch.  Returns DISCOEB_SUCCESS or
 * DISCOEB_EINVAL. */
int32_t discoeb_background(const DiscoebCosmoParams* par, const DiscoebCosmoParams* par_dot, int32_t n_dir,
                           int32_t num_thermo, double* out, double* out_dot, int32_t n_threads);

/* The same for n_cosmo cosmologies on the GPU, batched over cosmologies (one device thread per
 * cosmology and direction, each running the whole sequential background; stream-ordered):
 *   par_dev [n_cosmo], par_dot_dev [n_cosmo, n_dir]      device arrays (par_dot_dev NULL if n_dir = 0)
 *   out_dev [n_cosmo, size], out_dot_dev [n_cosmo, n_dir, size]   device, size = discoeb_background_size
 *   workspace: discoeb_background_batch_workspace_bytes(...) bytes of 256-byte-aligned device memory
 * Same layout as discoeb_background; the values agree with it up to the last bits of the device's
 * exp/log/pow (amplified downstream of Recfast's Saha x_H formula, as between any two libms). */
int64_t discoeb_background_batch_workspace_bytes(int32_t n_cosmo, int32_t n_dir, int32_t num_thermo);
int32_t discoeb_background_batch(const DiscoebCosmoParams* par_dev, const DiscoebCosmoParams* par_dot_dev,
                                 int32_t n_cosmo, int32_t n_dir, int32_t num_thermo, void* workspace,
                                 int64_t workspace_bytes, double* out_dev, double* out_dot_dev, void* stream);

/* Knot second derivatives S[n] of the natural cubic spline through (x[i], y[i]) (host memory, host
 * code): the Thomas recurrence of spline_interpolation.__init__ (spline_interpolation.py:19-75),
 * operation for operation, for the host layer's tables.  DISCOEB_EINVAL if n < 2. */
int32_t discoeb_natural_spline_second(int32_t n, const double* x, const double* y, double* S);

/* Measurement utility, no counterpart in the reference: the FP64 fused-multiply-add throughput of
 * the current GPU, the roofline denominator of the solver kernels (their arithmetic is FP64 FMA
 * work).  discoeb_fma_rate_threads() returns the thread count of one launch (4 blocks of 256 per
 * SM; negative on a CUDA error).  discoeb_fma_rate enqueues one launch on `stream` in which every
 * thread runs 8 independent FMA chains for `iters` iterations, writes one double per thread to
 * `out` (device, n_out >= discoeb_fma_rate_threads()) and stores the launch's flop count
 * (2 per FMA) in *flops (host); the caller times the launch. */
int64_t discoeb_fma_rate_threads(void);
int32_t discoeb_fma_rate(int64_t iters, double* out, int64_t n_out, double* flops, void* stream);

#ifdef __cplusplus
}
#endif
#endif
