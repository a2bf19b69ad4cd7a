/*
 * cdft_b200.h -- C ABI of the B200 (sm_100a) implementation of cDFT.jl's
 * converge! hot path for PC-SAFT weighted-density DFT.
 *
 * Every entry point replaces one call on the reference's Julia path
 * (ClapeyronThermo/cDFT.jl); the replaced function is cited beside each
 * declaration.  Julia reaches this library through ccall (see the shim
 * cdft.jl_b200/julia/CDFTB200.jl); Python through ctypes.
 *
 * Conventions
 *  - Host arrays are column-major with the grid fastest, exactly like the
 *    reference's Julia arrays: a profile rho(ngrid..., nc) is stored as
 *    rho[((i*Nz + z)*Ny + y)*Nx + x] for component i.
 *  - Densities in mol/m^3, lengths in m, energies eps/k_B in K.
 *  - Every call returns 0 on success or a negative CDFT_E* code; the message
 *    of the last error of the calling thread is available from
 *    cdft_last_error().  No exception or exit() crosses this boundary.
 *  - A plan is bound to the CUDA device current at cdft_plan_create and to
 *    one stream; it is not thread-safe.  Distinct plans may be used
 *    concurrently from distinct host threads.
 */
#ifndef CDFT_B200_H
#define CDFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CDFT_MAX_NC 4        /* components per system */
#define CDFT_MAX_ASSOC 8     /* association pairs per system: one pair takes the analytic path
                                (assoc.jl:702-769), two or more the general solve (:771-828) */
#define CDFT_MAX_SITES 8     /* distinct association sites over all components */
#define CDFT_MAX_M 16        /* Anderson history depth */

/* error codes */
#define CDFT_OK 0
#define CDFT_E_INVALID -1     /* invalid argument */
#define CDFT_E_CUDA -2        /* CUDA runtime error */
#define CDFT_E_UNSUPPORTED -3 /* valid request outside the implemented scope */
#define CDFT_E_BUDGET -4      /* host wall-clock budget exhausted before the solver ended */
#define CDFT_E_NOMEM -5

/* coordinate systems (Structure{Dim,Coord}, src/base/structure.jl:116-130) */
#define CDFT_COORD_CART 0
#define CDFT_COORD_SPH 1
#define CDFT_COORD_CYL 2

/* arithmetic of the convolutions and of Phi (DFTOptions precision, src/base/devices.jl:29-40) */
#define CDFT_PREC_FP64 0
#define CDFT_PREC_MIXED 1    /* FP32 convolutions and Phi; FP64 Anderson, norms, integrals.  A 1D
                                Cartesian system on the persistent engine converges in FP64 (the
                                FP32 phase gains nothing there) */

/* One Wertheim association pair, as packed by pack_assoc_params
 * (src/models/DFT/assoc.jl:18-56): site isite of component icomp bonds with
 * site jsite of component jcomp.  (icomp, isite) names one site: pairs that
 * share it refer to the same fraction X of non-bonded sites. */
typedef struct {
    int icomp, jcomp;          /* 0-based */
    int isite, jsite;          /* 0-based site index within the component */
    int n_ia, n_jb;            /* site multiplicities */
    double eps_ab;             /* epsilon_assoc / k_B, K */
    double kappa_ab;           /* bonding volume (dimensionless) */
} cdft_assoc_pair;

/* Everything the reference's DFTSystem (src/base/base.jl:50-73) carries into
 * the hot path, as plain numbers: the structure, the PC-SAFT parameters, the
 * species data of get_species (PCSAFT.jl:65-72) and the cached external
 * potential of preallocate_external_potential (devices.jl:71-102). */
typedef struct {
    int nd;                          /* 1 or 3 */
    int ngrid[3];                    /* points per dimension (unused entries ignored) */
    double bounds[3][2];             /* [lb, ub] per dimension, m */
    int coord;                       /* CDFT_COORD_* */
    int nc;                          /* components (one bead each) */
    double m[CDFT_MAX_NC];           /* segment numbers */
    double hsd[CDFT_MAX_NC];         /* hard-sphere diameters d_i(T), m (species.size) */
    double sigma[CDFT_MAX_NC * CDFT_MAX_NC]; /* sigma_ij, m, row-major nc x nc */
    double eps[CDFT_MAX_NC * CDFT_MAX_NC];   /* eps_ij / k_B, K, row-major nc x nc */
    double L;                        /* length scale, m (length_scale(model) = max sigma) */
    double T;                        /* temperature, K */
    int n_assoc;                     /* 0 .. CDFT_MAX_ASSOC */
    cdft_assoc_pair assoc[CDFT_MAX_ASSOC];
    double mu_res_plus_ln_rhob[CDFT_MAX_NC]; /* species.chempot_res + log(bulk_density), converge.jl:121 */
    const double* vext;              /* external potential / k_B T, (ngrid..., nc); NULL = none */
    int precision;                   /* CDFT_PREC_* */
} cdft_system_desc;

/* Called by cdft_converge / cdft_batch_converge every snapshot_every fixed-point
 * evaluations with the profile of system `system` (index in the batch) after
 * `evaluations` evaluations (the iterate the next evaluation receives), nc x N doubles in
 * host memory valid during the call.  The counterpart of DFTProblem's save_callback /
 * log_interval (src/methods/converge.jl:31-60,256-267).  It runs on the calling thread
 * between kernel launches and must not call the library with the plans being converged. */
typedef void (*cdft_snapshot_fn)(void* user, int system, int evaluations, const double* rho);

/* The AASol fields used by aasol (src/utils/anderson.jl:193-207).  The
 * converge! keyword form maps onto it as __AASol does (converge.jl:3-9):
 * rtol = atol = tol, picard_maxit = maxit, picard_beta = beta,
 * picard_rtol = picard_atol = anderson_start. */
typedef struct {
    int m;                 /* Anderson depth, 0 <= m <= CDFT_MAX_M */
    int maxit;
    double rtol, atol, beta;
    int picard_maxit;
    double picard_beta, picard_rtol, picard_atol;
    double time_budget_s;  /* host wall-clock cap for the whole call, <= 0: none */
    int iters_per_launch;  /* fixed-point evaluations per CUDA-graph launch (grid engine), <= 0: default */
    int engine;            /* CDFT_ENGINE_* */
    double mixed_switch_rtol; /* mixed plans: FP32 phase until ||r|| <= max(rtol, this) ||r0|| + atol,
                                 then FP64 (Anderson from the first step, no Picard warm-up) until
                                 ||r|| <= rtol ||r0|| + atol, the stopping test of an FP64 run (r0 of
                                 the initial profile); a system whose FP32 phase diverges is converged
                                 again in FP64 from its initial profile; <= 0: 1e-5 */
    int snapshot_every;    /* > 0: call snapshot every this many evaluations (runs the grid engine,
                              one CUDA-graph launch per interval); 0: never */
    cdft_snapshot_fn snapshot;
    void* snapshot_user;
} cdft_solver_opts;

/* execution engines of cdft_converge / cdft_batch_converge */
#define CDFT_ENGINE_AUTO 0        /* persistent when every system fits one CTA's shared memory */
#define CDFT_ENGINE_GRID 1        /* per-stage kernels over all systems, CUDA-graph iterations */
#define CDFT_ENGINE_PERSISTENT 2  /* one CTA per system runs the whole aasol loop, one launch */

/* The (idid, errcode, history) part of aasol's output (anderson.jl:81-103,727-757). */
typedef struct {
    int idid;              /* 1 converged, 0 not */
    int errcode;           /* -1 initial iterate within tol, -2 divergence (residual above 1e4 ||r0||
                              or not finite), 0 converged, 10 maxit */
    int iterations;        /* Anderson counter k of aasol */
    int evaluations;       /* fixed-point map evaluations */
    double resnorm;        /* final ||beta (G(x) - x)||_2 */
    double tol;            /* rtol * ||r0|| + atol */
    double* history;       /* optional caller buffer for resnorm per evaluation, or NULL */
    int history_cap;
    int history_len;       /* entries written */
} cdft_result;

typedef struct cdft_plan cdft_plan;

/* Build the device-side system: weighted-density kernels (get_fields,
 * PCSAFT.jl:47-62; SWeightedDensity/VWeightedDensity, weighted_densities.jl:28-80,
 * 193-246), reduced parameters (preallocate_params, PCSAFT.jl:213-285) and
 * work buffers (preallocate / preallocate_model, devices.jl:51-68,
 * models.jl:209-251). */
int cdft_plan_create(const cdft_system_desc* desc, cdft_plan** plan);
int cdft_plan_destroy(cdft_plan* plan);

/* dF/drho for every component: residual functional derivative plus external
 * field, in k_B T.  Replaces δFδρ_res(system, ρ), src/models/models.jl:194-200
 * (δFδρ_res! :131-186 followed by evaluate_external_field!). */
int cdft_functional_derivative(cdft_plan* plan, const double* rho, double* dFdrho);
int cdft_functional_derivative_dev(cdft_plan* plan, const double* d_rho, double* d_dFdrho);

/* Bulk molar densities (mol/m^3) of n state points at the temperature of desc, with its
 * m, hsd, sigma, eps and association (2B self-association only): pressure p[s] (Pa),
 * mole fractions x[s * nc + i] (normalised here).  phase 0: the stable root (lower Gibbs
 * energy of the densest and the most dilute root, the default of volume(model, p, T, x)
 * behind get_species, PCSAFT.jl:65-72, and adsorption, adsorption.jl:48-65); 1 the
 * densest root; 2 the most dilute root.  status[s] = 0, or 1 where no root exists (rho
 * NaN).  Fields of desc other than nc, m, hsd, sigma, eps, T and the pairs are ignored. */
int cdft_bulk_density(const cdft_system_desc* desc, int n, const double* p, const double* x, int phase,
                      double* rho, int* status);

/* Vapour-liquid coexistence of a pure component (nc = 1) at n temperatures T[s] (K), one
 * launch: p_sat[s] (Pa), rho_liquid[s] and rho_vapour[s] (mol/m^3).  Replaces the
 * saturation state that surface_tension(model, T, x) takes from bubble_pressure(model, T, x)
 * for a pure component (src/methods/surface_tension.jl:13-20; Clapeyron's
 * saturation_pressure).  Uses desc's m, sigma (m), eps (K) and 2B self-association; the
 * diameter at each T is PC-SAFT's sigma (1 - 0.12 exp(-3 eps / T)), so desc's hsd and T
 * are ignored.  Newton on (ln rho_l, ln rho_v) from the densest root at 1e3 Pa and the
 * ideal-gas vapour there; p_sat is the vapour root's pressure (the liquid's compressibility
 * factor is ~1e-6 at low T, so its pressure amplifies the last bits of rho_l).  status[s] = 0 ok, 1 no liquid root at 1e3 Pa, 2 not converged
 * in 100 steps, 3 the trivial solution (T at or above the critical temperature); outputs
 * NaN where status != 0. */
int cdft_saturation_pure(const cdft_system_desc* desc, int n, const double* T, double* p_sat, double* rho_liquid,
                         double* rho_vapour, int* status);

/* Right-hand side of dynamic DFT in eta = ln rho: deta = lap(eta) + lap(mu) +
 * sum_d (d_d eta)^2 + d_d mu d_d eta with rho = exp(clamp(eta, -50, 30)) and
 * mu = dF/drho_res + V_ext, derivatives spectral in reduced lengths (x / L) on the
 * periodic grid.  Replaces the function ddft_rhs_log! that
 * SciMLBase.ODEProblem(system, ρ, tspan) integrates, ext/SciMLBasecDFTExt.jl:10-61
 * (Cartesian 1D and 3D; the derivative maps act as exact periodic circulants along
 * each axis, the same linear operators as the reference's FFT products).  eta and
 * deta have the layout of rho. */
int cdft_ddft_rhs(cdft_plan* plan, const double* eta, double* deta);
int cdft_ddft_rhs_dev(cdft_plan* plan, const double* d_eta, double* d_deta);

/* Residual Helmholtz energy per unit area (1D) or total (3D) in units of k_B T
 * (per m^2 in 1D), evaluated in FP64 whatever the plan's precision.  Replaces F_res(system, ρ), src/models/models.jl:86-91
 * (Simpson rule of src/utils/integrals.jl:17-41 on the device f_res values,
 * compensated FP64 summation). */
int cdft_free_energy_res(cdft_plan* plan, const double* rho, double* F);

/* The integrals of several systems at given profiles, on the device in one batch:
 * out[(3 + nc) s + q] for system s, with q = 0 F_res (as cdft_free_energy_res), q = 1
 * F_ideal (BasicIdeal.jl:10-38, k_B T), q = 2 + i int rho_i, q = 2 + nc int 1 -- the
 * Simpson rule of src/utils/integrals.jl:17-41 (or the radial quadrature), compensated
 * FP64 summation.  From them: free_energy = F_ideal + F_res (utils/base.jl:8-10),
 * surface_tension's numerator F k_B T - sum mu_i int rho_i + p int 1
 * (surface_tension.jl:31-53) and adsorption int rho_i / V (adsorption.jl:26-32).
 * rho[s]: the profile of system s in host (rho_on_device = 0) or device memory; rho = NULL
 * takes the profiles the plans hold (e.g. right after a converge).  The systems must
 * share nc, dimension, coordinates and precision (as a batch). */
int cdft_batch_integrals(cdft_plan* const* plans, int nplans, double* const* rho, int rho_on_device, double* out);

/* Pointwise fused Phi and dPhi/dn_alpha at npts points: n and dphi are
 * (npts, NF, nc) column-major (point fastest), fval is (npts).  Replaces
 * the Enzyme kernels δf_fwd_kernel!/δf_rev_kernel! (models.jl:355-411) that
 * differentiate f_res (PCSAFT.jl:110-117). */
int cdft_phi_pointwise(cdft_plan* plan, const double* n, int npts, double* fval, double* dphi);

/* Phi at every grid point of the profile rho (FP64, reduced units: F_res = the quadrature
 * of Phi over the grid divided by L^3, models.jl:86-91), fval of length prod(ngrid). */
int cdft_phi_field(cdft_plan* plan, const double* rho, double* fval);

/* Parameter gradient of F_res at a fixed profile (1D): dF[3k + 0..2] =
 * dF_res/d(sigma_k [A], eps_k/k_B [K], m_k) in the units of cdft_free_energy_res,
 * with the PC-SAFT diameter d = sigma (1 - 0.12 exp(-3 eps/T)) and
 * sigma_ij = (sigma_i + sigma_j)/2 (CDFT_E_UNSUPPORTED otherwise).  Explicit
 * parameter dependence of Phi (f_res, PCSAFT.jl:110-117) from the same reverse sweep
 * as dPhi/dn; dependence through the kernels (weighted_densities.jl:48-69, widths
 * PCSAFT.jl:55-61) as sum_alpha <dPhi/dn_alpha, rho * d omega_alpha / d theta>.  The
 * reference has no counterpart (it differentiates f_res in n only, models.jl:355-411). */
int cdft_free_energy_res_grad(cdft_plan* plan, const double* rho, double* dF);

/* d Omega_ex / d theta at a converged profile (1D), theta = (sigma_k [A], eps_k/k_B [K],
 * m_k) for k < nc, Omega_ex = F k_B T - sum_i mu_i int rho_i + p int 1 (J/m^2): the
 * numerator of surface_tension(system, ρ), src/methods/surface_tension.jl:31-53
 * (interfacial tension = Omega_ex, or Omega_ex / 2 for the periodic two-interface
 * box, :28).  At a converged profile delta Omega / delta rho = 0, so
 *   dOmega_ex/dtheta = k_B T dF_res/dtheta|_rho - sum_i dmu_i/dtheta int rho_i + dp/dtheta int 1.
 * dmu_dtheta (nc x 3nc, row i = d mu_i / d theta in J/mol) and dp_dtheta (3nc, Pa) are
 * the caller's derivatives of the bulk state the structure was built on (e.g. along
 * phase coexistence); NULL means held fixed.  Plans with an external field are refused
 * (CDFT_E_UNSUPPORTED): V_ext depends on the parameters; cdft_grad_params_ext takes its
 * derivative. */
int cdft_grad_params(cdft_plan* plan, const double* rho, const double* dmu_dtheta, const double* dp_dtheta,
                     double* dOmega);

/* cdft_grad_params for plans with an external field (1D Cartesian): the derivative of the
 * grand potential Omega = F k_B T + k_B T sum_i int rho_i V_i - sum_i mu_i int rho_i + p int 1
 * (the functional whose stationary point converge! finds; surface_tension.jl:31-53 reports
 * it without the wall term), which at a converged profile gains
 * k_B T sum_i int rho_i dV_i/dtheta.  dvext_dtheta[(t*nc + i)*N + k] = d(V_i/k_B T)/d theta_t at
 * grid point k (e.g. the Steele wall's, steele.jl:49-81, through sigma_sf = (sigma_s +
 * sigma_i)/2 and eps_sf = sqrt(eps_s eps_i)).  No counterpart in the reference. */
int cdft_grad_params_ext(cdft_plan* plan, const double* rho, const double* dmu_dtheta, const double* dp_dtheta,
                         const double* dvext_dtheta, double* dOmega);

/* Converge rho in place.  Replaces converge!(prob::DFTProblem, method::AASol, ρ),
 * src/methods/converge.jl:220-254, running aasol (src/utils/anderson.jl:301-443)
 * on the device; rho_inout holds the initial profile on entry and
 * exp(result.solution) on exit.  `result` may be NULL. */
int cdft_converge(cdft_plan* plan, double* rho_inout, const cdft_solver_opts* opts, cdft_result* result);
int cdft_converge_dev(cdft_plan* plan, double* d_rho_inout, const cdft_solver_opts* opts, cdft_result* result);

/* Converge nplans independent systems (state points, pore widths; uneven grid
 * sizes allowed) together, every kernel launch covering all of them.  The
 * reference converges one system per converge! call; this replaces a loop of
 * converge! calls over state points (e.g. an isotherm of adsorption(model,
 * surface, p, T), src/methods/adsorption.jl:48-65). */
int cdft_batch_converge(cdft_plan* const* plans, int nplans, double* const* rho_inout,
                        const cdft_solver_opts* opts, cdft_result* results);
int cdft_batch_converge_dev(cdft_plan* const* plans, int nplans, double* const* d_rho_inout,
                            const cdft_solver_opts* opts, cdft_result* results);

/* Bind a plan to a caller-owned CUDA stream (a cudaStream_t, e.g. the stream of
 * a CUDA.jl task or of torch); NULL restores the plan's own stream.  The
 * reference has no counterpart: KernelAbstractions launches on the task's
 * default stream and synchronizes after every stage (models.jl:142-179). */
int cdft_plan_set_stream(cdft_plan* plan, void* stream);

/* Average device time of one launch of a converge! stage over the systems of
 * `plans` (the profiles currently held by the plans, e.g. after a converge),
 * timed with CUDA events on the plans' stream after 3 warm-up launches:
 * stage 0 weighted densities (evaluate_field!), 1 fused Phi/dPhi (AD stage),
 * 2 adjoint convolutions (integrate_field!), 3 the whole δFδρ_res! evaluation.
 * Instrumentation for roofline accounting; no reference counterpart. */
int cdft_batch_time_stage(cdft_plan* const* plans, int nplans, int stage, int reps, double* ms_per_launch);

/* dF/drho (residual functional derivative plus external field) computed
 * without allocating any device memory.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc -- hosts whose device memory
 * is owned entirely by a memory pool or caching allocator that must see every
 * allocation (a CUDA.jl or PyTorch process running at its pool limit), or
 * services that reserve their whole device budget at start-up and forbid
 * allocations afterwards.  It takes no plan (plan creation allocates): the
 * system comes as a descriptor, d_rho and d_dFdrho are caller-owned device
 * arrays of N*nc doubles, desc->vext is a host array or NULL, stream is a
 * cudaStream_t or NULL for the default stream; the call returns after the
 * stream has finished its work.  The call runs on the calling thread's current
 * CUDA device; the arrays and the stream must belong to that device (a stream
 * of another device is rejected with CDFT_E_INVALID).
 *
 * Scratch (kernel tables, weighted densities, partial sums) lives in one
 * fixed array of CDFT_NOALLOC_SCRATCH_BYTES inside the library, which every
 * GPU that loads the library holds until the process exits.  Limits: 1D
 * Cartesian, FP64, N <= CDFT_NOALLOC_MAX_N and N*nc <= CDFT_NOALLOC_MAX_ELEM;
 * larger systems are rejected with CDFT_E_UNSUPPORTED.  The first call on a
 * device looks up the array's device address (once per device); make that
 * first call before any stream capture.  That address is kept for the life of
 * the process: do not call this entry point again after cudaDeviceReset on that
 * device (the reset ends the context the address belongs to; plans are likewise
 * invalid after a reset).  All calls share the one array, so
 * calls that overlap on the GPU (from two host threads or two streams) race
 * and must be serialised by the caller.  Every value a call reads from the
 * array is written earlier in the same call, so no clearing is needed. */
#define CDFT_NOALLOC_SCRATCH_BYTES (4u * 1024u * 1024u)
#define CDFT_NOALLOC_MAX_N 4096
#define CDFT_NOALLOC_MAX_ELEM 8192
int cdft_functional_derivative_noalloc(const cdft_system_desc* desc, const double* d_rho, double* d_dFdrho,
                                       void* stream);

/* Launch shapes of the autotuner (cdft.jl_b200/tune.py), process-wide, by name: e.g.
 * "pers_warp_aa_max_elem" (persistent engine: systems of at most this many elements run
 * the Anderson vector slots on one warp).  The defaults are the tuned values; _set
 * overrides one (CDFT_E_INVALID for an unknown name or a value out of range).  No
 * counterpart in the reference (KernelAbstractions picks its own launch shapes). */
int cdft_tuning_get(const char* name, int* value);
int cdft_tuning_set(const char* name, int value);

/* Number of our kernel launches issued by the calling thread since the last
 * reset (instrumentation for benchmarks). */
long long cdft_launch_count(int reset);

/* Copy the last error message of the calling thread into buf (NUL-terminated);
 * returns the code of that error (0 if none). */
int cdft_last_error(char* buf, size_t len);

/* Library version string. */
const char* cdft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CDFT_B200_H */
