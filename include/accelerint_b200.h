/*
 * accelerint_b200 -- batched stiff-ODE integration on one NVIDIA B200 (sm_100a),
 * a drop-in for accelerInt's GPU library interface.
 *
 * The three legacy entry points keep the reference's signatures and meaning:
 *
 *   accelerInt_initialize   generic/solver_interface.cuh:35  (solver_interface.cu:88-147)
 *   accelerInt_integrate    generic/solver_interface.cuh:49  (solver_interface.cu:161-211)
 *   accelerInt_cleanup      generic/solver_interface.cuh:55  (solver_interface.cu:217-225)
 *
 * Layout (unchanged from the reference, examples/main.dox:70-82): y_host is
 * column-major with the IVP index fastest, y_host[i * NUM + ivp], overwritten
 * with the state at t_end; var_host[ivp] is the per-system parameter
 * (pressure in Pa for the mass-action mechanism, mu for van der Pol).
 *
 * Differences from the reference, by design:
 *   - no process exit on a failed system or CUDA error: the legacy void calls
 *     record the status (accelerInt_last_status) and per-system codes
 *     (accelerInt_get_codes, the reference's EC_* values 0..4, plus
 *     ACCELERINT_EC_NONFINITE where the reference would report success for a
 *     system whose final state is not finite);
 *   - no cudaDeviceReset in initialize/cleanup (it destroys other users'
 *     contexts in the same process);
 *   - solver, mechanism, tolerances and precision are chosen at run time
 *     through the extension calls below (the reference fixes them at compile
 *     time: generic/solver_props.h:9-16, SConstruct:181-185);
 *   - the global-step loop runs t_start -> t_end in steps of stepsize measured
 *     from t_start (the reference's GPU loop measures from 0 and seeds t_next
 *     from the end_time macro, solver_interface.cu:166,209).
 *
 * Thread safety: one integrator instance per process, as in the reference
 * (process-global state, solver_interface.cu:18-28).
 */
#ifndef ACCELERINT_B200_H
#define ACCELERINT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- legacy interface (generic/solver_interface.cuh) ---- */

/* Select the device (< 0 means 0) and size device memory for up to NUM systems
 * per batch.  Replaces solver_interface.cuh:35. */
void accelerInt_initialize(int NUM, int device);

/* Integrate NUM systems from t_start to t_end in global steps of stepsize
 * (stepsize < 0: one step of t_end - t_start).  Synchronous: y_host holds the
 * result when the call returns.  Replaces solver_interface.cuh:49-50. */
void accelerInt_integrate(const int NUM, const double t_start, const double t_end,
                          const double stepsize, double* y_host, const double* var_host);

/* Release device memory.  Replaces solver_interface.cuh:55. */
void accelerInt_cleanup(void);

/* ---- extensions (no counterpart in the reference's interface) ---- */

/* status codes returned by the extension calls */
#define ACCELERINT_OK 0
#define ACCELERINT_ERR_ARGUMENT -1      /* invalid argument */
#define ACCELERINT_ERR_CUDA -2          /* a CUDA call failed */
#define ACCELERINT_ERR_STATE -3         /* not initialised / no mechanism */
#define ACCELERINT_ERR_UNSUPPORTED -4   /* (solver, mechanism size, precision) not built */
#define ACCELERINT_ERR_SYSTEMS -5       /* at least one system returned a nonzero EC_* code */

/* Per-system code beyond the reference's EC_* values 0..4 (radau2a_props.h:288-296):
 * the integrator finished without an error but the final state holds a NaN or an
 * infinity.  The reference returns 0 for such a system (e.g. exp4, whose error norm
 * accepts a NaN estimate); here it is reported. */
#define ACCELERINT_EC_NONFINITE 5

/* solvers (generic/solver_props.h:9-16 selects one of these at compile time) */
#define ACCELERINT_RADAU2A 0
#define ACCELERINT_EXPRB43 1
#define ACCELERINT_EXP4 2
#define ACCELERINT_RKC 3

/* precision of the Radau simplified-Newton matrices E1/E2 */
#define ACCELERINT_LU_FP64 0
#define ACCELERINT_LU_FP32 1       /* complex E2 factored + solved in FP32, real E1 (error estimate) in FP64;
                                      residuals, error estimate, step control in FP64 */
#define ACCELERINT_LU_FP32_ALL 2   /* E1 and E2 in FP32; the error-estimate solve gets one FP64 refinement step */

/* Synthetic constant-pressure mass-action mechanism (plain tables; see
 * accelerint_b200/mechanism.py for the model).  Stands in for the pyJac
 * dydt/eval_jacob slot (examples/van_der_pol/dydt.h, jacob.h). */
typedef struct {
    int n_species;          /* K; state length N = K + 1 (T, Y_1..Y_K) */
    int n_reactions;        /* R */
    const double* mw;       /* [K] kg/mol */
    const double* cp;       /* [K] J/mol/K */
    const double* h_form;   /* [K] J/mol at 298.15 K */
    const double* s_ref;    /* [K] J/mol/K at 298.15 K */
    const int* reac;        /* [R*2] reactant species, -1 = empty slot */
    const int* prod;        /* [R*2] product species, -1 = empty slot */
    const double* log_a;    /* [R] ln A, (cm^3/mol)^(order-1)/s */
    const double* beta;     /* [R] temperature exponent */
    const double* ta;       /* [R] activation temperature Ea/R [K] */
} accelerInt_mass_action;

int accelerInt_set_solver(int solver);
int accelerInt_set_mechanism_van_der_pol(void);
int accelerInt_set_mechanism_mass_action(const accelerInt_mass_action* mech);
int accelerInt_set_tolerances(double atol, double rtol);   /* defaults 1e-10 / 1e-6 */
int accelerInt_set_lu_precision(int precision);             /* ACCELERINT_LU_FP64 (default) */
/* Radau IIA starting values of the simplified Newton iteration after an accepted
 * step (RK_Interpolate, radau2a/radau2a.c:302-314): 0 (default) the reference's,
 * which evaluates Z3 with x2 in its outer factor (radau2a.c:312), for trajectory
 * parity with the reference; 1 the collocation polynomial of the last step
 * evaluated at all three new nodes (x3 in both factors), a change of the starting
 * values only -- the error estimate still accepts or rejects every step.  Every
 * entry point honours it. */
int accelerInt_set_stage_extrapolation(int mode);

/* Like accelerInt_integrate, returning ACCELERINT_OK, ACCELERINT_ERR_SYSTEMS or an error. */
int accelerInt_integrate_status(int NUM, double t_start, double t_end, double stepsize,
                                double* y_host, const double* var_host);

/* Device-resident form: y_dev[i * NUM + ivp] and var_dev[NUM] are device
 * pointers; codes_dev[NUM] (optional, may be NULL) receives the EC_* code of
 * each system; stats_dev (optional) receives ACCELERINT_NSTATS int counters per
 * system, stats_dev[ivp * ACCELERINT_NSTATS + k], added to what the array holds
 * (zero it before the first call).  Asynchronous on `stream`
 * (a cudaStream_t, NULL = the legacy default stream). */
#define ACCELERINT_NSTATS 10  /* steps, accept, reject, jac, decomp, newton, rhs, errsolve, krylov dims, arnoldi calls */
int accelerInt_integrate_device(int NUM, double t_start, double t_end, double stepsize,
                                double* y_dev, const double* var_dev, int* codes_dev,
                                int* stats_dev, void* stream);

/* Allocation-free form of accelerInt_integrate_device, for hosts that cannot
 * let a library allocate device memory during a run -- for example a CFD code
 * that plans all device memory up front or hands out memory from its own pool,
 * or a caller that must not risk the device-wide synchronisation that
 * cudaMalloc/cudaFree can imply.  No counterpart in the reference (its
 * library allocates in accelerInt_initialize).  The caller passes the device
 * state y_dev[i * NUM + ivp], var_dev[NUM] and optionally codes_dev[NUM];
 * the integrator's own scratch (a work-queue counter and one N x N Jacobian
 * per system in flight) lives in a 16 MiB array compiled into the library,
 * which every GPU that loads the library holds until the process exits.
 * Limits: mass-action mechanism and Radau only; the number of systems in flight
 * is capped by what fits in 16 MiB (719 at N = 54, so it can be slower than
 * accelerInt_integrate_device); a state length whose single N x N Jacobian does
 * not fit is rejected with ACCELERINT_ERR_ARGUMENT.  The Jacobian mode and LU
 * precision are honoured as accelerInt_integrate_device honours them (finite
 * differences: plain FP64 only); with learned proposals or step recording
 * installed the call returns ACCELERINT_ERR_UNSUPPORTED.  The first call on a
 * device looks up the array's device address; make that first call before any
 * stream capture.  accelerInt_initialize and accelerInt_cleanup drop the looked-up
 * addresses, so the next call looks them up again.  All calls share the array:
 * calls that overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller.  accelerInt_initialize and the mechanism setters must
 * have run before. */
int accelerInt_integrate_device_noalloc(int NUM, double t_start, double t_end, double stepsize,
                                        double* y_dev, const double* var_dev, int* codes_dev, void* stream);

int accelerInt_last_status(void);
/* Copies the EC_* codes of the last accelerInt_integrate* call (host pointer, NUM entries). */
int accelerInt_get_codes(int* codes_host, int NUM);
/* Poles and residues of the (10,10) Caratheodory-Fejer approximant of exp on
 * (-inf, 0] that the exp methods use, computed on the host for the current ATOL
 * (exponential_integrators/rational_approximant.c:23-44, cf.c:41-312); no GPU
 * needed.  Conjugate pairs, positive imaginary part first. */
int accelerInt_get_poles(double* poles_re, double* poles_im, double* res_re, double* res_im);
/* ---- Learned step proposals (extension; no counterpart in the reference) ----
 * A multilayer perceptron 64 -> 128 -> 128 -> 128 -> 176 (GELU) maps the state at
 * the start of a Radau step -- T, log10 max(Y_k, 1e-20), log10 of the last
 * accepted step size, log10(P / 1 atm) -- to symlog-scaled initial Newton stage
 * values and log10 of the next step size over the last accepted one.  Parameters are one FP32 vector
 * (W0 b0 W1 b1 W2 b2 W3 b3, W_l row-major [out x in]); the solver and the
 * kernels below compute with BF16-rounded weights and activations and FP32
 * accumulation.  norm holds in_mu[64] in_sd[64] out_mu[176] out_sd[176].
 * All pointers are device pointers; M (batch) must be a multiple of 16. */
#define ACCELERINT_MLP_USE_H 1   /* limit step growth: min(controller, max(proposal, floor x last accepted)) */
#define ACCELERINT_MLP_USE_Z 2   /* start Newton from the proposed stages; on failure retry from the extrapolation */
int accelerInt_mlp_sizes(int* nparam, int* nnorm, int* d_in, int* d_out);
/* y[M x 176] = de-standardised network output for raw inputs x[M x 64] */
int accelerInt_mlp_forward(const float* params_dev, const float* norm_dev, const float* x_dev, int M, float* y_dev,
                           void* stream);
/* loss = sum_m sum_j w_j (f(xs_m)_j - ts_mj)^2 / M on standardised xs[M x 64], ts[M x 176]; grad[nparam] */
int accelerInt_mlp_loss_grad(const float* params_dev, const float* xs_dev, const float* ts_dev, const float* w_dev,
                             int M, float* grad_dev, float* loss_dev, void* stream);
/* one Adam update (bias-corrected) of the FP32 parameters */
int accelerInt_mlp_adam_step(float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, int step,
                             float lr, float beta1, float beta2, float eps, void* stream);
/* Install (flags != 0) or remove (flags == 0) the model for the mass-action Radau
 * kernels; the parameter and norm buffers must stay valid while installed. */
int accelerInt_set_learned(const float* params_dev, const float* norm_dev, int flags);
/* Growth floor of ACCELERINT_MLP_USE_H (default 2): the proposal limits the step to
 * no less than floor x the last accepted step.  1.05 <= floor <= 8. */
int accelerInt_set_learned_growth_floor(double floor);
/* Capture one record per accepted Radau step (block teams): raw features [64] then
 * raw targets [176] -- symlog(Z_c,i / (atol + rtol |y_i|)) for c = 1..3, then
 * log10(H / H_previous) -- into rec_dev[capacity][240]; *count_dev counts records claimed (it may
 * exceed capacity; the surplus is dropped).  rec_dev == NULL switches capture off. */
int accelerInt_set_step_recording(float* rec_dev, int* count_dev, int capacity);

/* ---- Launch mapping and CUDA-graph launches (extensions) ----
 * accelerInt_set_graph_launch(1): accelerInt_integrate_device records each call's
 * launch sequence (work-queue reset + kernel) by stream capture into a cached
 * executable graph (updated in place when only the arguments change) and
 * launches that graph on the caller's stream.
 * accelerInt_set_launch_config: resident blocks per SM of the persistent team
 * kernels (0: occupancy maximum) and the block size of the thread-per-system
 * kernels (0: unchanged).
 * accelerInt_set_queue_order: order in which the persistent teams take systems:
 * 0 index order; 1 largest y_0 first (the temperature of a mass-action state:
 * hot systems are the stiff ones); 2 most Radau steps in the previous call first
 * (mode 1 on the first call); 3 largest learned cost first: a model installed
 * with accelerInt_set_cost_model (the MLP layout above, output 0 = predicted
 * log10(1 + Radau steps) of the call from the state's features with h = t_end -
 * t_start) is evaluated for every system on the tensor cores before the launch.
 * Longest-first order shortens the tail of a launch, whose end waits for the
 * slowest system.  Every call of this setter starts the step-count history afresh.
 * accelerInt_set_mapping: team_lanes 0 runs a mass-action system on the default
 * team (one warp for state lengths up to 32, two warps up to 64); 16 runs two
 * systems per warp, 16 lanes each, for state lengths up to 16 (Radau with the
 * analytic Jacobian and no learned proposals; other settings keep the default
 * team).  grain: work-queue slots a persistent team claims per atomic (1..64).
 * Results do not depend on grain; with team_lanes 16 the team reductions run over
 * 16 lanes, so results agree with the default team to rounding, not bit for bit.
 * accelerInt_get_mapping: the current team_lanes, grain and the resident blocks
 * per SM of the last persistent launch.
 * accelerInt_autotune: times the candidate mappings (resident blocks per SM,
 * then queue order 0 / 1, then two systems per warp where the state fits 16
 * lanes, then the queue granularity 1 / 2 / 4 / 8; or the thread-per-system
 * block size) on a copy of the first `sample` systems of y_dev (grown to 16 per
 * resident team, at most NUM, for the team kernels) for the given interval
 * (y_dev is not modified) and keeps the fastest (a candidate must beat the current
 * choice by 3 %); reports the choice
 * (occupancy_cap_out: cap | order << 16; the rest through accelerInt_get_mapping)
 * and its time. */
int accelerInt_set_graph_launch(int enable);
/* enable = 1 (default): the team kernels run a persistent grid (resident
 * blocks x SMs) whose teams pull systems from a device work queue.  enable = 0:
 * the plain form, one team per system over a grid of NUM teams (one Jacobian
 * scratch per system). */
int accelerInt_set_persistent(int enable);
/* Jacobian of the mechanism: 0 analytic (default); 1 first-order finite
 * differences over dydt with the increments of generic/fd_jacob.c (the
 * reference's FINITE_DIFFERENCE build), for plain FP64 Radau. */
int accelerInt_set_jacobian(int mode);
int accelerInt_set_queue_order(int mode);
int accelerInt_set_cost_model(const float* params_dev, const float* norm_dev);
int accelerInt_set_launch_config(int occupancy_cap, int tps_block);
int accelerInt_set_mapping(int team_lanes, int grain);
int accelerInt_get_mapping(int* team_lanes, int* grain, int* occupancy);
int accelerInt_autotune(int NUM, double t_start, double t_end, double stepsize, const double* y_dev,
                        const double* var_dev, int sample, int* occupancy_cap_out, int* tps_block_out,
                        double* best_ms_out);

/* Diagnostic: the factorisations of the Radau simplified-Newton matrices alone.
 * For each of `count` Jacobians jac_dev[m * n * n + i + j * n] (column-major) and
 * step sizes h_dev[m], factors E1 = (gamma/h) I - J and E2 = ((alpha + i beta)/h) I - J
 * with the routine the Radau kernels use at `precision` (RK_Decomp,
 * radau2a/radau2a.c:256-278: partial-pivot LU with xGETF2 semantics) and writes
 * the factors column-major: e1_dev[m * n * n + ...] (double, or float for
 * ACCELERINT_LU_FP32_ALL), e2_dev (interleaved complex: double pairs for
 * ACCELERINT_LU_FP64, float pairs otherwise), perm_dev[m * 2n + position] = original
 * row (E1 then E2) and info_dev[2m], info_dev[2m + 1] (k + 1 at the first zero
 * pivot, else 0).  State lengths n = 14 and 54.  Device pointers; asynchronous. */
int accelerInt_radau_decomp(int n, int precision, int count, const double* jac_dev, const double* h_dev,
                            void* e1_dev, void* e2_dev, int* perm_dev, int* info_dev, void* stream);

/* Extension: number of kernels this library has launched in the process. */
long long accelerInt_kernel_launches(void);
const char* accelerInt_version(void);

/* Diagnostic: measured FMA throughput of the current device in TFLOP/s (FMA = 2
 * flops): fp64 = 1 double precision, 0 single precision (scalar FFMA), 2 single
 * precision as packed FP32x2 FMAs (two FMAs per instruction, the form the
 * single-precision factorisations use).  The roofline denominators of the
 * integrator kernels. */
int accelerInt_measure_fma_peak(int fp64, double* tflops);

#ifdef __cplusplus
}
#endif
#endif
