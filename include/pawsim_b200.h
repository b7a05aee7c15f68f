/*
 * pawsim_b200.h -- C ABI of the B200 implementation of PAWSIM's timestep hot path.
 *
 * The library keeps one model's layered fields resident on one GPU and replaces the
 * reference's hot-path entry points (paths are within the reference project):
 *
 *   pawsim_gpu_tendency_eval       <- pawsim_tendency_eval        model_code/tendency.c:81-115
 *                                                                  (model_code/tendency.h:20-22)
 *   pawsim_gpu_integrator_step     <- pawsim_integrator_step      model_code/integrator.c:138-198
 *                                                                  (model_code/integrator.h:20)
 *   pawsim_gpu_pressure_correct    <- pawsim_pressure_correct_rigid_lid
 *                                                                  model_code/pressure.c:2254-2300
 *                                                                  (model_code/pressure.h:16)
 *   pawsim_gpu_prelim              <- timeSteppingPreliminaries   model_code/pawsim.c:266-304
 *   pawsim_gpu_step                <- one pass of the main loop   model_code/pawsim.c:471-492
 *   pawsim_gpu_solve_mg            <- solve_MG                     model_code/multigrid.c:1304-1343
 *                                                                  (model_code/multigrid.h:12-24)
 *
 * Conventions: plain pointers and sizes, no library types in the signatures. Host arrays
 * are float64, x fastest (the AWSIM disk order), Nx*Ny values per 2-D field. Return codes
 * are 0 on success and negative PAWSIM_GPU_E* values on failure; the text of the last
 * failure is available from pawsim_gpu_last_error(). A handle is not thread-safe; its work
 * runs on one CUDA stream (the default stream unless pawsim_gpu_set_stream is called).
 */
#ifndef PAWSIM_B200_H
#define PAWSIM_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define PAWSIM_API __attribute__((visibility("default")))
#else
#define PAWSIM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PAWSIM_GPU_OK 0
#define PAWSIM_GPU_EBADCONFIG (-1)
#define PAWSIM_GPU_ECUDA (-2)
#define PAWSIM_GPU_ENOTCONVERGED (-3)
#define PAWSIM_GPU_ENONFINITE (-4)
#define PAWSIM_GPU_EUNSUPPORTED (-5)
#define PAWSIM_GPU_EBADNAME (-6)

/* Solver identifiers (model_code/config.h:12-15). */
#define PAWSIM_GPU_SOLVER_SOR 0
#define PAWSIM_GPU_SOLVER_MG 1
#define PAWSIM_GPU_SOLVER_MG_DISTRIBUTED 2

/* Mirrors the parsed parameters of pawsim_config (model_code/config.h:17-130) that the hot
 * path reads; derived feature flags are passed as parsed (config.c:285-312). */
typedef struct pawsim_gpu_config
{
  int Nx, Ny, Nlay;
  int wall_ew, wall_ns;
  int ts_scheme;            /* 3 AB1, 4 AB2, 5 AB3 */
  int mom_scheme;           /* 0 AL81, 1 HK83, 2 S75e, 3 TW81 */
  int thick_scheme;         /* 0 AL81, 1 HK83, 2 UP3, 3 KT00 */
  int use_rl, ocean_surf_drag, wind_feedback;
  int use_wind, use_fbaro, use_relax, use_wdia, use_diavisc, use_wdia_file;
  int tau_nrecs, wdia_nrecs;
  int solver;               /* PAWSIM_GPU_SOLVER_* (pressureSolver, or use_MG 0/1) */
  int use_full_mg, maxiters, pressure_timing;
  double Lx, Ly, dt, tmin;
  double A2, A4, A2smag, A4smag, h0, hsml, hmin_surf, hbbl, hmin_bot, KT00_sigma;
  double lin_drag, quad_drag, lin_drag_surf, quad_drag_surf;
  double tau_period, wdia_period, conv_diff;
  double pi_tol, sor_rp, omega_mg;
  /* GPU multigrid controls: 0 FP64 V-cycles, 1 FP32 V-cycles inside FP64 defect
   * correction; red-black sweeps before/after the coarse correction and their weight
   * (0 selects the defaults 1, 1, 1.0). A negative mg_omega lets the solver choose the
   * weight on its first time-step solve: each of 1.0, 1.05, 1.1, 1.15, 1.2, 1.3 solves from
   * the same pi and the one with the fewest V-cycles is kept. */
  int mg_fp32, mg_pre, mg_post;
  double mg_omega;
  /* Global sums (the pressure RHS mean, the solve norms and the energy diagnostics):
   * 1 in the reference's serial order (bitwise parity), 0 in a fixed pairwise tree,
   * -1 serial order for grids of at most 65536 cells. */
  int serial_sums;
  /* Shape of the multigrid's fused level kernels: 0 times every shape on each level
   * when the solver is first used and keeps the fastest; 1..4 forces one tile shape
   * (32x8, 32x16, 64x8, 64x16 cells), 5 the streamed strips (levels of at least 64 x 48
   * cells). The shape changes only the speed, never the result. */
  int mg_tile;
  /* tracer b (work.c:1947-2144): useTracer, tracerScheme (0 AL81, 1 UP3, 2 KT00) and the
   * Laplacian / biharmonic diffusivities K2, K4 (the buoyancy coupling is use_buoyancy
   * below, its diapycnal diffusion use_diadiff). */
  int use_tracer, tracer_scheme;
  double K2, K4;
  /* First guess of the multigrid solves (pressureSolver 1 and 2): 0 the previous pressure,
   * as the reference; 1 the linear extrapolation 2 pi(n-1) - pi(n-2) of the last two
   * solutions (from the third solve on). The stopping test is unchanged, so the solution
   * meets the same tolerance; only the number of V-cycles changes. SOR ignores it. */
  int pi_guess;
  /* Tendency budgets kept on the device (work.c:1753-1937 and the terms of forcing.c,
   * restoring.c, diapycnal.c and the pressure correction): a bit mask of the families,
   * PAWSIM_GPU_BUDGET_UMOM (savefreqUMom), _VMOM, _THIC, _ENERGY, _TRAC. Each step then adds
   * every term times dt to its running sum; the sums are read with pawsim_gpu_get_field under
   * the reference's output names (UMom_PVadvection, ..., Tracer_relaxation; k = layer). */
  int budgets;
  /* useBuoyancy: the tracer acts as a buoyancy anomaly in the Bernoulli pressure, the
   * momentum (-hz db/dx), the tracer's diapycnal advection and the local reduced gravity of
   * the convective viscosity (convDiff); needs use_tracer. */
  int use_buoyancy;
  /* useDiaDiff (diaDiffFile, bFluxFile or convDiff != 0) with a tracer: diapycnal diffusion of
   * b through the interfaces (diapycnal.c:140-197) with the diffusivity kappa_dia per
   * interface and the surface flux Fsurf_b (fields of those names). */
  int use_diadiff;
  /* With mg_fp32 = 1: FP32 V-cycles per FP64 defect-correction step (0 or 1: one; at most 8).
   * Each after the first continues from the correction the previous one left, so a step
   * reduces the defect further before the FP64 residual pass; stats.iters counts steps. */
  int mg_fp32_inner;
  /* Failure reporting (no counterpart in the reference, which prints "WARNING: PAWSIM pressure
   * solve reached maxiters" and runs on, to NaN if the state blows up). Both are off (0) by
   * default, which keeps the reference's behaviour. check_nonfinite = K > 0: the fused step
   * kernel raises a device flag when a new u, v or h is not finite (NaN or infinite); every K-th
   * call of pawsim_gpu_step / pawsim_gpu_integrator_step reads and clears it and returns
   * PAWSIM_GPU_ENONFINITE when it was raised. fail_on_maxiters = 1: a rigid-lid solve that
   * stopped at maxiters makes pawsim_gpu_step / pawsim_gpu_pressure_correct return
   * PAWSIM_GPU_ENOTCONVERGED. In both cases the step itself completes as the reference's does
   * (the state is advanced and the report filled), so the caller may inspect or continue. */
  int check_nonfinite;
  int fail_on_maxiters;
  /* Corner ghosts on x-periodic, y-walled grids (the only domain where the two builds of the
   * reference differ): 0 reproduces the serial build (model_code/field.c:353-532 copies whole
   * columns periodically before filling the wall rows, so the corner ghosts of a work array
   * keep the values of its previous fill; those feed the PV, viscosity and face-thickness
   * stencils next to the walls at the periodic seam); 1 uses the current values there, as the
   * MPI build's y-then-x exchange does. Other domains are unaffected. */
  int mpi_corners;
} pawsim_gpu_config;

enum
{
  PAWSIM_GPU_BUDGET_UMOM = 1,
  PAWSIM_GPU_BUDGET_VMOM = 2,
  PAWSIM_GPU_BUDGET_THIC = 4,
  PAWSIM_GPU_BUDGET_ENERGY = 8,
  PAWSIM_GPU_BUDGET_TRAC = 16
};

/* Per-solve report, the numbers of the "PAWSIM pressure solve" line (pawsim.c:100-108). */
typedef struct pawsim_gpu_stats
{
  int iters;                 /* SOR iterations or V-cycles */
  double residual_max, residual_rms;   /* rhs - L(pi), pressure.c:652-690 (pressure_timing) */
  double div_max, div_rms;             /* sum_k div(h u) after projection, pressure.c:693-737 */
  double stop_measure;       /* value of the solver's own stopping test at exit */
  double solve_ms;           /* device time of the solve alone (with the warm start's guess) */
  int warm_start;            /* learned warm start: 0 none, 1 guess used, 2 guess rejected
                                (the solve started from the previous pressure) */
  int fallback;              /* 1 when pressureSolver 2 fell back to the gathered multigrid
                                (grid without a first clean 2:1 coarsening) */
  double mg_omega;           /* red-black weight the gathered multigrid used (0 for SOR, DMG) */
} pawsim_gpu_stats;

typedef struct pawsim_gpu pawsim_gpu;

PAWSIM_API int pawsim_gpu_create (const pawsim_gpu_config * cfg, pawsim_gpu ** out);
PAWSIM_API void pawsim_gpu_destroy (pawsim_gpu * m);

/* Upload or read one input/state field by name. Names and shapes:
 *   u v h uRelax vRelax hRelax eRelax uTime vTime eTime nu_u_dia nu_v_dia  (k = layer)
 *   hhs hhb uLid vLid Fbaro_x Fbaro_y hTime                                 (k = 0)
 *   omegaz (Nx+1)*(Ny+1), taux tauy (k = record), wdia_ff (k = record*(Nlay+1)+interface)
 *   gg (vector of Nlay, n = Nlay)
 * Readable only: pi, pi_rhs, dt_u dt_v dt_h (last tendency), wdia (k <= Nlay), Hc.
 * n is the number of doubles in host. */
PAWSIM_API int pawsim_gpu_set_field (pawsim_gpu * m, const char * name, int k, const double * host, size_t n);
PAWSIM_API int pawsim_gpu_get_field (pawsim_gpu * m, const char * name, int k, double * host, size_t n);

/* Finish set-up after the uploads: wall faces, pressure operator, multigrid hierarchy. */
PAWSIM_API int pawsim_gpu_init (pawsim_gpu * m);

PAWSIM_API int pawsim_gpu_tendency_eval (pawsim_gpu * m);
PAWSIM_API int pawsim_gpu_integrator_step (pawsim_gpu * m, unsigned n);
PAWSIM_API int pawsim_gpu_pressure_correct (pawsim_gpu * m, int update_diags, pawsim_gpu_stats * st);
PAWSIM_API int pawsim_gpu_prelim (pawsim_gpu * m, pawsim_gpu_stats * st);
/* integrator step n followed by the rigid-lid correction (one pass of pawsim.c:471-492) */
PAWSIM_API int pawsim_gpu_step (pawsim_gpu * m, unsigned n, pawsim_gpu_stats * st);
/* nsteps passes starting at step n0 (the main loop of pawsim.c:471-511 without its outputs);
 * st receives the last step's report. Steps whose correction needs no report formed on the
 * host (SOR or the gathered multigrid once its first solves have tuned it, without
 * pressure_timing or the learned warm start) are enqueued back to back without a host
 * synchronisation: their iteration counts go to a device ring read once at the end (st's
 * solve_ms and norms are 0 for them). check_nonfinite and fail_on_maxiters are evaluated at the
 * end of the run. */
PAWSIM_API int pawsim_gpu_run (pawsim_gpu * m, unsigned n0, unsigned nsteps, pawsim_gpu_stats * st);
/* The iteration count of each step of the last pawsim_gpu_run (n = its nsteps): the numbers of
 * the reference's per-step "PAWSIM pressure solve" lines (pawsim.c:95-108). */
PAWSIM_API int pawsim_gpu_run_iterations (pawsim_gpu * m, int * iters, size_t n);

/* Batched ensemble (no reference counterpart: the reference runs one model per process, its
 * multigrid state being file-scope globals, model_code/multigrid.c:54-63; this replaces n such
 * processes). Members are initialised models of any grid sizes that share Nlay, the momentum
 * and thickness schemes, use_rl and the fused kernel's feature set, without tracer, budgets or
 * a quadratic drag over a fraction depth. create moves each member onto its own stream (destroy
 * gives back the previous one). run advances every member nsteps integrator steps numbered
 * n0.. : per step one launch of the fused kernel over all members' tiles, then each member's
 * rigid-lid correction on its own stream, with no host synchronisation until the end; each
 * member's results equal those of pawsim_gpu_run on that member alone, and its per-step
 * iteration counts are read with pawsim_gpu_run_iterations. Members must outlive the
 * ensemble and are not stepped on their own while it exists; after an error return of run
 * the members' states are unspecified. */
typedef struct pawsim_gpu_ensemble pawsim_gpu_ensemble;
PAWSIM_API int pawsim_gpu_ensemble_create (pawsim_gpu * const * members, int n, pawsim_gpu_ensemble ** out);
PAWSIM_API int pawsim_gpu_ensemble_run (pawsim_gpu_ensemble * e, unsigned n0, unsigned nsteps);
/* Mean device time (ms) of one step's batched fused-kernel launch (with its exact pass) over
 * the stream-mode steps of the last run, from CUDA events on the ensemble's launch stream
 * (0 when every step replayed a graph). */
PAWSIM_API double pawsim_gpu_ensemble_kernel_ms (const pawsim_gpu_ensemble * e);
/* Steps whose every member has a fixed form (AB3 with its history shifting, the multigrid
 * loop built, no host-side warm start) run as replays of CUDA graphs that capture the whole
 * step, one per arrangement of the members' state buffers; on = 0 keeps every step on streams.
 * Results are identical either way. graph_steps: how many steps of the last run replayed. */
PAWSIM_API int pawsim_gpu_ensemble_set_graphs (pawsim_gpu_ensemble * e, int on);
PAWSIM_API int pawsim_gpu_ensemble_graph_steps (const pawsim_gpu_ensemble * e);
/* 1 when the captured steps solve every member's pressure in one batched multigrid loop (all
 * members use the multigrid with FP64 cycles, one smoothing sweep each way, no use_fullMG):
 * per V-cycle one launch per level for all members of a grid size, the loop running until
 * every member meets its own stopping test; each member's solution and V-cycle count are
 * those of its own solve. 0 when the members' solves are captured one by one. */
PAWSIM_API int pawsim_gpu_ensemble_batched_mg (const pawsim_gpu_ensemble * e);
PAWSIM_API void pawsim_gpu_ensemble_destroy (pawsim_gpu_ensemble * e);

/* Online time averages (diagnostics.c:307-470, the savefreqAvg outputs). accumulate adds
 * avg_fac * dt times the current state to the running sums (call it after each step, with
 * avg_fac = 1, or 1 - (t - t_next_avg) / dt on the step that crosses the window's end, as
 * pawsim_diagnostics_accumulate_averages does); scale multiplies every sum by factor
 * (1 / savefreqAvg when a window is written); zero resets them. The sums are read with
 * pawsim_gpu_get_field under the output names U_avg, V_avg, H_avg, M_avg, HU_avg, HV_avg,
 * HUU_avg, HVV_avg, HUV_avg, B_avg (tracer; k < Nlay), W_avg (k <= Nlay) and P_avg. They live in device
 * memory allocated by the first call of accumulate. */
PAWSIM_API int pawsim_gpu_accumulate_averages (pawsim_gpu * m, double avg_fac);
PAWSIM_API int pawsim_gpu_scale_averages (pawsim_gpu * m, double factor);
PAWSIM_API int pawsim_gpu_zero_averages (pawsim_gpu * m);

/* Budget windows (pawsim_diagnostics_write_budgets_if_due, diagnostics.c:756-866): scale
 * multiplies every sum of the families in `mask` by factor (1 / ((n - n_prev) dt) when a
 * family's window is written); zero resets them. The sums accumulate in
 * pawsim_gpu_integrator_step / pawsim_gpu_step (the tendency, forcing, restoring, diapycnal
 * and tracer terms) and in the step's pressure correction (the Montgomery terms). */
PAWSIM_API int pawsim_gpu_scale_budgets (pawsim_gpu * m, int mask, double factor);
PAWSIM_API int pawsim_gpu_zero_budgets (pawsim_gpu * m, int mask);

/* Energy and enstrophy diagnostics (replaces the sums of pawsim_diagnostics_write_EZ_if_due,
 * model_code/diagnostics.c:478-700, whose line of EZdiags.dat the caller writes): the
 * domain's kinetic energy *KE, potential energy *PE and the potential enstrophy Z[k] of each
 * of the Nlay layers, for the current state. The interface heights are built upward from the
 * bottom topography with the layer thickness the reference last copied into its work arrays:
 * the current one (eta_from_step_start = 0; rigid lid, or online averages on, which reload the
 * state every step) or the thickness at the start of the last step (1; free surface without
 * averages), which needs a step since the last upload of h. The sums follow
 * serial_sums: the reference's serial order (layer, x, y), or a fixed tree. Synchronous. */
PAWSIM_API int pawsim_gpu_energy (pawsim_gpu * m, int eta_from_step_start, double * KE, double * PE,
                                  double * Z);

/* Asynchronous state output (replaces the synchronous reads and writes of
 * pawsim_diagnostics_write_model_state, model_code/diagnostics.c:874-908; no reference
 * counterpart for the overlap). save_begin copies, on the device and in stream order with the
 * steps, the planes of one save into one of two staging slots: u, v, h (and b with a tracer)
 * of each layer in turn, w_dia on the Nlay+1 interfaces, and pi under the rigid lid
 * (pawsim_gpu_save_planes planes of Nx*Ny doubles, x fastest). Their device-to-host copy into
 * page-locked memory held by the library runs on a second stream, and the call returns at once
 * with the slot index: the model steps on while the copy and the caller's file writes proceed.
 * save_wait (any thread) blocks until the slot's host copy is complete and returns it;
 * save_release hands the slot back. save_begin blocks (up to 600 s) while its slot is held. */
PAWSIM_API int pawsim_gpu_save_begin (pawsim_gpu * m, int * slot);
PAWSIM_API int pawsim_gpu_save_wait (pawsim_gpu * m, int slot, const double ** host);
PAWSIM_API int pawsim_gpu_save_release (pawsim_gpu * m, int slot);
PAWSIM_API size_t pawsim_gpu_save_planes (const pawsim_gpu * m);

/* Solve L(pi) = rhs on the resident pi/pi_rhs with the GPU multigrid (no projection). */
PAWSIM_API int pawsim_gpu_solve_mg (pawsim_gpu * m, pawsim_gpu_stats * st);

/* Use the caller's CUDA stream (a cudaStream_t passed as void*) for all later work. */
PAWSIM_API int pawsim_gpu_set_stream (pawsim_gpu * m, void * stream);
PAWSIM_API int pawsim_gpu_synchronize (pawsim_gpu * m);
PAWSIM_API double pawsim_gpu_time (const pawsim_gpu * m);
/* kernels this library launched since creation (the launch counter) */
PAWSIM_API long long pawsim_gpu_launch_count (const pawsim_gpu * m);
PAWSIM_API const char * pawsim_gpu_last_error (void);
/* Self-check of the library's correctly rounded division by a known divisor (used by the
 * stencils for 1/dx, 1/dy, 1/24 and per-cell thickness) against the GPU's IEEE division on
 * n host values x / d; *bad receives the number of results that differ in any bit. */
PAWSIM_API int pawsim_gpu_check_division (const double * x, size_t n, double d, long long * bad);

/* ---- Learned pressure warm start: network building blocks (no reference counterpart).
 * Device pointers; activations NHWC bf16 with C in {16, 32, 48, 64}; weights [Cout][3][3][Cin]
 * bf16; dev_err (nullable) is a device int set to 1 when a bounded wait inside a kernel
 * gave up. Convolutions run on the tcgen05 tensor cores with FP32 accumulation. */
PAWSIM_API int pawsim_nn_conv3x3 (const void * in_bf16, int B, int H, int W, int Cin, const void * w_bf16,
                                  const float * bias, int Cout, int relu, void * out_bf16, float * out_f32,
                                  int * dev_err, void * stream);
/* dw[co][ky][kx][ci] += sum_p dout[p][co] in[p shifted][ci]; db[co] += sum_p dout[p][co] (FP32) */
PAWSIM_API int pawsim_nn_conv3x3_wgrad (const void * in_bf16, const void * dout_bf16, int B, int H, int W,
                                        int Cin, int Cout, float * dw, float * db, int * dev_err,
                                        void * stream);
/* w_t[ci][ky][kx][co] = w[co][2-ky][2-kx][ci]: input-gradient weights of a convolution */
PAWSIM_API int pawsim_nn_flip_weights (const void * w_bf16, int Cout, int Cin, void * w_t_bf16, void * stream);

/* ---- Learned warm start of a model's multigrid solve (no reference counterpart).
 * mode bit 0: after every solve, store a training pair (network inputs and the solved
 * correction) in a device ring of max_pairs pairs; bit 1: start each solve from the trained
 * network's guess when its stopping measure is below that of the previous pressure.
 * batch: training batch size. Needs the multigrid solver and a grid whose side, coarsened
 * to at most 512 cells, is a multiple of 8. The first call allocates; later calls change
 * the mode only. */
PAWSIM_API int pawsim_gpu_nn_setup (pawsim_gpu * m, int mode, int max_pairs, int batch,
                                    unsigned long long seed);
/* Adam (learning rate lr) over the collected pairs for `epochs` passes; *loss receives the
 * last epoch's mean squared error of the normalised correction. */
PAWSIM_API int pawsim_gpu_nn_train (pawsim_gpu * m, int epochs, float lr, double * loss);
PAWSIM_API int pawsim_gpu_nn_pairs (pawsim_gpu * m);
/* the model's network (owned by the model: do not destroy), for pawsim_nn_net_* below */
PAWSIM_API void * pawsim_gpu_nn_net (pawsim_gpu * m);

/* A standalone warm-start network on an H x W grid (multiples of 8) for batches of at most
 * Bmax: parameters flattened per layer as w[Cout][3][3][Cin] then b[Cout] (FP32 master
 * copy; the kernels use its bf16 rounding). forward/backward take device inputs
 * (B, H, W, 16) bf16; forward copies output channel 0 (B, H, W) to the host; backward
 * recomputes the loss mean((out0 - target)^2) and all parameter gradients. */
PAWSIM_API int pawsim_nn_net_create (int H, int W, int Bmax, unsigned long long seed, void ** net);
PAWSIM_API void pawsim_nn_net_destroy (void * net);
PAWSIM_API long long pawsim_nn_net_param_count (void * net);
PAWSIM_API int pawsim_nn_net_get_params (void * net, float * host, size_t n);
PAWSIM_API int pawsim_nn_net_set_params (void * net, const float * host, size_t n);
PAWSIM_API int pawsim_nn_net_get_grads (void * net, float * host, size_t n);
PAWSIM_API int pawsim_nn_net_forward (void * net, const void * in_bf16, int B, float * out_host);
PAWSIM_API int pawsim_nn_net_backward (void * net, const void * in_bf16, const float * target, int B,
                                       double * loss);
PAWSIM_API int pawsim_nn_net_adam (void * net, float lr);

/* No counterpart in the reference. For callers that cannot allocate device memory (code
 * running under an allocator or memory pool it does not own, hosts that forbid device
 * allocation after start-up): builds the rigid-lid right-hand side, sum_k div(h_k u_k)/dt
 * with its mean removed, from device arrays the caller holds (u, v, h: Nlay planes of Ny
 * rows x pitch doubles, thickness already corrected to the column constraint) into the
 * caller's device array rhs (Ny rows x pitch), on `stream` (a cudaStream_t, may be NULL).
 * It allocates nothing: the partial sums of the mean use a static device array of 4096
 * doubles, so grids are limited to Ny <= 32760 rows (any Nx); larger grids, Nx or Ny
 * below 4 and thickness schemes other than AL81/HK83 are rejected with an error code.
 * serial_sum: 1 sums in the reference's serial order, 0 in a fixed tree, -1 picks the
 * serial order for grids of at most 65536 cells. The first call on a device looks up the
 * array's device address, so make it before any stream capture. All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller. */
PAWSIM_API int pawsim_pressure_rhs_noalloc (const double * u, const double * v, const double * h,
                                            int Nx, int Ny, int Nlay, int pitch, double dx, double dy,
                                            double dt, int wall_ew, int wall_ns, int thick_scheme,
                                            int serial_sum, double * rhs, void * stream);

#ifdef __cplusplus
}
#endif

#endif
