/*
 * pawsim_oracle.h -- CPU restatement of PAWSIM's timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA path is compared
 * against; nothing in the product links it. It restates, in serial C on ghosted
 * arrays, the algorithm of the reference's serial build:
 *
 *   tendency (model_code/tendency.c:81-115 and the stages it calls in work.c,
 *   forcing.c, restoring.c, diapycnal.c), Adams-Bashforth stepping
 *   (model_code/integrator.c:138-198) and the rigid-lid pressure correction
 *   (model_code/pressure.c:2254-2300) with red-black SOR (pressure.c:743-814) and the
 *   serial AWSIM multigrid (model_code/multigrid.c:196-1343).
 *
 * Every stage keeps the reference's loop extents, zeroing and halo-fill order, so the
 * results are bit-identical to the reference build for closed basins, doubly periodic
 * domains and x-walled/y-periodic channels. One deliberate difference: for x-periodic,
 * y-walled domains the reference fills the four corner ghost blocks of scalar/u/v fields
 * from values left over by the previous fill (the periodic x copy in field.c:137-150 runs
 * before the y-wall fill of field.c:158-198, which covers only owned columns). This
 * oracle fills corners as the composition of the two fills instead.
 *
 * Storage: x-fastest interior arrays at the API (the AWSIM disk order).
 * Pinning: tests/test_oracle_pin.py compares this library with the reference binary
 * built by oracle/Makefile and with the committed fixtures under tests/golden/.
 */
#ifndef PAWSIM_ORACLE_H
#define PAWSIM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_cfg
{
  int Nx, Ny, Nlay;
  int wall_ew, wall_ns;
  int ts_scheme;      /* 3 = AB1, 4 = AB2, 5 = AB3 (defs.h:23-25) */
  int mom_scheme;     /* 0 AL81, 1 HK83, 2 S75e, 3 TW81 (defs.h:29-32) */
  int thick_scheme;   /* 0 AL81, 1 HK83, 2 UP3, 3 KT00 (defs.h:35-38) */
  int use_rl, ocean_surf_drag, wind_feedback;
  int use_wind, use_fbaro, use_relax, use_wdia, use_diavisc, use_wdia_file;
  int tau_nrecs, wdia_nrecs;
  int solver;         /* 0 SOR, 1 gathered MG, 2 distributed MG */
  int use_full_mg, maxiters, pressure_timing;
  double Lx, Ly, dt, tmin;
  double A2, A4, A2smag, A4smag, h0, hsml, hmin_surf, hbbl, hmin_bot, KT00_sigma;
  double lin_drag, quad_drag, lin_drag_surf, quad_drag_surf;
  double tau_period, wdia_period, conv_diff;
  double pi_tol, sor_rp, omega_mg;
  /* 1: halo fills in the serial build's order (model_code/field.c:353-532: periodic copies,
   * then wall ghosts), whose corner ghosts on x-periodic, y-walled grids keep the values of
   * the array's previous fill; 0: walls first (the MPI build's order, current corners) */
  int serial_corners;
} orc_cfg;

typedef struct orc_model orc_model;

typedef struct orc_pstats
{
  int iters;
  double residual_max, residual_rms, div_max, div_rms;
} orc_pstats;

orc_model * orc_create (const orc_cfg * cfg);
void orc_destroy (orc_model * m);

/*
 * Load or read a field. Names: u v h (per layer), hhs hhb, omegaz ((Nx+1)x(Ny+1)),
 * taux tauy (k = record), uLid vLid Fbaro_x Fbaro_y, uRelax vRelax hRelax eRelax
 * uTime vTime eTime (per layer), hTime, wdia_ff (k = rec*(Nlay+1)+interface),
 * nu_u_dia nu_v_dia (per layer), gg (vector, length Nlay).
 * Readable work fields: dt_u dt_v dt_h h_west h_south eta(k<=Nlay) zeta hhq qq alpha
 * beta gamma delta epsilon phi lambda mu pp KE MM wdia(k<=Nlay) pi pi_rhs Hc Hw Hs
 * hhs_west hhs_south hhb_west hhb_south, tend_u tend_v tend_h (history level k/Nlay).
 * Returns 0 on success, -1 for an unknown name or index.
 */
int orc_set (orc_model * m, const char * name, int k, const double * src);
int orc_get (orc_model * m, const char * name, int k, double * dst);

/* Finish loading: fill halos of all inputs, compute geff (state.c:957-1100). */
int orc_init (orc_model * m);

/* One tendency evaluation at the model time into the newest history level. */
int orc_tendency (orc_model * m);

/* Work arrays plus the deterministic core, without a tendency copy (tendency.c:38-75). */
void orc_prepare_and_core (orc_model * m);

/* The time-stepping preliminaries of pawsim.c:266-304 (without output). */
int orc_prelim (orc_model * m, orc_pstats * st);

/* One explicit step n (integrator.c:138-198). */
int orc_integrator_step (orc_model * m, int n);

/* The rigid-lid correction (pressure.c:2254-2300). */
int orc_pressure (orc_model * m, int update_diags, orc_pstats * st);

/* n steps of the main loop, starting at step index n0 (pawsim.c:471-492). */
int orc_run_steps (orc_model * m, int n0, int nsteps, orc_pstats * last);

double orc_time (const orc_model * m);

/* Kinetic and potential energy and per-layer potential enstrophy of the current state
 * (diagnostics.c:478-700); reload = copy the state into the work arrays first. */
int orc_energy (orc_model * m, int reload, double * ke, double * pe, double * z);

#ifdef __cplusplus
}
#endif

#endif
