// tracer.cuh -- the passive tracer equation and its Adams-Bashforth update.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace pawsim {

// One step of the tracer b (model_code/work.c:1947-2144 without the buoyancy coupling and
// the diapycnal diffusion, and integrator.c:15-198): advection by the layer mass fluxes in
// the AL81 / UP3 / KT00 form, Laplacian (K2) and biharmonic (K4) diffusion weighted by the
// face thickness, diapycnal advection by w_dia, relaxation to bRelax on bTime, then the
// same AB1/AB2/AB3 update and history rotation as the momentum and thickness.
struct TracerParams {
  int Nx, Ny, L, pitch;
  size_t lstride;
  int wall_ew, wall_ns;
  int scheme;          // tracerScheme: 0 AL81, 1 UP3, 2 KT00
  int thick_scheme;    // thicknessScheme of the face thickness (0 AL81, 1 HK83, 2 UP3, 3 KT00)
  double kt00_sigma;   // KT00_sigma (both KT00 limiters)
  double dx, dy, K2, K4;
  double rdx, rdy, rdxsq, rdysq;    // 1/dx, 1/dy, 1/(dx dx), 1/(dy dy) rounded to nearest (div_rn)
  int use_wdia;
  const double *u, *v, *h, *b;      // state at the start of the step
  const double *bRelax, *bTime;
  const double* wdia;               // interface velocities of the same tendency evaluation
  int ab_mode;                      // 0: tendency only (into fb_out), 1: AB1, 2: AB2, 3: AB3
  double c0, c1, c2;
  int write_hist;
  const double *f1b, *f2b;
  double *fb_out, *b_out;
  // Tracer_* budget (work.c:2131-2136): [term][layer] planes lstride apart, or nullptr
  double* bud_b;
  double dt;
  // useBuoyancy: the diapycnal jumps include the layers' reduced gravities (work.c:2088-2093)
  int use_buoy;
  double gg[8];
  // diapycnal diffusion (diapycnal.c:140-197, work.c:2098-2102): interface diffusivity
  // kappa_dia (layer planes; interface k between layers k-1 and k), surface flux Fsurf_b
  int use_diadiff;
  const double *kappa, *fsurf;
  double conv_diff;
  // corner shadow of the previous fill (common.cuh; nullable: current corner values)
  const double* corners;
};

void launch_tracer(const TracerParams& p, cudaStream_t s);

}  // namespace pawsim
