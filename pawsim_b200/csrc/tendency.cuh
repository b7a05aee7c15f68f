// tendency.cuh -- parameters of the fused tendency + Adams-Bashforth kernel.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace pawsim {

constexpr int LMAX = 8;   // layers supported by the fused kernel

struct TendParams {
  int Nx, Ny, L, pitch, qpitch;
  size_t lstride;                 // elements between layers
  int wall_ew, wall_ns;
  int use_rl;
  double dx, dy;
  double rdx, rdy, r24;           // 1/dx, 1/dy, 1/24 rounded to nearest (for div_rn)
  // Adams-Bashforth epilogue. mode 0 writes the tendency itself to f_out.
  int ab_mode;                    // 0: tendency only, 1: AB1, 2: AB2, 3: AB3
  double c0, c1, c2;              // AB coefficients, computed on the host as the reference does
  int write_hist;                 // store the new tendency into f_out
  int fuse_thickness_fix;         // apply the rigid-lid column correction to the new h
  // state and history
  const double *u, *v, *h;        // S_n
  double *u_out, *v_out, *h_out;  // S_{n+1} (or unused in mode 0)
  const double *f1u, *f1v, *f1h;  // tendency one step back
  const double *f2u, *f2v, *f2h;  // tendency two steps back (may alias f_out)
  double *fu_out, *fv_out, *fh_out;
  // statics
  const double *hhb, *hhs, *Hc, *omz;
  double gg[LMAX], geff[LMAX];
  double h0;
  double A2, A4sqrt;
  int useA2, useA4;
  // Smagorinsky coefficients (work.c:1587-1610): A2f * |D|, A4f * |D| with floors A2, A4
  int use_smag;
  double A2f, A4f, A4;
  double kt00_sigma;              // KT00 slope limiter (thickness scheme 3)
  // forcing (model_code/forcing.c)
  int use_wind, use_fbaro;
  const double *taux0, *taux1, *tauy0, *tauy1;
  double tw0, tw1;
  const double *fbx, *fby;
  double lin_drag, lin_drag_surf;
  double quad_drag, quad_drag_surf;   // quadratic bottom / surface drag coefficients
  double wfb;                         // wind feedback: 0.3 when windFeedback, else 0
  int ocean_surf_drag;
  // surface / bottom layer fractions (work.c:2151-2340); off when both depths are <= 0
  int use_fractions;
  double hsml, hmin_surf, hbbl, hmin_bot;
  const double *uLid, *vLid;
  // restoring and diapycnal (model_code/restoring.c, diapycnal.c)
  int use_relax, use_wdia, use_wdia_file, use_diavisc;
  const double *wd0, *wd1;        // wDia records n0, n1 (L+1 interfaces each)
  double ww0, ww1;
  const double *hRelax, *eRelax, *eTime, *hTime;
  const double *uRelax, *vRelax, *uTime, *vTime;
  const double *nu_u, *nu_v;
  // outputs for diagnostics
  double *wdia_out;               // interface velocities [L+1] (nullable)
  // tendency budgets (work.c:1753-1937, forcing.c:243-389, restoring.c:190-214,
  // diapycnal.c:243-284): running sums of each term times dt, one family per array of
  // [term][layer] planes lstride apart, nullptr when the family is off. Used only by the
  // budget build of the kernel (launch_tendency_budget).
  double dt;
  double *bud_u, *bud_v, *bud_h, *bud_e, *bud_b;
  const double* b;                // tracer at the start of the step (budgets, buoyancy)
  // the tracer as a buoyancy anomaly (useBuoyancy; work.c:190-212, 1438-1452, 1745-1748,
  // 1829-1832; diapycnal.c:40-66, 104-114): also only in the budget build
  int use_buoy;
  double conv_diff;               // convDiff: added viscosity where the local g' < 0
  // set to 1 when a new u, v or h is not finite (nullable: no check)
  int* nonfinite;
  // corner shadow of the previous fill (common.cuh; nullable: corner ghosts hold the current
  // values, as in the MPI build)
  const double* corners;
  // quadratic drag over a fraction depth (forcing.c:95-143, 181-223): planes of the
  // thickness-weighted bottom-boundary-layer velocity u_bot, v_bot (hbbl > 0) and surface
  // mixed-layer velocity u_surf, v_surf (hsml > 0), written by a pre-pass of the same launch;
  // nullptr when the drag acts on the bottom (top) layer alone
  double* dragv;
  int drag_bot, drag_surf;
  // tiles for the exact recomputation of the plain build: [0] count, [1] completion counter of
  // the exact pass (both zero between launches), [2..] tile indices (one slot per tile)
  int* tile_list;
};

// budget term indices (work.h:18-91)
enum { BU_Q, BU_GRADM, BU_GRADKE, BU_DHDT, BU_A2, BU_A4, BU_RDRAG, BU_RSURF, BU_CDBOT, BU_CDSURF,
       BU_WIND, BU_BUOY, BU_RELAX, BU_WDIA, BU_FBARO, BU_DIAVISC, BU_NTERMS };
enum { BH_ADV, BH_RELAX, BH_NTERMS };
enum { BE_ADV, BE_GRADM, BE_WIND, BE_RDRAG, BE_RSURF, BE_CDBOT, BE_CDSURF, BE_A2, BE_A4, BE_WDIAPE,
       BE_WDIAKE, BE_FBARO, BE_BUOY, BE_RELAX, BE_DIAVISC, BE_NTERMS };
enum { BB_ADV, BB_WDIA, BB_K2, BB_K4, BB_DIADIFF, BB_RELAX, BB_NTERMS };

// family[term][k] += v at one cell (a no-op for a family that is off)
__device__ inline void budget_add(double* fam, int term, int k, int L, size_t lstride, size_t cell, double v) {
  if (fam) {
    double* q = fam + ((size_t)term * L + k) * lstride + cell;
    *q = *q + v;
  }
}

// returns the number of kernels launched, or -1 when the combination is not available
int launch_tendency(const TendParams& p, int momentum_scheme, int thickness_scheme,
                    cudaStream_t stream);
// tile height (16 or 8 rows) launch_tendency uses for this set-up
int tendency_tile_height(const TendParams& p, int thickness_scheme);

// The set-up needs none of the paths the lean instantiation of the fused kernel leaves out
// (w_dia, restoring, diapycnal viscosity, fractions, Fbaro, A4, Smagorinsky, corner shadow,
// quadratic and surface drag, buoyancy); the launch then takes the lean build.
inline bool tendency_lean(const TendParams& p) {
  return !p.use_wdia && !p.use_relax && !p.use_diavisc && !p.use_fractions && !p.use_fbaro && !p.useA4 &&
         !p.use_smag && !p.corners && !(p.quad_drag > 0) && !(p.quad_drag_surf > 0) && !(p.lin_drag_surf > 0) &&
         !p.drag_bot && !p.drag_surf && !p.use_buoy;
}
// The fused step of several members in one launch (ensemble): ps (device) holds each member's
// parameters, work (device) the (member << 20 | tile) pairs of nwork tiles, on the tile height
// tendency_tile_height gives; the members share p0's momentum and thickness schemes, feature
// set and layer count. Then the exact pass over every member's tile list (done: a device int,
// zero between launches). Returns the kernels launched, or -1.
int launch_tendency_batch(const TendParams& p0, const TendParams* ps, const int* work, int nwork, int members,
                          int* done, int momentum_scheme, int thickness_scheme, cudaStream_t stream);
// the same step with every enabled budget family accumulated and the buoyancy coupling
// (32 x 8 tiles)
int launch_tendency_budget(const TendParams& p, int momentum_scheme, int thickness_scheme,
                           cudaStream_t stream);

}  // namespace pawsim
