// pressure.cuh -- rigid-lid pressure kernels: RHS, mean removal, red-black SOR,
// projection and the solve-quality diagnostics.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace pawsim {

struct Grid2 {
  int Nx, Ny, pitch, L;
  size_t lstride;
  int wall_ew, wall_ns;
  double dx, dy, dt;
  int thick_scheme;
  double rdx, rdy, rdxdt, rdydt;   // reciprocals rounded to nearest, for div_rn
  double kt00_sigma;               // KT00 slope-limiter factor (thick_scheme 3)
};

// rhs = sum_k div(h_k u_k) / dt with the gathered face thickness (pressure.c:570-606)
int launch_pressure_rhs(const Grid2& g, const double* u, const double* v, const double* h,
                         double* rhs, cudaStream_t s);

// Record the corner shadow (common.cuh) of a work-array fill of the state u, v, h (b nullable)
// into `next`.
void launch_corner_capture(const Grid2& g, const double* u, const double* v, const double* h, const double* b,
                           double* next, cudaStream_t s);

// sum of the owned cells in the reference's serial order (x outer, y inner) or in a fixed
// pairwise tree; the result is written to *out (device). `partials` needs
// reduce_scratch_elems(n) doubles.
size_t reduce_scratch_elems(int Nx, int Ny);
void launch_sum(const double* f, int Nx, int Ny, int pitch, bool serial_order, double* partials,
                double* out, cudaStream_t s);
// f -= mean, mean = *sum / (Nx*Ny) (pressure.c:55-88)
void launch_subtract_mean(double* f, int Nx, int Ny, int pitch, const double* sum, cudaStream_t s);

// operator coefficients Ow, Os (pressure.c:609-637) and the SOR factor SOR_rp/Osum
struct Operator {
  double* Ow;    // (Nx+1) columns x Ny rows, pitch `opitch`
  double* Os;    // Nx columns x (Ny+1) rows, pitch `opitch`
  double* csor;  // Nx x Ny, pitch `pitch`; 0 marks a cell whose Osum is zero
  int opitch;
};
void launch_operator(const Grid2& g, const double* Hc, const Operator& op, double sor_rp,
                     cudaStream_t s);

// red-black SOR (pressure.c:743-814) as one persistent cooperative kernel; the iteration
// count is written to *iters (device int).
int launch_sor(const Grid2& g, double* pi, const double* rhs, const Operator& op, double sor_rp,
               double tol, int maxiters, unsigned long long* slots, int* iters, cudaStream_t s);

// u -= dt dpi/dx, v -= dt dpi/dy on every layer, skipping wall faces (pressure.c:2182-2248)
void launch_projection(const Grid2& g, const double* pi, double* u, double* v, cudaStream_t s);
// the same, adding the Montgomery terms of the u, v and energy budgets (nullable families)
void launch_projection_budget(const Grid2& g, const double* pi, double* u, double* v, const double* h, double* bu,
                              double* bv, double* be, cudaStream_t s);

// per-cell residual rhs - L(pi) and barotropic divergence (pressure.c:652-737)
void launch_residual_field(const Grid2& g, const double* pi, const double* rhs,
                           const Operator& op, double* out, cudaStream_t s);
int launch_divergence_field(const Grid2& g, const double* u, const double* v, const double* h,
                             double* out, cudaStream_t s);
// Running time averages of the state (diagnostics.c:307-375): at every cell each field
// is incremented by dtfac * value. u, v, h, M (Montgomery potential plus pi under the
// rigid lid), h_west u, h_south v, h_west u^2, h_south v^2 and hq uq vq (q-point means) per
// layer, w_dia per interface, pi; face thickness gathered as in the pressure RHS. Per-layer
// arrays are lstride apart.
constexpr int AVG_LMAX = 8;
struct AvgParams {
  double dtfac;
  int use_rl;
  double h0;
  double gg[AVG_LMAX], geff[AVG_LMAX];
  const double *u, *v, *h, *pi, *hhb, *wdia;
  double *au, *av, *ah, *aM, *aW, *ahu, *ahv, *ahuu, *ahvv, *ahuv, *api;
  const double* b;   // tracer (nullable) and its sums
  double* ab;
  int use_buoy;      // the tracer as buoyancy in the Montgomery potential (work.c:1438-1452)
};
void launch_accumulate_averages(const Grid2& g, const AvgParams& a, cudaStream_t s);
// f[i] *= factor for n contiguous doubles
void launch_scale(double* f, size_t n, double factor, cudaStream_t s);

// Kinetic and potential energy of the domain and the potential enstrophy of each layer
// (diagnostics.c:478-700). h, u, v are the current state; eta is built upward from hhb with
// the thickness `hw` (the state the reference last copied into its work arrays). Results go
// to out[0] = KE, out[1] = PE, out[2 + k] = Z_k (device). serial_order sums every cell in the
// reference's order (layer, then x, then y) from per-cell terms in `terms`
// (ez_scratch_elems doubles); otherwise a fixed tree sums per-block partials held in `terms`.
struct EzParams {
  double h0;
  double geff[AVG_LMAX];
  const double *u, *v, *h, *hw, *hhb, *omz;
  int qpitch;
  const double* b;   // useBuoyancy: g_tot = geff - b (diagnostics.c:653-655), else nullptr
};
size_t ez_scratch_elems(const Grid2& g, bool serial_order);
int launch_energy(const Grid2& g, const EzParams& e, bool serial_order, double* terms, double* out,
                  cudaStream_t s);

// max |f| and sum f^2 (serial order or tree) into out[0], out[1]
void launch_norms(const double* f, int Nx, int Ny, int pitch, bool serial_order,
                  double* partials, double* out, cudaStream_t s);

}  // namespace pawsim
