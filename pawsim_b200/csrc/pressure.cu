// pressure.cu -- rigid-lid pressure kernels (RHS, mean, SOR, projection, diagnostics).
//
// Compiled with -fmad=false; every expression keeps the association order of
// model_code/pressure.c so the SOR path reproduces the reference bit for bit.
#include <cooperative_groups.h>

#include "common.cuh"
#include "pressure.cuh"
#include "tendency.cuh"

namespace cg = cooperative_groups;

namespace pawsim {

namespace {

__device__ inline double ld_s(const double* f, const Grid2& g, int i, int j) {
  return load_mapped(f, g.pitch, i, j, g.Nx, g.Ny, g.wall_ew, g.wall_ns, MAP_S, MAP_S);
}

// minmod of three slopes (defs.c:1000-1014): zero unless all share a sign, else the smallest
__device__ inline double minmod3(double a, double b, double c) {
  if ((a > 0) && (b > 0) && (c > 0)) return fmin(a, fmin(b, c));
  if ((a < 0) && (b < 0) && (c < 0)) return fmax(a, fmax(b, c));
  return 0;
}

// Gathered face thickness with wrapped indices (work.c:865-1030), at an owned cell; u, v are
// the layer's velocities (the upwind schemes read their sign at the face).
__device__ inline double hw_gathered(const Grid2& g, const double* h, const double* u, int i, int j) {
  int Nx = g.Nx, Ny = g.Ny;
  int im1 = i == 0 ? Nx - 1 : i - 1;
  int jm1 = j == 0 ? Ny - 1 : j - 1, jp1 = j + 1 == Ny ? 0 : j + 1;
  const int P = g.pitch;
#define H(ii, jj) h[(size_t)(jj) * P + (ii)]
  if (g.thick_scheme == 1) {
    if (g.wall_ns && j == 0)
      return (1.0 / 3) * (1.25 * (H(i, j) + H(im1, j)) + 0.25 * (H(i, jp1) + H(im1, jp1)));
    if (g.wall_ns && j == Ny - 1)
      return (1.0 / 3) * (1.25 * (H(i, j) + H(im1, j)) + 0.25 * (H(i, jm1) + H(im1, jm1)));
    return (1.0 / 3) * (H(i, j) + H(im1, j) + 0.25 * (H(i, jp1) + H(im1, jp1) + H(i, jm1) + H(im1, jm1)));
  }
  if (g.thick_scheme >= 2) {
    const int im2 = im1 == 0 ? Nx - 1 : im1 - 1, ip1 = i + 1 == Nx ? 0 : i + 1;
    const double uc = u[(size_t)j * P + i];
    if (g.thick_scheme == 2) {
      // UP3 (work.c:600-629): centred mean minus a sixth of the upwind second difference
      const double d2m = H(i, j) - 2 * H(im1, j) + H(im2, j);
      const double d2c = H(ip1, j) - 2 * H(i, j) + H(im1, j);
      return 0.5 * (H(i, j) + H(im1, j)) - (1 / 6.0) * ((uc > 0) ? d2m : d2c);
    }
    // KT00 (work.c:630-684): limited linear reconstruction from the upwind side
    const double s = g.kt00_sigma;
    const double dm = minmod3(s * (H(i, j) - H(im1, j)), 0.5 * (H(i, j) - H(im2, j)), s * (H(im1, j) - H(im2, j)));
    const double dc = minmod3(s * (H(ip1, j) - H(i, j)), 0.5 * (H(ip1, j) - H(im1, j)), s * (H(i, j) - H(im1, j)));
    const double xm = H(im1, j) + 0.5 * dm;
    const double xp = H(i, j) - 0.5 * dc;
    return (uc > 0) ? xm : xp;
  }
  return 0.5 * (H(i, j) + H(im1, j));
}

__device__ inline double hs_gathered(const Grid2& g, const double* h, const double* v, int i, int j) {
  int Nx = g.Nx, Ny = g.Ny;
  int im1 = i == 0 ? Nx - 1 : i - 1, ip1 = i + 1 == Nx ? 0 : i + 1;
  int jm1 = j == 0 ? g.Ny - 1 : j - 1;
  const int P = g.pitch;
  if (g.thick_scheme == 1) {
    if (g.wall_ew && i == 0)
      return (1.0 / 3) * (1.25 * (H(i, j) + H(i, jm1)) + 0.25 * (H(ip1, j) + H(ip1, jm1)));
    if (g.wall_ew && i == Nx - 1)
      return (1.0 / 3) * (1.25 * (H(i, j) + H(i, jm1)) + 0.25 * (H(im1, j) + H(im1, jm1)));
    return (1.0 / 3) * (H(i, j) + H(i, jm1) + 0.25 * (H(ip1, j) + H(im1, j) + H(ip1, jm1) + H(im1, jm1)));
  }
  if (g.thick_scheme >= 2) {
    const int jm2 = jm1 == 0 ? Ny - 1 : jm1 - 1, jp1 = j + 1 == Ny ? 0 : j + 1;
    const double vc = v[(size_t)j * P + i];
    if (g.thick_scheme == 2) {
      const double d2m = H(i, j) - 2 * H(i, jm1) + H(i, jm2);
      const double d2c = H(i, jp1) - 2 * H(i, j) + H(i, jm1);
      return 0.5 * (H(i, j) + H(i, jm1)) - (1 / 6.0) * ((vc > 0) ? d2m : d2c);
    }
    const double s = g.kt00_sigma;
    const double dm = minmod3(s * (H(i, j) - H(i, jm1)), 0.5 * (H(i, j) - H(i, jm2)), s * (H(i, jm1) - H(i, jm2)));
    const double dc = minmod3(s * (H(i, jp1) - H(i, j)), 0.5 * (H(i, jp1) - H(i, jm1)), s * (H(i, j) - H(i, jm1)));
    const double ym = H(i, jm1) + 0.5 * dm;
    const double yp = H(i, j) + 0.5 * dc;   // the reference adds the half slope on this side too
    return (vc > 0) ? ym : yp;
  }
  return 0.5 * (H(i, j) + H(i, jm1));
#undef H
}

// the gathered face arrays are scalar-filled afterwards: a face one past the last cell
// copies the last face on a wall and the first face when periodic (field.c:121-241)
__device__ inline double hw_face(const Grid2& g, const double* h, const double* u, int i, int j) {
  if (i >= g.Nx) i = g.wall_ew ? 2 * g.Nx - i - 1 : i - g.Nx;
  return hw_gathered(g, h, u, i, j);
}
__device__ inline double hs_face(const Grid2& g, const double* h, const double* v, int i, int j) {
  if (j >= g.Ny) j = g.wall_ns ? 2 * g.Ny - j - 1 : j - g.Ny;
  return hs_gathered(g, h, v, i, j);
}

__device__ inline double ld_u(const Grid2& g, const double* u, int i, int j) {
  return load_mapped(u, g.pitch, i, j, g.Nx, g.Ny, g.wall_ew, g.wall_ns, MAP_N, MAP_S);
}
__device__ inline double ld_v(const Grid2& g, const double* v, int i, int j) {
  return load_mapped(v, g.pitch, i, j, g.Nx, g.Ny, g.wall_ew, g.wall_ns, MAP_S, MAP_N);
}

// divergence terms of one cell (all layers): the gathered face thickness of the thickness
// scheme at every face, with the boundary maps
__device__ double rhs_cell(const Grid2& g, const double* __restrict__ u, const double* __restrict__ v,
                           const double* __restrict__ h, int i, int j, int with_dt) {
  double acc = 0;
  const double dxdt = g.dx * g.dt, dydt = g.dy * g.dt;
  for (int k = 0; k < g.L; ++k) {
    const double* uk = u + k * g.lstride;
    const double* vk = v + k * g.lstride;
    const double* hk = h + k * g.lstride;
    const double hu_w = ld_u(g, uk, i, j) * hw_face(g, hk, uk, i, j);
    const double hu_e = ld_u(g, uk, i + 1, j) * hw_face(g, hk, uk, i + 1, j);
    const double hv_s = ld_v(g, vk, i, j) * hs_face(g, hk, vk, i, j);
    const double hv_n = ld_v(g, vk, i, j + 1) * hs_face(g, hk, vk, i, j + 1);
    if (with_dt)
      acc += div_rn(hu_e - hu_w, dxdt, g.rdxdt) + div_rn(hv_n - hv_s, dydt, g.rdydt);
    else
      acc += div_rn(hu_e - hu_w, g.dx, g.rdx) + div_rn(hv_n - hv_s, g.dy, g.rdy);
  }
  return acc;
}

// cells whose four faces lie between owned cells, with the AL81 face average
// (work.c:889-901): plain loads, no boundary maps; the border ring and the other thickness
// schemes go through rhs_cell
__global__ void rhs_inner_kernel(const Grid2 g, const double* __restrict__ u, const double* __restrict__ v,
                                 const double* __restrict__ h, double* __restrict__ rhs, int with_dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < 1 || j < 1 || i + 1 >= g.Nx || j + 1 >= g.Ny) return;
  const double dxdt = g.dx * g.dt, dydt = g.dy * g.dt;
  const size_t c = (size_t)j * g.pitch + i;
  const size_t P = g.pitch;
  double acc = 0;
#pragma unroll 2
  for (int k = 0; k < g.L; ++k) {
    const double* uk = u + k * g.lstride;
    const double* vk = v + k * g.lstride;
    const double* hk = h + k * g.lstride;
    const double hc = hk[c];
    const double hu_w = uk[c] * (0.5 * (hc + hk[c - 1]));
    const double hu_e = uk[c + 1] * (0.5 * (hk[c + 1] + hc));
    const double hv_s = vk[c] * (0.5 * (hc + hk[c - P]));
    const double hv_n = vk[c + P] * (0.5 * (hk[c + P] + hc));
    if (with_dt)
      acc += div_rn(hu_e - hu_w, dxdt, g.rdxdt) + div_rn(hv_n - hv_s, dydt, g.rdydt);
    else
      acc += div_rn(hu_e - hu_w, g.dx, g.rdx) + div_rn(hv_n - hv_s, g.dy, g.rdy);
  }
  rhs[c] = acc;
}

// every cell (all thickness schemes), or with `border` only the outermost ring of cells,
// enumerated as rows 0 and Ny-1, then columns 0 and Nx-1 of the rows between
__global__ void rhs_kernel(const Grid2 g, const double* __restrict__ u, const double* __restrict__ v,
                           const double* __restrict__ h, double* __restrict__ rhs, int with_dt, int border) {
  int i, j;
  if (border) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int rows = g.Ny > 1 ? 2 * g.Nx : g.Nx;
    if (p < rows) {
      i = p % g.Nx;
      j = p < g.Nx ? 0 : g.Ny - 1;
    } else {
      const int q = p - rows;
      if (g.Ny <= 2 || q >= 2 * (g.Ny - 2)) return;
      j = 1 + (q >> 1);
      i = (q & 1) ? g.Nx - 1 : 0;
    }
  } else {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.Nx || j >= g.Ny) return;
  }
  rhs[(size_t)j * g.pitch + i] = rhs_cell(g, u, v, h, i, j, with_dt);
}

// ---------------------------------------------------------------- reductions

constexpr int RED_BLOCK = 256;
constexpr int RED_ROWS = 8;   // rows per partial in the tree sum

// serial order of pressure.c:62-69: x outer, y inner (sequence index k = i * Ny + j). The
// dependent additions are one thread's (thread 0); the other warps stage the sequence into
// shared memory a chunk ahead, so that the additions read shared memory instead of waiting on
// strided global loads.
constexpr int SS_THREADS = 256, SS_CHUNK = 2048;
__global__ void __launch_bounds__(SS_THREADS) serial_sum_kernel(const double* __restrict__ f, int Nx, int Ny,
                                                                int pitch, double* out, int squares) {
  __shared__ __align__(16) double buf[2][SS_CHUNK];
  // grids of the serial order hold far fewer than 2^31 cells (the order is the reference's for
  // small grids; larger ones take it only when forced), so 32-bit sequence indices suffice
  const int n = Nx * Ny;
  const int nchunks = (n + SS_CHUNK - 1) / SS_CHUNK;
  auto stage = [&](int c, double* b) {
    for (int q = threadIdx.x - 32; q < SS_CHUNK; q += SS_THREADS - 32) {
      const int k = c * SS_CHUNK + q;
      if (k < n) {
        const int i = k / Ny, j = k - i * Ny;
        b[q] = f[(size_t)j * pitch + i];
      }
    }
  };
  if (threadIdx.x >= 32) stage(0, buf[0]);
  __syncthreads();
  double s = 0;
  for (int c = 0; c < nchunks; ++c) {
    if (threadIdx.x >= 32) {
      if (c + 1 < nchunks) stage(c + 1, buf[(c + 1) & 1]);
    } else if (threadIdx.x == 0) {
      const double* b = buf[c & 1];
      const int m = n - c * SS_CHUNK < SS_CHUNK ? n - c * SS_CHUNK : SS_CHUNK;
      int q = 0;
      // sixteen shared-memory loads in flight ahead of the chain of additions
      for (; q + 16 <= m; q += 16) {
        double a[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) a[r] = b[q + r];
#pragma unroll
        for (int r = 0; r < 16; ++r) s += squares ? a[r] * a[r] : a[r];
      }
      for (; q < m; ++q) s += squares ? b[q] * b[q] : b[q];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s;
}

// fixed-shape tree: each block sums RED_ROWS rows (one column per thread, looping over
// columns), then a fixed shuffle tree; a second pass adds the partials in index order.
__global__ void tree_partial_kernel(const double* __restrict__ f, int Nx, int Ny, int pitch,
                                    double* partials, int squares) {
  __shared__ double ws[RED_BLOCK / 32];
  int r0 = blockIdx.x * RED_ROWS;
  double s = 0;
  for (int r = r0; r < r0 + RED_ROWS && r < Ny; ++r)
    for (int i = threadIdx.x; i < Nx; i += RED_BLOCK) {
      double a = f[(size_t)r * pitch + i];
      s += squares ? a * a : a;
    }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_BLOCK / 32; ++w) t += ws[w];
    partials[blockIdx.x] = t;
  }
}

__global__ void tree_final_kernel(const double* partials, int n, double* out) {
  __shared__ double ws[RED_BLOCK / 32];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += RED_BLOCK) s += partials[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_BLOCK / 32; ++w) t += ws[w];
    out[0] = t;
  }
}

__global__ void max_abs_kernel(const double* __restrict__ f, int Nx, int Ny, int pitch,
                               unsigned long long* out) {
  // fmax semantics: NaN entries are ignored, as C's fmax does
  double m = 0;
  for (int j = blockIdx.y; j < Ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Nx; i += gridDim.x * blockDim.x)
      m = fmax(m, fabs(f[(size_t)j * pitch + i]));
  __shared__ double wm[32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, wm[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(b));
  }
}

__global__ void store_max_kernel(const unsigned long long* bits, double* out) {
  out[0] = __longlong_as_double((long long)bits[0]);
}

__global__ void subtract_mean_kernel(double* f, int Nx, int Ny, int pitch, const double* sum) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  double mean = sum[0] / ((double)Nx * (double)Ny);
  f[(size_t)j * pitch + i] -= mean;
}

// ------------------------------------------------------------------ operator

__global__ void operator_kernel(const Grid2 g, const double* __restrict__ Hc, Operator op, double sor_rp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  // Ow on faces i in [0, Nx], Os on faces j in [0, Ny] (pressure.c:609-637): Hw, Hs are the
  // centered averages of Hc (work.c:1160-1166), scalar-filled past the last cell.
  if (i <= g.Nx && j < g.Ny) {
    double Hw = 0.5 * (ld_s(Hc, g, i, j) + ld_s(Hc, g, i - 1, j));
    if (i == g.Nx) {
      int ii = g.wall_ew ? g.Nx - 1 : 0;
      Hw = 0.5 * (ld_s(Hc, g, ii, j) + ld_s(Hc, g, ii - 1, j));
    }
    double o = Hw / (g.dx * g.dx);
    if (g.wall_ew && (i == 0 || i == g.Nx)) o = 0;
    op.Ow[(size_t)j * op.opitch + i] = o;
  }
  if (i < g.Nx && j <= g.Ny) {
    double Hs = 0.5 * (ld_s(Hc, g, i, j) + ld_s(Hc, g, i, j - 1));
    if (j == g.Ny) {
      int jj = g.wall_ns ? g.Ny - 1 : 0;
      Hs = 0.5 * (ld_s(Hc, g, i, jj) + ld_s(Hc, g, i, jj - 1));
    }
    double o = Hs / (g.dy * g.dy);
    if (g.wall_ns && (j == 0 || j == g.Ny)) o = 0;
    op.Os[(size_t)j * op.opitch + i] = o;
  }
}

__global__ void sor_factor_kernel(const Grid2 g, Operator op, double sor_rp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  double Ow = op.Ow[(size_t)j * op.opitch + i], Oe = op.Ow[(size_t)j * op.opitch + i + 1];
  double Os = op.Os[(size_t)j * op.opitch + i], On = op.Os[(size_t)(j + 1) * op.opitch + i];
  double Osum = Ow + Oe + Os + On;
  op.csor[(size_t)j * g.pitch + i] = (Osum == 0) ? 0.0 : sor_rp / Osum;
}

// ----------------------------------------------------------------------- SOR

__device__ inline double sor_point(const Grid2& g, double* pi, const double* rhs, const Operator& op,
                                   double one_minus_w, int i, int j) {
  size_t c = (size_t)j * g.pitch + i;
  double cs = op.csor[c];
  if (cs == 0) return 0;   // Osum == 0: the reference skips the cell
  double Ow = op.Ow[(size_t)j * op.opitch + i], Oe = op.Ow[(size_t)j * op.opitch + i + 1];
  double Os = op.Os[(size_t)j * op.opitch + i], On = op.Os[(size_t)(j + 1) * op.opitch + i];
  double pn = ld_s(pi, g, i, j + 1), ps = ld_s(pi, g, i, j - 1);
  double pe = ld_s(pi, g, i + 1, j), pw = ld_s(pi, g, i - 1, j);
  double prev = pi[c];
  double nw = one_minus_w * prev + cs * (On * pn + Os * ps + Oe * pe + Ow * pw - rhs[c]);
  pi[c] = nw;
  double d = fabs(nw - prev);
  return d;
}

__global__ void __launch_bounds__(512) sor_kernel(const Grid2 g, double* pi, const double* __restrict__ rhs,
                                                  const Operator op, double sor_rp, double tol, int maxiters,
                                                  unsigned long long* slots, int* iters_out) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double wmax[16];
  const double one_minus_w = 1 - sor_rp;
  int iters = 0;
  double gmax = tol + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) { slots[0] = 0; slots[1] = 0; }
  grid.sync();
  while ((gmax > tol) && (iters < maxiters)) {
    double lmax = 0;
    for (int color = 0; color < 2; ++color) {
      // rows are dealt to blocks; within a row a thread visits only cells of this colour
      for (int j = blockIdx.x; j < g.Ny; j += gridDim.x)
        for (int i = 2 * threadIdx.x + ((j + color) & 1); i < g.Nx; i += 2 * blockDim.x) {
          double d = sor_point(g, pi, rhs, op, one_minus_w, i, j);
          lmax = fmax(lmax, d);
        }
      grid.sync();
    }
    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = lmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, wmax[w]);
      atomicMax(&slots[iters & 1], (unsigned long long)__double_as_longlong(b));
    }
    grid.sync();
    gmax = __longlong_as_double((long long)slots[iters & 1]);
    if (blockIdx.x == 0 && threadIdx.x == 0) slots[(iters + 1) & 1] = 0;
    ++iters;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) iters_out[0] = iters;
}

// ---------------------------------------------------------------- projection

__global__ void projection_kernel(const Grid2 g, const double* __restrict__ pi, double* __restrict__ u,
                                  double* __restrict__ v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  size_t c = (size_t)j * g.pitch + i;
  double pc = pi[c];
  double pw = i > 0 ? pi[c - 1] : ld_s(pi, g, i - 1, j);
  double ps = j > 0 ? pi[c - g.pitch] : ld_s(pi, g, i, j - 1);
  bool skip_u = g.wall_ew && i == 0;
  bool skip_v = g.wall_ns && j == 0;
  const double du = div_rn(-g.dt * (pc - pw), g.dx, g.rdx);
  const double dv = div_rn(-g.dt * (pc - ps), g.dy, g.rdy);
#pragma unroll 4
  for (int k = 0; k < g.L; ++k) {
    size_t o = k * g.lstride + c;
    if (!skip_u) u[o] += du;
    if (!skip_v) v[o] += dv;
  }
}

// the projection with its budget terms (pressure.c:2182-2245): the face thickness of the
// state being corrected (as in the RHS, with the velocity before the update) times the
// increment, and that times the updated velocity
__global__ void projection_budget_kernel(const Grid2 g, const double* __restrict__ pi, double* __restrict__ u,
                                         double* __restrict__ v, const double* __restrict__ h, double* bu,
                                         double* bv, double* be) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  size_t c = (size_t)j * g.pitch + i;
  double pc = pi[c];
  double pw = i > 0 ? pi[c - 1] : ld_s(pi, g, i - 1, j);
  double ps = j > 0 ? pi[c - g.pitch] : ld_s(pi, g, i, j - 1);
  bool skip_u = g.wall_ew && i == 0;
  bool skip_v = g.wall_ns && j == 0;
  const double du = div_rn(-g.dt * (pc - pw), g.dx, g.rdx);
  const double dv = div_rn(-g.dt * (pc - ps), g.dy, g.rdy);
  for (int k = 0; k < g.L; ++k) {
    const size_t o = k * g.lstride + c;
    const double* hk = h + k * g.lstride;
    if (!skip_u) {
      const double hw = hw_face(g, hk, u + k * g.lstride, i, j);
      const double un = u[o] + du;
      u[o] = un;
      budget_add(bu, BU_GRADM, k, g.L, g.lstride, c, hw * du);
      budget_add(be, BE_GRADM, k, g.L, g.lstride, c, hw * du * un);
    }
    if (!skip_v) {
      const double hs = hs_face(g, hk, v + k * g.lstride, i, j);
      const double vn = v[o] + dv;
      v[o] = vn;
      budget_add(bv, BU_GRADM, k, g.L, g.lstride, c, hs * dv);
      budget_add(be, BE_GRADM, k, g.L, g.lstride, c, hs * dv * vn);
    }
  }
}

__global__ void residual_field_kernel(const Grid2 g, const double* __restrict__ pi, const double* __restrict__ rhs,
                                      const Operator op, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  size_t c = (size_t)j * g.pitch + i;
  double Ow = op.Ow[(size_t)j * op.opitch + i], Oe = op.Ow[(size_t)j * op.opitch + i + 1];
  double Os = op.Os[(size_t)j * op.opitch + i], On = op.Os[(size_t)(j + 1) * op.opitch + i];
  double pc = pi[c];
  double Lp = Oe * (ld_s(pi, g, i + 1, j) - pc) + Ow * (ld_s(pi, g, i - 1, j) - pc)
            + On * (ld_s(pi, g, i, j + 1) - pc) + Os * (ld_s(pi, g, i, j - 1) - pc);
  out[c] = rhs[c] - Lp;
}

// running averages (diagnostics.c:307-375), one thread per owned cell and all layers; the
// column's eta and Montgomery potential as work.c:1173-1203 and 1410-1512 form them. The
// sums of a layer are all read before any is written (restrict-qualified, so the loads of
// the ten sums are in flight together).
__global__ void accumulate_averages_kernel(const Grid2 g, const AvgParams a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  const size_t c = (size_t)j * g.pitch + i;
  const int L = g.L;
  double* __restrict__ au = a.au;
  double* __restrict__ av = a.av;
  double* __restrict__ ah = a.ah;
  double* __restrict__ aM = a.aM;
  double* __restrict__ aW = a.aW;
  double* __restrict__ ahu = a.ahu;
  double* __restrict__ ahv = a.ahv;
  double* __restrict__ ahuu = a.ahuu;
  double* __restrict__ ahvv = a.ahvv;
  double* __restrict__ ahuv = a.ahuv;
  const double* __restrict__ wdia = a.wdia;
  double hk[AVG_LMAX], eta[AVG_LMAX];
  double e_acc = a.hhb[c];
#pragma unroll
  for (int k = AVG_LMAX - 1; k >= 0; --k) {
    if (k < L) {
      hk[k] = a.h[k * g.lstride + c];
      e_acc = e_acc + hk[k];
      eta[k] = e_acc;
    }
  }
  const double d = a.dtfac;
  const double pic = a.pi[c];
  double pp = 0;
#pragma unroll
  for (int k = 0; k < AVG_LMAX; ++k) {
    if (k < L) {
      const size_t o = k * g.lstride + c;
      const double su = au[o], sv = av[o], sh = ah[o], sM = aM[o], sW = aW[o], shu = ahu[o], shv = ahv[o],
                   shuu = ahuu[o], shvv = ahvv[o], shuv = ahuv[o], wd = wdia[o];
      if (k == 0) pp = a.use_rl ? 0 : a.gg[0] * eta[0];
      else pp = pp + a.gg[k] * eta[k];
      if (a.use_buoy) {
        if (k == 0) {
          if (!a.use_rl) pp -= a.b[c] * eta[0];
        } else {
          pp += eta[k] * (a.b[(k - 1) * g.lstride + c] - a.b[k * g.lstride + c]);
        }
      }
      double mm = pp;
      if (a.h0 != 0) {
        const double h0 = a.h0, hc = hk[k];
        mm -= a.geff[k] * (h0 * h0 * h0 * h0) / (hc * hc * hc) / 3;
      }
      const double* uk = a.u + k * g.lstride;
      const double* vk = a.v + k * g.lstride;
      const double* hkp = a.h + k * g.lstride;
      const double uc = uk[c], vc = vk[c], hc = hk[k];
      const double hw = hw_face(g, hkp, uk, i, j), hs = hs_face(g, hkp, vk, i, j);
      const double hq = 0.25 * (hc + ld_s(hkp, g, i - 1, j) + ld_s(hkp, g, i, j - 1) + ld_s(hkp, g, i - 1, j - 1));
      const double uq = 0.5 * (uc + ld_u(g, uk, i, j - 1));
      const double vq = 0.5 * (vc + ld_v(g, vk, i - 1, j));
      au[o] = su + d * uc;
      av[o] = sv + d * vc;
      ah[o] = sh + d * hc;
      aM[o] = sM + d * (mm + (a.use_rl ? pic : 0));
      aW[o] = sW + d * wd;
      ahu[o] = shu + d * hw * uc;
      ahv[o] = shv + d * hs * vc;
      ahuu[o] = shuu + d * hw * uc * uc;
      ahvv[o] = shvv + d * hs * vc * vc;
      ahuv[o] = shuv + d * hq * uq * vq;
      if (a.ab) a.ab[o] += d * a.b[o];
    }
  }
  const size_t oL = (size_t)L * g.lstride + c;
  aW[oL] += d * wdia[oL];
  a.api[c] += d * pic;
}

__global__ void scale_kernel(double* f, size_t n, double factor) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    f[q] *= factor;
}

// ------------------------------------------------ energy and enstrophy diagnostics

constexpr int EZ_BX = 32, EZ_BY = 8;

// The energy terms of one cell of layer k (diagnostics.c:514-646): the kinetic energy KE, the
// two potential-energy increments PE1, PE2 and the enstrophy increment Z (-0.0, the identity
// of addition, where h_q is zero and the reference adds nothing).
struct EzCell {
  double ke, pe1, pe2, z;
};

// HK: the HK83 kinetic energy; PLAIN: the whole block is at least one cell inside the grid,
// so every neighbour is an owned cell and loads need no boundary map
template <bool HK, bool PLAIN>
__device__ inline EzCell ez_cell(const Grid2& g, const EzParams& e, int k, int i, int j, double eta,
                                 double gtot) {
  const double* __restrict__ h = e.h + k * g.lstride;
  const double* __restrict__ u = e.u + k * g.lstride;
  const double* __restrict__ v = e.v + k * g.lstride;
  const bool inner = PLAIN || (i >= 1 && i + 1 < g.Nx && j >= 1 && j + 1 < g.Ny);
  const size_t c = (size_t)j * g.pitch + i;
  auto H = [&](int di, int dj) {
    return inner ? h[c + (ptrdiff_t)dj * g.pitch + di] : ld_s(h, g, i + di, j + dj);
  };
  auto U = [&](int di, int dj) {
    return inner ? u[c + (ptrdiff_t)dj * g.pitch + di] : ld_u(g, u, i + di, j + dj);
  };
  auto V = [&](int di, int dj) {
    return inner ? v[c + (ptrdiff_t)dj * g.pitch + di] : ld_v(g, v, i + di, j + dj);
  };
  const double dx = g.dx, dy = g.dy;
  const double hc = h[c];
  EzCell r;
  double hq, zeta;
  if (!PLAIN && g.wall_ns && j == 0) {
    hq = 0.5 * (H(-1, 0) + hc);
    zeta = 0;
  } else if (!PLAIN && g.wall_ew && i == 0) {
    hq = 0.5 * (H(0, -1) + hc);
    zeta = 0;
  } else {
    hq = 0.25 * (hc + H(-1, -1) + H(-1, 0) + H(0, -1));
    zeta = div_rn(U(0, -1) - U(0, 0), dy, g.rdy) + div_rn(V(0, 0) - V(-1, 0), dx, g.rdx);
  }
  r.z = -0.0;
  if (hq != 0) {
    const double pv = (2 * e.omz[(size_t)j * e.qpitch + i] + zeta) / hq;
    r.z = dx * dy * 0.5 * hq * (pv * pv);
  }
  double ked;
  if (HK) {
    // HK83 (diagnostics.c:577-642)
    const double he = hc + H(1, 0), hwst = H(-1, 0) + hc, hn = hc + H(0, 1), hs = H(0, -1) + hc;
    const double ue = U(1, 0), uw = U(0, 0), vn = V(0, 1), vs = V(0, 0);
    ked = 0;
    if (!PLAIN && g.wall_ns && j == 0) {
      ked += he * (1.25 * (ue * ue) + 0.25 * (U(1, 1) * U(1, 1))) + hwst * (1.25 * (uw * uw) + 0.25 * (U(0, 1) * U(0, 1)));
    } else if (!PLAIN && g.wall_ns && j == g.Ny - 1) {
      ked += he * (1.25 * (ue * ue) + 0.25 * (U(1, -1) * U(1, -1))) + hwst * (1.25 * (uw * uw) + 0.25 * (U(0, -1) * U(0, -1)));
    } else {
      const double a = U(1, 1), b = U(1, -1), cc = U(0, 1), d = U(0, -1);
      ked += he * (ue * ue + 0.25 * (a * a) + 0.25 * (b * b)) + hwst * (uw * uw + 0.25 * (cc * cc) + 0.25 * (d * d));
    }
    if (!PLAIN && g.wall_ew && i == 0) {
      ked += hn * (1.25 * (vn * vn) + 0.25 * (V(1, 1) * V(1, 1))) + hs * (1.25 * (vs * vs) + 0.25 * (V(1, 0) * V(1, 0)));
    } else if (!PLAIN && g.wall_ew && i == g.Nx - 1) {
      ked += hn * (1.25 * (vn * vn) + 0.25 * (V(-1, 1) * V(-1, 1))) + hs * (1.25 * (vs * vs) + 0.25 * (V(-1, 0) * V(-1, 0)));
    } else {
      const double a = V(1, 1), b = V(-1, 1), cc = V(1, 0), d = V(-1, 0);
      ked += hn * (vn * vn + 0.25 * (a * a) + 0.25 * (b * b)) + hs * (vs * vs + 0.25 * (cc * cc) + 0.25 * (d * d));
    }
    ked *= dx * dy / 12.0;
  } else {
    // AL81, UP3, KT00 (diagnostics.c:562-575)
    const double ue = U(1, 0), uw = U(0, 0), vn = V(0, 1), vs = V(0, 0);
    ked = 0.125 * dx * dy
        * ((hc + H(1, 0)) * (ue * ue) + (H(-1, 0) + hc) * (uw * uw) + (hc + H(0, 1)) * (vn * vn)
           + (H(0, -1) + hc) * (vs * vs));
  }
  r.ke = ked;
  r.pe1 = dx * dy * gtot * hc * (eta - 0.5 * hc);
  const double h0 = e.h0;
  constexpr double kSixth = 1.0 / 6.0;   // rounded to nearest at compile time
  r.pe2 = div_rn(dx * dy * gtot * (h0 * h0 * h0 * h0) / (hc * hc), 6.0, kSixth);
  return r;
}

// geff[k] for a runtime k without a local copy of the parameter array
__device__ inline double ez_geff(const EzParams& e, int k) {
  double x = 0;
#pragma unroll
  for (int q = 0; q < AVG_LMAX; ++q)
    if (q == k) x = e.geff[q];
  return x;
}

// g_tot of layer k at one cell
__device__ inline double ez_gtot(const Grid2& g, const EzParams& e, int k, size_t c) {
  const double gt = ez_geff(e, k);
  return e.b ? gt - e.b[k * g.lstride + c] : gt;
}

__device__ inline EzCell ez_cell_any(const Grid2& g, const EzParams& e, int k, int i, int j, double eta) {
  const double gt = ez_gtot(g, e, k, (size_t)j * g.pitch + i);
  return g.thick_scheme == 1 ? ez_cell<true, false>(g, e, k, i, j, eta, gt)
                             : ez_cell<false, false>(g, e, k, i, j, eta, gt);
}

// per-cell terms in four planes of L*lstride: KE, PE1, PE2, Z
__global__ void ez_terms_kernel(const Grid2 g, const EzParams e, double* __restrict__ terms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.Nx || j >= g.Ny) return;
  const size_t c = (size_t)j * g.pitch + i;
  const size_t P = (size_t)g.L * g.lstride;
  double eta = e.hhb[c];
  for (int k = g.L - 1; k >= 0; --k) {
    eta = eta + e.hw[k * g.lstride + c];
    const EzCell r = ez_cell_any(g, e, k, i, j, eta);
    const size_t o = k * g.lstride + c;
    terms[o] = r.ke;
    terms[P + o] = r.pe1;
    terms[2 * P + o] = r.pe2;
    terms[3 * P + o] = r.z;
  }
}

// the reference's order: layer outer, then x, then y; KE, PE (two increments per cell) and
// Z_k are independent chains. One thread; loads are batched ahead of the additions.
__global__ void ez_serial_kernel(const Grid2 g, const double* __restrict__ terms, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const size_t P = (size_t)g.L * g.lstride;
  double ke = 0, pe = 0;
  for (int k = 0; k < g.L; ++k) {
    double z = 0;
    for (int i = 0; i < g.Nx; ++i) {
      const double* t = terms + k * g.lstride + i;
      int j = 0;
      for (; j + 4 <= g.Ny; j += 4) {
        double a[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int p = 0; p < 4; ++p) a[p][q] = t[p * P + (size_t)(j + q) * g.pitch];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ke += a[0][q];
          pe += a[1][q];
          pe += a[2][q];
          z += a[3][q];
        }
      }
      for (; j < g.Ny; ++j) {
        const size_t o = (size_t)j * g.pitch;
        ke += t[o];
        pe += t[P + o];
        pe += t[2 * P + o];
        z += t[3 * P + o];
      }
    }
    out[2 + k] = z;
  }
  out[0] = ke;
  out[1] = pe;
}

// sum of one value over the block (32x8 threads) in a fixed order, valid in thread 0
__device__ inline double ez_block_sum(double x, double* ws) {
  const int t = threadIdx.y * EZ_BX + threadIdx.x;
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if ((t & 31) == 0) ws[t >> 5] = x;
  __syncthreads();
  double s = 0;
  if (t == 0)
    for (int w = 0; w < EZ_BX * EZ_BY / 32; ++w) s += ws[w];
  __syncthreads();
  return s;
}

// fixed tree: one thread per column of one 32x8 tile walks the layers bottom-up; the block
// sums each layer's enstrophy, then KE and PE, into partials[q * blocks + block]
template <bool HK>
__global__ void __launch_bounds__(EZ_BX * EZ_BY, HK ? 2 : 4) ez_partial_kernel(const Grid2 g, const EzParams e,
                                                                   double* __restrict__ partials) {
  __shared__ double ws[EZ_BX * EZ_BY / 32];
  const int i = blockIdx.x * EZ_BX + threadIdx.x;
  const int j = blockIdx.y * EZ_BY + threadIdx.y;
  const bool in = i < g.Nx && j < g.Ny;
  const bool plain = blockIdx.x * EZ_BX >= 1 && (blockIdx.x + 1) * EZ_BX + 1 <= g.Nx &&
                     blockIdx.y * EZ_BY >= 1 && (blockIdx.y + 1) * EZ_BY + 1 <= g.Ny;
  const int L = g.L;
  const size_t c = in ? (size_t)j * g.pitch + i : 0;
  const size_t nb = (size_t)gridDim.x * gridDim.y;
  double* out = partials + (blockIdx.y * gridDim.x + blockIdx.x);
  double ke = 0, pe = 0;
  double eta = in ? e.hhb[c] : 0;
#pragma unroll 1
  for (int k = L - 1; k >= 0; --k) {
    double z = 0;
    if (in) {
      eta = eta + e.hw[k * g.lstride + c];
      const double gt = ez_gtot(g, e, k, c);
      const EzCell r = plain ? ez_cell<HK, true>(g, e, k, i, j, eta, gt) : ez_cell<HK, false>(g, e, k, i, j, eta, gt);
      ke += r.ke;
      pe += r.pe1;
      pe += r.pe2;
      z = r.z;
    }
    z = ez_block_sum(z, ws);
    if (threadIdx.x == 0 && threadIdx.y == 0) out[(2 + k) * nb] = z;
  }
  ke = ez_block_sum(ke, ws);
  pe = ez_block_sum(pe, ws);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    out[0] = ke;
    out[nb] = pe;
  }
}

// one block per quantity q: the partials of all blocks in a fixed order
__global__ void ez_final_kernel(const double* __restrict__ partials, int nblocks, double* out) {
  __shared__ double ws[RED_BLOCK / 32];
  const int q = blockIdx.x;
  double s = 0;
  for (int b = threadIdx.x; b < nblocks; b += RED_BLOCK) s += partials[(size_t)q * nblocks + b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_BLOCK / 32; ++w) t += ws[w];
    out[q] = t;
  }
}

inline dim3 grid2(int Nx, int Ny, dim3 b) { return dim3((Nx + b.x - 1) / b.x, (Ny + b.y - 1) / b.y); }

// ---------------------------------------------------------------- corner shadow capture
// A fill of the work arrays in the reference (pawsim_work_load_state, work.c:538-559) leaves
// in the wall rows next to the periodic seam the values that the next fill copies into the
// corner ghosts: the state it copied. This kernel records them (u, v, h, and b when given).
__global__ void corner_capture_kernel(const Grid2 g, const double* __restrict__ u, const double* __restrict__ v,
                                      const double* __restrict__ h, const double* __restrict__ b,
                                      double* __restrict__ next) {
  const int L = g.L;
  const int per_layer = 2 * CORNER_R * CORNER_C;
  const int total = CORNER_F * L * per_layer;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int f = t / (L * per_layer);
    const int k = (t / per_layer) % L;
    const int side = (t / (CORNER_R * CORNER_C)) % 2;
    const int r = (t / CORNER_C) % CORNER_R;
    const int c = t % CORNER_C;
    const int x = corner_x(c, g.Nx), y = corner_y(side, r, g.Ny);
    const size_t o = (size_t)k * g.lstride + (size_t)y * g.pitch + x;
    double val = 0;
    if (f == CF_U) val = u[o];
    else if (f == CF_V) val = v[o];
    else if (f == CF_H) val = h[o];
    else val = b ? b[o] : 0.0;
    next[corner_slot(f, k, L, side, r, c)] = val;
  }
}

}  // namespace

void launch_corner_capture(const Grid2& g, const double* u, const double* v, const double* h, const double* b,
                           double* next, cudaStream_t s) {
  corner_capture_kernel<<<1, 256, 0, s>>>(g, u, v, h, b, next);
}

void launch_accumulate_averages(const Grid2& g, const AvgParams& a, cudaStream_t s) {
  dim3 b(32, 8);
  accumulate_averages_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, a);
}

void launch_scale(double* f, size_t n, double factor, cudaStream_t s) {
  scale_kernel<<<1184, 256, 0, s>>>(f, n, factor);
}

static dim3 ez_tree_grid(const Grid2& g) {
  return dim3((g.Nx + EZ_BX - 1) / EZ_BX, (g.Ny + EZ_BY - 1) / EZ_BY);
}

size_t ez_scratch_elems(const Grid2& g, bool serial) {
  if (serial) return 4 * (size_t)g.L * g.lstride;
  const dim3 gr = ez_tree_grid(g);
  return (size_t)(g.L + 2) * gr.x * gr.y;
}

int launch_energy(const Grid2& g, const EzParams& e, bool serial, double* terms, double* out, cudaStream_t s) {
  if (serial) {
    dim3 b(32, 8);
    ez_terms_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, e, terms);
    ez_serial_kernel<<<1, 32, 0, s>>>(g, terms, out);
    return 2;
  }
  const dim3 gr = ez_tree_grid(g);
  if (g.thick_scheme == 1)
    ez_partial_kernel<true><<<gr, dim3(EZ_BX, EZ_BY), 0, s>>>(g, e, terms);
  else
    ez_partial_kernel<false><<<gr, dim3(EZ_BX, EZ_BY), 0, s>>>(g, e, terms);
  ez_final_kernel<<<g.L + 2, RED_BLOCK, 0, s>>>(terms, gr.x * gr.y, out);
  return 2;
}

// interior cells with plain loads when the face thickness is the AL81 average, then the
// border ring through the boundary maps; otherwise every cell through the maps
static int launch_rhs(const Grid2& g, const double* u, const double* v, const double* h, double* out,
                      int with_dt, cudaStream_t s) {
  dim3 b(32, 8);
  if (g.thick_scheme == 0 && g.Nx >= 3 && g.Ny >= 3) {
    rhs_inner_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, u, v, h, out, with_dt);
    const int ring = 2 * g.Nx + 2 * (g.Ny - 2);
    rhs_kernel<<<(ring + 127) / 128, 128, 0, s>>>(g, u, v, h, out, with_dt, 1);
    return 2;
  }
  rhs_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, u, v, h, out, with_dt, 0);
  return 1;
}

int launch_pressure_rhs(const Grid2& g, const double* u, const double* v, const double* h, double* rhs,
                        cudaStream_t s) {
  return launch_rhs(g, u, v, h, rhs, 1, s);
}

int launch_divergence_field(const Grid2& g, const double* u, const double* v, const double* h, double* out,
                            cudaStream_t s) {
  return launch_rhs(g, u, v, h, out, 0, s);
}

size_t reduce_scratch_elems(int Nx, int Ny) { (void)Nx; return (size_t)(Ny + RED_ROWS - 1) / RED_ROWS + 4; }

void launch_sum(const double* f, int Nx, int Ny, int pitch, bool serial, double* partials, double* out,
                cudaStream_t s) {
  if (serial) {
    serial_sum_kernel<<<1, SS_THREADS, 0, s>>>(f, Nx, Ny, pitch, out, 0);
    return;
  }
  int nb = (Ny + RED_ROWS - 1) / RED_ROWS;
  tree_partial_kernel<<<nb, RED_BLOCK, 0, s>>>(f, Nx, Ny, pitch, partials, 0);
  tree_final_kernel<<<1, RED_BLOCK, 0, s>>>(partials, nb, out);
}

void launch_subtract_mean(double* f, int Nx, int Ny, int pitch, const double* sum, cudaStream_t s) {
  dim3 b(32, 8);
  subtract_mean_kernel<<<grid2(Nx, Ny, b), b, 0, s>>>(f, Nx, Ny, pitch, sum);
}

void launch_norms(const double* f, int Nx, int Ny, int pitch, bool serial, double* partials, double* out,
                  cudaStream_t s) {
  // out[0] = max |f| (via an integer max on the bit pattern, in out[2] as scratch), out[1] = sum f^2
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(out + 2);
  cudaMemsetAsync(bits, 0, sizeof(unsigned long long), s);
  max_abs_kernel<<<dim3(1, Ny < 1184 ? Ny : 1184), 256, 0, s>>>(f, Nx, Ny, pitch, bits);
  store_max_kernel<<<1, 1, 0, s>>>(bits, out);
  if (serial) {
    serial_sum_kernel<<<1, SS_THREADS, 0, s>>>(f, Nx, Ny, pitch, out + 1, 1);
  } else {
    int nb = (Ny + RED_ROWS - 1) / RED_ROWS;
    tree_partial_kernel<<<nb, RED_BLOCK, 0, s>>>(f, Nx, Ny, pitch, partials, 1);
    tree_final_kernel<<<1, RED_BLOCK, 0, s>>>(partials, nb, out + 1);
  }
}

void launch_operator(const Grid2& g, const double* Hc, const Operator& op, double sor_rp, cudaStream_t s) {
  dim3 b(32, 8);
  operator_kernel<<<grid2(g.Nx + 1, g.Ny + 1, b), b, 0, s>>>(g, Hc, op, sor_rp);
  sor_factor_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, op, sor_rp);
}

int launch_sor(const Grid2& g, double* pi, const double* rhs, const Operator& op, double sor_rp, double tol,
               int maxiters, unsigned long long* slots, int* iters, cudaStream_t s) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 512;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sor_kernel, threads, 0);
  int want = g.Ny;   // one block per row at most
  int cap = nsm * (per_sm < 1 ? 1 : per_sm);
  int blocks = want < cap ? want : cap;
  if (blocks < 1) blocks = 1;
  Grid2 gg = g;
  Operator oo = op;
  double* ppi = pi;
  const double* prhs = rhs;
  void* args[] = {&gg, &ppi, &prhs, &oo, &sor_rp, &tol, &maxiters, &slots, &iters};
  cudaError_t e = cudaLaunchCooperativeKernel((void*)sor_kernel, dim3(blocks), dim3(threads), args, 0, s);
  return e == cudaSuccess ? 0 : -1;
}

void launch_projection(const Grid2& g, const double* pi, double* u, double* v, cudaStream_t s) {
  dim3 b(32, 8);
  projection_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, pi, u, v);
}

void launch_projection_budget(const Grid2& g, const double* pi, double* u, double* v, const double* h, double* bu,
                              double* bv, double* be, cudaStream_t s) {
  dim3 b(32, 8);
  projection_budget_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, pi, u, v, h, bu, bv, be);
}

void launch_residual_field(const Grid2& g, const double* pi, const double* rhs, const Operator& op, double* out,
                           cudaStream_t s) {
  dim3 b(32, 8);
  residual_field_kernel<<<grid2(g.Nx, g.Ny, b), b, 0, s>>>(g, pi, rhs, op, out);
}

}  // namespace pawsim
