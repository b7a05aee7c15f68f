// mg.cu -- GPU multigrid for the rigid-lid pressure equation (see mg.cuh).
//
// Per level above the coarse block, one fused "down" kernel (red-black pre-smoothing,
// residual and 2x2 restriction on a shared-memory tile with a 2*nu+1 halo) and one fused
// "up" kernel (bilinear prolongation of the coarse correction, correction and red-black
// post-smoothing on a tile with a 2*nu halo). Cells of the halo are smoothed redundantly by
// neighbouring tiles from the same inputs, so every tile sees the values a global sweep
// would produce. Levels of at most 1024 cells run inside one CTA in shared memory. The whole
// V-cycle plus the stopping test is a CUDA graph whose body sits in a device-side `while`
// conditional node: no host round trip per V-cycle.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "common.cuh"
#include "mg.cuh"

namespace pawsim {

namespace {

inline int coarsen(int n) { return n > 1 ? (n + 1) / 2 : 1; }

template <typename T>
struct LV {
  int Nx, Ny, pitch;
  const T *Ow, *Os, *Osum, *rOsum;
  T *e, *rhs, *res;
  T* tmp;   // output of the fused down kernel, input of the fused up kernel
};

template <typename T>
LV<T> view(const Multigrid::Level& l);
template <>
LV<double> view<double>(const Multigrid::Level& l) {
  return LV<double>{l.Nx, l.Ny, l.pitch, l.Ow, l.Os, l.Osum, l.rOsum, l.e, l.rhs, l.res, l.tmp};
}
template <>
LV<float> view<float>(const Multigrid::Level& l) {
  return LV<float>{l.Nx, l.Ny, l.pitch, l.Ow32, l.Os32, l.Osum32, l.rOsum32, l.e32, l.rhs32, l.res32, l.tmp32};
}

#define IX(l, i, j) ((size_t)(j) * (l).pitch + (i))

__host__ __device__ inline int wrapi(int i, int n) { return wrap_index(i, n); }

// ---------------------------------------------------------------- generic kernels
// (levels whose transfer is not an exact 2:1 coarsening, and the fine-level checks)

// operator sum around a cell with the multigrid's periodic indexing (multigrid.c:604-623)
template <typename T>
__device__ inline T neighbour_sum(const LV<T>& l, const T* e, int i, int j) {
  int ip1 = i + 1 == l.Nx ? 0 : i + 1, im1 = i == 0 ? l.Nx - 1 : i - 1;
  int jp1 = j + 1 == l.Ny ? 0 : j + 1, jm1 = j == 0 ? l.Ny - 1 : j - 1;
  return l.Os[IX(l, i, jp1)] * e[IX(l, i, jp1)] + l.Os[IX(l, i, j)] * e[IX(l, i, jm1)]
       + l.Ow[IX(l, ip1, j)] * e[IX(l, ip1, j)] + l.Ow[IX(l, i, j)] * e[IX(l, im1, j)];
}

template <typename T>
__global__ void smooth_kernel(LV<T> l, int color, T omega) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny || ((i + j) & 1) != color) return;
  size_t c = IX(l, i, j);
  T s = neighbour_sum(l, l.e, i, j);
  l.e[c] = omega * l.rOsum[c] * (s - l.rhs[c]) + (T(1) - omega) * l.e[c];
}

template <typename T>
__global__ void residual_kernel(LV<T> l) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny) return;
  size_t c = IX(l, i, j);
  l.res[c] = neighbour_sum(l, l.e, i, j) - l.Osum[c] * l.e[c] - l.rhs[c];
}

// area-weighted restriction for uneven pairs (multigrid.c:681-740)
template <typename T>
__device__ inline T restrict_general_at(int fNx, int fNy, int cNx, int cNy, int ic, int jc,
                                        const T* src, int spitch) {
  double x0 = (double)ic * fNx / cNx, x1 = (double)(ic + 1) * fNx / cNx;
  double y0 = (double)jc * fNy / cNy, y1 = (double)(jc + 1) * fNy / cNy;
  double acc = 0, wsum = 0;
  for (int fi = (int)floor(x0); fi < (int)ceil(x1); ++fi) {
    double wx = fmin(x1, (double)(fi + 1)) - fmax(x0, (double)fi);
    if (wx <= 0) continue;
    for (int fj = (int)floor(y0); fj < (int)ceil(y1); ++fj) {
      double wy = fmin(y1, (double)(fj + 1)) - fmax(y0, (double)fj);
      if (wy <= 0) continue;
      double w = wx * wy;
      acc += w * (double)src[(size_t)fj * spitch + fi];
      wsum += w;
    }
  }
  return (T)(wsum > 0 ? acc / wsum : acc);
}

template <typename T>
__global__ void restrict_general_kernel(LV<T> f, LV<T> c) {
  int ic = blockIdx.x * blockDim.x + threadIdx.x;
  int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (ic >= c.Nx || jc >= c.Ny) return;
  c.rhs[IX(c, ic, jc)] = restrict_general_at<T>(f.Nx, f.Ny, c.Nx, c.Ny, ic, jc, f.res, f.pitch);
  c.e[IX(c, ic, jc)] = T(0);
}

// bilinear prolongation weights of fine cell (i, j) of an exact 2:1 transfer, including
// the wall and corner overrides (multigrid.c:376-442): m/p = coarse point west/east (first
// letter) and south/north (second letter) of the cell
template <typename T>
__device__ inline void prolong_weights(int i, int j, int fNx, int fNy, bool wew, bool wns, T& wmm, T& wpm, T& wmp,
                                       T& wpp) {
  const bool io = (i & 1) != 0, jo = (j & 1) != 0;
  T ai = io ? T(0.75) : T(0.25), bi = io ? T(0.25) : T(0.75);
  T aj = jo ? T(0.75) : T(0.25), bj = jo ? T(0.25) : T(0.75);
  wmm = ai * aj;
  wmp = ai * bj;
  wpm = bi * aj;
  wpp = bi * bj;
  if (wns) {
    if (j == 0) { wmm = 0; wpm = 0; wmp = ai; wpp = bi; }
    if (j == fNy - 1) { wmp = 0; wpp = 0; wmm = ai; wpm = bi; }
  }
  if (wew) {
    if (i == 0) { wmm = 0; wmp = 0; wpm = aj; wpp = bj; }
    if (i == fNx - 1) { wpm = 0; wpp = 0; wmm = aj; wmp = bj; }
  }
  if (wns && wew) {
    if (i == 0 && j == 0) { wmm = 0; wmp = 0; wpm = 0; wpp = 1; }
    if (i == 0 && j == fNy - 1) { wmm = 0; wmp = 0; wpm = 1; wpp = 0; }
    if (i == fNx - 1 && j == 0) { wmm = 0; wmp = 1; wpm = 0; wpp = 0; }
    if (i == fNx - 1 && j == fNy - 1) { wmm = 1; wmp = 0; wpm = 0; wpp = 0; }
  }
}

// bilinear prolongation weights and coarse indices of one fine cell (multigrid.c:376-442,
// 827-932); returns the interpolated coarse correction
template <typename T, typename Get>
__device__ inline T prolong_at(int i, int j, int fNx, int fNy, int cNx, int cNy, bool power2, bool wew,
                               bool wns, Get ec) {
  if (power2) {
    // coarse points east/west and north/south of fine point (i, j), i, j >= 0
    int hx = fNx / 2, hy = fNy / 2;
    int ip = (i + 1) >> 1, jp = (j + 1) >> 1;
    if (ip >= hx) ip -= hx;
    if (jp >= hy) jp -= hy;
    int im = ip == 0 ? hx - 1 : ip - 1, jm = jp == 0 ? hy - 1 : jp - 1;
    T wmm, wpm, wmp, wpp;
    prolong_weights<T>(i, j, fNx, fNy, wew, wns, wmm, wpm, wmp, wpp);
    return wmm * ec(im, jm) + wpm * ec(ip, jm) + wmp * ec(im, jp) + wpp * ec(ip, jp);
  }
  double x = ((double)i + 0.5) * cNx / fNx - 0.5, y = ((double)j + 0.5) * cNy / fNy - 0.5, tx, ty;
  int imr, jmr;
  if (wew && x <= 0) { imr = 0; tx = 0; }
  else if (wew && x >= cNx - 1) { imr = cNx - 1; tx = 0; }
  else { imr = (int)floor(x); tx = x - imr; }
  if (wns && y <= 0) { jmr = 0; ty = 0; }
  else if (wns && y >= cNy - 1) { jmr = cNy - 1; ty = 0; }
  else { jmr = (int)floor(y); ty = y - jmr; }
  auto idx = [](int v, int n, bool wall) {
    if (n <= 1) return 0;
    if (wall) return v < 0 ? 0 : (v >= n ? n - 1 : v);
    return ((v % n) + n) % n;
  };
  int im = idx(imr, cNx, wew), ip = idx(imr + 1, cNx, wew);
  int jm = idx(jmr, cNy, wns), jp = idx(jmr + 1, cNy, wns);
  return (T)((1 - tx) * (1 - ty) * (double)ec(im, jm) + tx * (1 - ty) * (double)ec(ip, jm)
             + (1 - tx) * ty * (double)ec(im, jp) + tx * ty * (double)ec(ip, jp));
}

template <typename T>
__global__ void prolong_correct_kernel(LV<T> f, LV<T> c, int power2, int wew, int wns) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= f.Nx || j >= f.Ny) return;
  auto ec = [&](int a, int b) { return c.e[IX(c, a, b)]; };
  f.e[IX(f, i, j)] -= prolong_at<T>(i, j, f.Nx, f.Ny, c.Nx, c.Ny, power2, wew, wns, ec);
}

// use_fullMG: restriction of a level's right-hand side to the next coarser level
// (restrict_MG of multigrid.c:1248-1254; 2x2 mean or area-weighted)
__global__ void restrict_rhs_kernel(LV<double> f, LV<double> c, int power2) {
  int ic = blockIdx.x * blockDim.x + threadIdx.x;
  int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (ic >= c.Nx || jc >= c.Ny) return;
  double v;
  if (power2) {
    const double* r = f.rhs + IX(f, 2 * ic, 2 * jc);
    v = 0.25 * (r[0] + r[1] + r[f.pitch] + r[f.pitch + 1]);
  } else {
    v = restrict_general_at<double>(f.Nx, f.Ny, c.Nx, c.Ny, ic, jc, f.rhs, f.pitch);
  }
  c.rhs[IX(c, ic, jc)] = v;
}

// use_fullMG: the coarser solution interpolated onto this level, replacing its values
// (interpolate_MG into the level's pi, multigrid.c:1259-1265)
__global__ void prolong_set_kernel(LV<double> f, LV<double> c, int power2, int wew, int wns) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= f.Nx || j >= f.Ny) return;
  auto ec = [&](int a, int b) { return c.e[IX(c, a, b)]; };
  f.e[IX(f, i, j)] = prolong_at<double>(i, j, f.Nx, f.Ny, c.Nx, c.Ny, power2, wew, wns, ec);
}

// ---------------------------------------------------------------- fused tile kernels

// max over the block (warp shuffles, then the warps' maxima), one atomic per block
__device__ inline void block_max_to(double m, unsigned long long* bits) {
  __shared__ double wm[32];
  const int t = threadIdx.x + threadIdx.y * blockDim.x;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) wm[t >> 5] = m;
  __syncthreads();
  if (t == 0) {
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    double b = 0;
    for (int w = 0; w < nw; ++w) b = fmax(b, wm[w]);
    if (b > 0) atomicMax(bits, (unsigned long long)__double_as_longlong(b));
  }
}

// A CTA owns OX x OY cells at (X0, Y0) and keeps a shared-memory tile of e, rhs, 1/Osum,
// Ow and Os over [X0-H, X0+OX+H) x [Y0-H, Y0+OY+H). In shared memory each array is split
// into two planes by the parity of the tile column, so the cells of one colour along a
// row are contiguous: a red-black half sweep gives each thread one cell of a (red, black)
// pair and every shared access of a warp is stride 1. A half sweep at reach R updates the
// cells of one colour within R of the owned block; R shrinks by one per half sweep, so
// after the sweeps the owned cells (and, with one spare halo row, their neighbours) hold
// what a global sweep would give. Tiles read their halo from the kernel's input array and
// write their owned cells to a different output array, so no tile can see a neighbour's
// result. The tile arrives by cp.async, straight from global to shared memory.
__host__ __device__ constexpr int plane_pad(int n, int bytes) {
  // the second plane starts half a 128-byte bank row after the first, so a half warp
  // touching 8 cells of each plane (FP64) or a warp touching 16 of each (FP32) hits
  // disjoint banks
  while ((n * bytes) % 128 != 64) ++n;
  return n;
}

template <typename T, int OX, int OY, int H>
struct PT {
  static constexpr int W = OX + 2 * H, Hh = OY + 2 * H, N = W * Hh;
  static constexpr int PW = (W + 1) / 2, PL = plane_pad(PW * Hh, (int)sizeof(T)), ARR = 2 * PL;
  // coarse cells read by the bilinear prolongation of the tile (fine H <= 3)
  static constexpr int CW = OX / 2 + 4, CH = OY / 2 + 4, NC = CW * CH;
  static constexpr int BUF = 5 * ARR + NC;   // elements of one tile buffer
  __device__ static int at(int lx, int ly) { return (lx & 1) * PL + ly * PW + (lx >> 1); }
  // east and west neighbours of the cell at index q in column parity s
  __device__ static int east(int q, int s) { return q + (s ? 1 - PL : PL); }
  __device__ static int west(int q, int s) { return q + (s ? -PL : PL - 1); }
};

template <typename T, int OX, int OY, int H>
constexpr size_t tile_bytes() {
  return (size_t)PT<T, OX, OY, H>::BUF * sizeof(T);
}

// interior tiles: halo, the prolongation's coarse cells and the wall-special cells all lie
// inside the level, so loads need no wrap and the prolongation weights no wall cases
template <int OX, int OY, int H>
__device__ inline bool tile_inner(int X0, int Y0, int Nx, int Ny) {
  constexpr int M = H + 1 > 4 ? H + 1 : 4;
  return X0 >= M && X0 + OX + M <= Nx && Y0 >= M && Y0 + OY + M <= Ny;
}

template <typename T>
__device__ inline void cp_async(T* dst, const T* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T, int OX, int OY, int H>
struct TileBuf {
  T *e, *rhs, *rO, *Ow, *Os, *ce;
  __device__ explicit TileBuf(T* base) {
    using G = PT<T, OX, OY, H>;
    e = base;
    rhs = e + G::ARR;
    rO = rhs + G::ARR;
    Ow = rO + G::ARR;
    Os = Ow + G::ARR;
    ce = Os + G::ARR;
  }
};

// issue the asynchronous loads of one tile (and, for the up kernel, of its coarse cells)
template <typename T, int OX, int OY, int H, int NT>
__device__ inline void issue_tile(const LV<T>& l, const LV<T>& c, int X0, int Y0, bool zero_e, bool coarse,
                                  const TileBuf<T, OX, OY, H>& b) {
  using G = PT<T, OX, OY, H>;
  const bool inner = tile_inner<OX, OY, H>(X0, Y0, l.Nx, l.Ny);
  if (inner) {
    const int base = (Y0 - H) * l.pitch + (X0 - H);
    const T *pe = l.e + base, *pr = l.rhs + base, *po = l.rOsum + base, *pw = l.Ow + base, *ps = l.Os + base;
    for (int k = threadIdx.x; k < G::N; k += NT) {
      const int ly = k / G::W, lx = k - ly * G::W;
      const int g = ly * l.pitch + lx, s = G::at(lx, ly);
      if (zero_e) b.e[s] = T(0);
      else cp_async(b.e + s, pe + g);
      cp_async(b.rhs + s, pr + g);
      cp_async(b.rO + s, po + g);
      cp_async(b.Ow + s, pw + g);
      cp_async(b.Os + s, ps + g);
    }
    if (coarse) {
      const T* pc = c.e + ((Y0 / 2 - 2) * c.pitch + (X0 / 2 - 2));
      for (int k = threadIdx.x; k < G::NC; k += NT) {
        const int cy = k / G::CW, cx = k - cy * G::CW;
        cp_async(b.ce + k, pc + cy * c.pitch + cx);
      }
    }
  } else {
    for (int k = threadIdx.x; k < G::N; k += NT) {
      const int ly = k / G::W, lx = k - ly * G::W;
      const size_t g = IX(l, wrapi(X0 - H + lx, l.Nx), wrapi(Y0 - H + ly, l.Ny));
      const int s = G::at(lx, ly);
      if (zero_e) b.e[s] = T(0);
      else cp_async(b.e + s, l.e + g);
      cp_async(b.rhs + s, l.rhs + g);
      cp_async(b.rO + s, l.rOsum + g);
      cp_async(b.Ow + s, l.Ow + g);
      cp_async(b.Os + s, l.Os + g);
    }
  }
  cp_async_commit();
}

// one red-black half sweep at reach R; par0 = colour + X0 + Y0
template <typename T, int OX, int OY, int H, int NT, int R>
__device__ inline void half_sweep(int par0, T omega, const TileBuf<T, OX, OY, H>& b) {
  using G = PT<T, OX, OY, H>;
  constexpr int hw = (OX + 2 * R) / 2, U = hw * (OY + 2 * R);
#pragma unroll 2
  for (int k = threadIdx.x; k < U; k += NT) {
    const int row = k / hw, p = k - row * hw;
    const int a = H - R + ((par0 + row) & 1);   // tile column = a + 2p
    const int sp = a & 1;
    const int q = sp * G::PL + (H - R + row) * G::PW + p + (a >> 1);
    const int qe = G::east(q, sp), qw = G::west(q, sp);
    T s = b.Os[q + G::PW] * b.e[q + G::PW] + b.Os[q] * b.e[q - G::PW] + b.Ow[qe] * b.e[qe] + b.Ow[q] * b.e[qw];
    b.e[q] = omega * b.rO[q] * (s - b.rhs[q]) + (T(1) - omega) * b.e[q];
  }
}

// NU red-black sweeps (red first), reach H-1 down to H-2NU
template <typename T, int OX, int OY, int H, int NT, int NU, int S = 0>
__device__ inline void tile_sweeps(int xy, T omega, const TileBuf<T, OX, OY, H>& b) {
  if constexpr (S < NU) {
    half_sweep<T, OX, OY, H, NT, H - (2 * S + 1)>(xy, omega, b);
    __syncthreads();
    half_sweep<T, OX, OY, H, NT, H - (2 * S + 2)>(xy + 1, omega, b);
    __syncthreads();
    tile_sweeps<T, OX, OY, H, NT, NU, S + 1>(xy, omega, b);
  }
}

// pre-smoothing of f.e (or of zero) into `out`, residual and 2x2 restriction into the
// coarse rhs (the coarse correction starts from zero: the coarse kernels never read it)
template <typename T, int OX, int OY, int NT, int NU>
__device__ __forceinline__ void down_tile_body(const LV<T>& f, const LV<T>& c, T omega, int zero_e,
                                               T* __restrict__ out, int bx, int by) {
  constexpr int H = 2 * NU + 1;
  using G = PT<T, OX, OY, H>;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const TileBuf<T, OX, OY, H> b(reinterpret_cast<T*>(sm_raw));
  const int X0 = bx * OX, Y0 = by * OY;
  const bool inner = tile_inner<OX, OY, H>(X0, Y0, f.Nx, f.Ny);
  issue_tile<T, OX, OY, H, NT>(f, c, X0, Y0, zero_e != 0, false, b);
  cp_async_wait<0>();
  __syncthreads();
  tile_sweeps<T, OX, OY, H, NT, NU>(X0 + Y0, omega, b);
  // write the smoothed owned cells and form their residuals (multigrid.c:604-623); the
  // residuals go, split by column parity, where 1/Osum was (the residual does not read it)
  T* res = b.rO;
  constexpr int RP = plane_pad((OX / 2) * OY, (int)sizeof(T));
  for (int k = threadIdx.x; k < OX * OY; k += NT) {
    const int ly = k / OX, lx = k - ly * OX;
    const int gi = X0 + lx, gj = Y0 + ly;
    const int sp = (lx + H) & 1;
    const int q = G::at(lx + H, ly + H), qe = G::east(q, sp), qw = G::west(q, sp);
    T r = 0;
    if (inner || (gi < f.Nx && gj < f.Ny)) {
      const T ec = b.e[q];
      out[IX(f, gi, gj)] = ec;
      const T osum = b.Ow[q] + b.Ow[qe] + b.Os[q] + b.Os[q + G::PW];
      const T s = b.Os[q + G::PW] * b.e[q + G::PW] + b.Os[q] * b.e[q - G::PW] + b.Ow[qe] * b.e[qe]
                + b.Ow[q] * b.e[qw];
      r = s - osum * ec - b.rhs[q];
    }
    res[(lx & 1) * RP + ly * (OX / 2) + (lx >> 1)] = r;
  }
  __syncthreads();
  // restriction, order of restrict_power2_MG: (2i,2j) + (2i+1,2j) + (2i,2j+1) + (2i+1,2j+1)
  for (int k = threadIdx.x; k < (OX / 2) * (OY / 2); k += NT) {
    const int cy = k / (OX / 2), cx = k - cy * (OX / 2);
    const int ic = X0 / 2 + cx, jc = Y0 / 2 + cy;
    if (inner || (ic < c.Nx && jc < c.Ny)) {
      const T* r0 = res + (2 * cy) * (OX / 2) + cx;
      c.rhs[IX(c, ic, jc)] = T(0.25) * (r0[0] + r0[RP] + r0[OX / 2] + r0[RP + OX / 2]);
    }
  }
}

template <typename T, int OX, int OY, int NT, int NU>
__global__ void __launch_bounds__(NT) down_tile(LV<T> f, LV<T> c, T omega, int zero_e, T* __restrict__ out) {
  down_tile_body<T, OX, OY, NT, NU>(f, c, omega, zero_e, out, blockIdx.x, blockIdx.y);
}

// prolongation of the coarse correction c.e, correction of f.e and post-smoothing, into
// `out`. With MEASURE the tile carries one more halo row and the kernel also folds
// max |e - Jacobi(e)| over its owned cells into *bits: the stopping measure of the
// finished V-cycle (multigrid.c:1123-1156).
template <typename T, int OX, int OY, int NT, int NU, bool MEASURE>
__device__ __forceinline__ void up_tile_body(const LV<T>& f, const LV<T>& c, T omega, int wew, int wns,
                                             unsigned long long* bits, T* __restrict__ out, int bx, int by) {
  constexpr int H = 2 * NU + (MEASURE ? 1 : 0);
  using G = PT<T, OX, OY, H>;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const TileBuf<T, OX, OY, H> b(reinterpret_cast<T*>(sm_raw));
  const int X0 = bx * OX, Y0 = by * OY;
  const bool inner = tile_inner<OX, OY, H>(X0, Y0, f.Nx, f.Ny);
  issue_tile<T, OX, OY, H, NT>(f, c, X0, Y0, false, true, b);
  cp_async_wait<0>();
  __syncthreads();
  if (inner) {
    // interior cells: plain bilinear weights (multigrid.c:376-400) from the staged coarse cells
#pragma unroll 2
    for (int k = threadIdx.x; k < G::N; k += NT) {
      const int ly = k / G::W, lx = k - ly * G::W;
      const int cip = (lx + 5 - H) >> 1, cjp = (ly + 5 - H) >> 1;
      const bool io = ((lx + H) & 1) != 0, jo = ((ly + H) & 1) != 0;
      const T ai = io ? T(0.75) : T(0.25), bi = io ? T(0.25) : T(0.75);
      const T aj = jo ? T(0.75) : T(0.25), bj = jo ? T(0.25) : T(0.75);
      const T wmm = ai * aj, wmp = ai * bj, wpm = bi * aj, wpp = bi * bj;
      const T* cc = b.ce + cjp * G::CW + cip;
      b.e[G::at(lx, ly)] -= wmm * cc[-G::CW - 1] + wpm * cc[-G::CW] + wmp * cc[-1] + wpp * cc[0];
    }
  } else {
    auto ec = [&](int a, int bb) { return c.e[IX(c, a, bb)]; };
    for (int k = threadIdx.x; k < G::N; k += NT) {
      const int ly = k / G::W, lx = k - ly * G::W;
      const int gi = wrapi(X0 - H + lx, f.Nx), gj = wrapi(Y0 - H + ly, f.Ny);
      b.e[G::at(lx, ly)] -= prolong_at<T>(gi, gj, f.Nx, f.Ny, c.Nx, c.Ny, true, wew, wns, ec);
    }
  }
  __syncthreads();
  tile_sweeps<T, OX, OY, H, NT, NU>(X0 + Y0, omega, b);
  double m = 0;
  for (int k = threadIdx.x; k < OX * OY; k += NT) {
    const int ly = k / OX, lx = k - ly * OX;
    const int gi = X0 + lx, gj = Y0 + ly;
    if (inner || (gi < f.Nx && gj < f.Ny)) {
      const int q = G::at(lx + H, ly + H);
      out[IX(f, gi, gj)] = b.e[q];
      if constexpr (MEASURE) {
        const int sp = (lx + H) & 1;
        const int qe = G::east(q, sp), qw = G::west(q, sp);
        const T s = b.Os[q + G::PW] * b.e[q + G::PW] + b.Os[q] * b.e[q - G::PW] + b.Ow[qe] * b.e[qe]
                  + b.Ow[q] * b.e[qw];
        const T r = b.e[q] - b.rO[q] * (s - b.rhs[q]);
        m = fmax(m, fabs((double)r));
      }
    }
  }
  if constexpr (MEASURE) block_max_to(m, bits);
}

template <typename T, int OX, int OY, int NT, int NU, bool MEASURE>
__global__ void __launch_bounds__(NT) up_tile(LV<T> f, LV<T> c, T omega, int wew, int wns,
                                              unsigned long long* bits, T* __restrict__ out) {
  up_tile_body<T, OX, OY, NT, NU, MEASURE>(f, c, omega, wew, wns, bits, out, blockIdx.x, blockIdx.y);
}

#include "mg_strip.cuh"

// shapes the autotuner chooses from (tiles of owned OX x OY cells with NT threads, or
// streamed strips): 0: 32x8/256, 1: 32x16/256, 2: 64x8/256, 3: 64x16/512, 4: strips
constexpr int kNumTileShapes = 5;
constexpr int kStripShape = 4;

// strips need a few segments' worth of rows and at least one full strip of columns
inline bool strip_ok(int Nx, int Ny) { return Nx >= 64 && Ny >= 48; }

inline int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

struct StripGrid {
  int S, nstrips, nsegs;
  unsigned blocks;
};
inline StripGrid strip_grid(int Nx, int Ny) {
  StripGrid g;
  g.S = strip_rows(Nx, Ny, num_sms());
  g.nstrips = (Nx + SP_OWN - 1) / SP_OWN;
  g.nsegs = (Ny + g.S - 1) / g.S;
  g.blocks = (unsigned)((g.nstrips * g.nsegs + SP_WARPS - 1) / SP_WARPS);
  return g;
}

template <typename T, int OX, int OY, int NT>
void set_tile_attrs() {
  cudaFuncSetAttribute(down_tile<T, OX, OY, NT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<T, OX, OY, 3>());
  cudaFuncSetAttribute(up_tile<T, OX, OY, NT, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<T, OX, OY, 2>());
  cudaFuncSetAttribute(up_tile<T, OX, OY, NT, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<T, OX, OY, 3>());
}

template <typename T, int OX, int OY, int NT>
void launch_down_shape(const LV<T>& f, const LV<T>& c, T omega, int zero_e, T* out, cudaStream_t s) {
  const dim3 grid((f.Nx + OX - 1) / OX, (f.Ny + OY - 1) / OY);
  down_tile<T, OX, OY, NT, 1><<<grid, NT, tile_bytes<T, OX, OY, 3>(), s>>>(f, c, omega, zero_e, out);
}

template <typename T, int OX, int OY, int NT>
void launch_up_shape(const LV<T>& f, const LV<T>& c, T omega, int wew, int wns, unsigned long long* bits,
                     T* out, cudaStream_t s) {
  const dim3 grid((f.Nx + OX - 1) / OX, (f.Ny + OY - 1) / OY);
  if (bits)
    up_tile<T, OX, OY, NT, 1, true><<<grid, NT, tile_bytes<T, OX, OY, 3>(), s>>>(f, c, omega, wew, wns, bits, out);
  else
    up_tile<T, OX, OY, NT, 1, false><<<grid, NT, tile_bytes<T, OX, OY, 2>(), s>>>(f, c, omega, wew, wns, bits, out);
}

template <typename T>
void set_all_tile_attrs() {
  cudaFuncSetAttribute(down_strip<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)strip_smem_bytes<T>(false));
  cudaFuncSetAttribute(up_strip<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)strip_smem_bytes<T>(true));
  cudaFuncSetAttribute(up_strip<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)strip_smem_bytes<T>(true));
  set_tile_attrs<T, 32, 8, 256>();
  set_tile_attrs<T, 32, 16, 256>();
  set_tile_attrs<T, 64, 8, 256>();
  set_tile_attrs<T, 64, 16, 512>();
}

template <typename T>
void launch_down(int shape, const LV<T>& f, const LV<T>& c, T omega, int zero_e, T* out, cudaStream_t s) {
  if (shape == kStripShape && !strip_ok(f.Nx, f.Ny)) shape = 3;
  switch (shape) {
    case 0: launch_down_shape<T, 32, 8, 256>(f, c, omega, zero_e, out, s); break;
    case 1: launch_down_shape<T, 32, 16, 256>(f, c, omega, zero_e, out, s); break;
    case 2: launch_down_shape<T, 64, 8, 256>(f, c, omega, zero_e, out, s); break;
    case 3: launch_down_shape<T, 64, 16, 512>(f, c, omega, zero_e, out, s); break;
    default: {
      const StripGrid g = strip_grid(f.Nx, f.Ny);
      down_strip<T><<<g.blocks, SP_WARPS * 32, strip_smem_bytes<T>(false), s>>>(f, c, omega, zero_e, out, g.S,
                                                                                 g.nstrips, g.nsegs);
    }
  }
}

template <typename T>
void launch_up(int shape, const LV<T>& f, const LV<T>& c, T omega, int wew, int wns, unsigned long long* bits,
               T* out, cudaStream_t s) {
  if (shape == kStripShape && !strip_ok(f.Nx, f.Ny)) shape = 3;
  switch (shape) {
    case 0: launch_up_shape<T, 32, 8, 256>(f, c, omega, wew, wns, bits, out, s); break;
    case 1: launch_up_shape<T, 32, 16, 256>(f, c, omega, wew, wns, bits, out, s); break;
    case 2: launch_up_shape<T, 64, 8, 256>(f, c, omega, wew, wns, bits, out, s); break;
    case 3: launch_up_shape<T, 64, 16, 512>(f, c, omega, wew, wns, bits, out, s); break;
    default: {
      const StripGrid g = strip_grid(f.Nx, f.Ny);
      const size_t shm = strip_smem_bytes<T>(true);
      if (bits)
        up_strip<T, true><<<g.blocks, SP_WARPS * 32, shm, s>>>(f, c, omega, wew, wns, bits, out, g.S, g.nstrips,
                                                               g.nsegs);
      else
        up_strip<T, false><<<g.blocks, SP_WARPS * 32, shm, s>>>(f, c, omega, wew, wns, bits, out, g.S, g.nstrips,
                                                                g.nsegs);
    }
  }
}

// a level runs the tile kernels when its transfer is exactly 2:1 (so every coloured
// neighbour across a periodic wrap keeps its parity) and it holds the tile's halo
inline bool tile_ok(int Nx, int Ny, bool power2, int pre, int post) {
  return power2 && pre == 1 && post == 1 && Nx >= 8 && Ny >= 8;
}

// ---------------------------------------------------------------- coarse levels in one CTA

}  // namespace

constexpr int CMAX_LEVELS = 12;

struct CoarseDesc {
  int n;                        // levels 0..n-1, index n-1 is the top of the block
  int Nx[CMAX_LEVELS], Ny[CMAX_LEVELS], pitch[CMAX_LEVELS], power2[CMAX_LEVELS];
  int lgx[CMAX_LEVELS];         // log2(Nx) when Nx is a power of two, else -1
  int off[CMAX_LEVELS];         // offset of each level inside every smem array
  int total;                    // cells of all levels
  const void *Ow[CMAX_LEVELS], *Os[CMAX_LEVELS], *rO[CMAX_LEVELS];
  const void* top_rhs;          // rhs of the top level (global, pitched)
  void* top_e;                  // output correction of the top level
  int top_from_e;               // start the top level from top_e instead of zero
  int wew, wns, pre, post;
  // tabulation mode: CTA b solves for the unit rhs at top cell b and writes the top
  // correction as column b of the row-major unit_n x unit_n matrix unit_out
  void* unit_out;
  int unit_n;
};

namespace {

constexpr int CT = 1024;

// levels of at most this many cells run on one warp, with warp barriers between phases
constexpr int CWARP_CELLS = 64;

// The coarse levels of the V-cycle in one CTA, all in shared memory. Levels above
// CWARP_CELLS cells run each phase (colour of a sweep, residual, restriction,
// prolongation) on the whole block with a block barrier after it; the small levels at the
// bottom of the cycle (down, coarsest, up) run on warp 0 alone with warp barriers, while
// the other warps wait at one block barrier.
template <typename T>
__global__ void __launch_bounds__(CT) coarse_kernel(const __grid_constant__ CoarseDesc d, T omega) {
  extern __shared__ unsigned char sm_raw[];
  T* E = reinterpret_cast<T*>(sm_raw);
  T* R = E + d.total;
  T* W = R + d.total;
  T* S = W + d.total;
  T* Q = S + d.total;
  T* RES = Q + d.total;
  const int tid = threadIdx.x;
  for (int l = 0; l < d.n; ++l) {
    const T* ow = (const T*)d.Ow[l];
    const T* os = (const T*)d.Os[l];
    const T* ro = (const T*)d.rO[l];
    int nx = d.Nx[l], ny = d.Ny[l], cnt = nx * ny;
    for (int q = tid; q < cnt; q += CT) {
      int i = q % nx, j = q / nx;
      size_t g = (size_t)j * d.pitch[l] + i;
      W[d.off[l] + q] = ow[g];
      S[d.off[l] + q] = os[g];
      Q[d.off[l] + q] = ro[g];
      E[d.off[l] + q] = (l == d.n - 1 && d.top_from_e) ? ((const T*)d.top_e)[g] : T(0);
      if (l == d.n - 1)
        R[d.off[l] + q] = d.unit_out ? T(q == (int)blockIdx.x ? 1 : 0) : ((const T*)d.top_rhs)[g];
    }
  }
  __syncthreads();
  auto cell = [&](int l, int q, int& i, int& j) {
    const int lg = d.lgx[l];
    if (lg >= 0) {
      i = q & ((1 << lg) - 1);
      j = q >> lg;
    } else {
      i = q % d.Nx[l];
      j = q / d.Nx[l];
    }
  };
  auto nsum = [&](int l, int i, int j) {
    int nx = d.Nx[l], ny = d.Ny[l], b = d.off[l];
    int ip1 = i + 1 == nx ? 0 : i + 1, im1 = i == 0 ? nx - 1 : i - 1;
    int jp1 = j + 1 == ny ? 0 : j + 1, jm1 = j == 0 ? ny - 1 : j - 1;
    return S[b + jp1 * nx + i] * E[b + jp1 * nx + i] + S[b + j * nx + i] * E[b + jm1 * nx + i]
         + W[b + j * nx + ip1] * E[b + j * nx + ip1] + W[b + j * nx + i] * E[b + j * nx + im1];
  };
  // the phases of one level, executed by threads q0, q0 + dq, ... with sync() after each
  auto smooth = [&](int l, int sweeps, int q0, int dq, auto sync) {
    int nx = d.Nx[l], b = d.off[l], cnt = nx * d.Ny[l];
    for (int s = 0; s < sweeps; ++s)
      for (int color = 0; color < 2; ++color) {
        for (int q = q0; q < cnt; q += dq) {
          int i, j;
          cell(l, q, i, j);
          if (((i + j) & 1) != color) continue;
          T sm = nsum(l, i, j);
          E[b + q] = omega * Q[b + q] * (sm - R[b + q]) + (T(1) - omega) * E[b + q];
        }
        sync();
      }
  };
  auto down = [&](int l, int q0, int dq, auto sync) {
    smooth(l, d.pre, q0, dq, sync);
    int nx = d.Nx[l], ny = d.Ny[l], b = d.off[l], cnt = nx * ny;
    for (int q = q0; q < cnt; q += dq) {
      int i, j;
      cell(l, q, i, j);
      int ip1 = i + 1 == nx ? 0 : i + 1, jp1 = j + 1 == ny ? 0 : j + 1;
      T osum = W[b + q] + W[b + j * nx + ip1] + S[b + q] + S[b + jp1 * nx + i];
      RES[q] = nsum(l, i, j) - osum * E[b + q] - R[b + q];
    }
    sync();
    int cnx = d.Nx[l - 1], cny = d.Ny[l - 1], cb = d.off[l - 1];
    for (int q = q0; q < cnx * cny; q += dq) {
      int ic, jc;
      cell(l - 1, q, ic, jc);
      T v;
      if (d.power2[l]) {
        const T* rr = RES + (2 * jc) * nx + 2 * ic;
        v = T(0.25) * (rr[0] + rr[1] + rr[nx] + rr[nx + 1]);
      } else {
        v = restrict_general_at<T>(nx, ny, cnx, cny, ic, jc, RES, nx);
      }
      R[cb + q] = v;
      E[cb + q] = 0;
    }
    sync();
  };
  auto up = [&](int l, int q0, int dq, auto sync) {
    int nx = d.Nx[l], ny = d.Ny[l], b = d.off[l];
    int cnx = d.Nx[l - 1], cny = d.Ny[l - 1], cb = d.off[l - 1];
    auto ec = [&](int a, int bb) { return E[cb + bb * cnx + a]; };
    for (int q = q0; q < nx * ny; q += dq) {
      int i, j;
      cell(l, q, i, j);
      E[b + q] -= prolong_at<T>(i, j, nx, ny, cnx, cny, d.power2[l] != 0, d.wew, d.wns, ec);
    }
    sync();
    smooth(l, d.post, q0, dq, sync);
  };
  auto block_sync = [] { __syncthreads(); };
  auto warp_sync = [] { __syncwarp(); };
  // levels 0..ls are small (level sizes grow with the index)
  int ls = -1;
  while (ls + 1 < d.n && d.Nx[ls + 1] * d.Ny[ls + 1] <= CWARP_CELLS) ++ls;
  for (int l = d.n - 1; l > ls && l >= 1; --l) down(l, tid, CT, block_sync);
  if (tid < 32) {
    if (ls >= 0) {
      for (int l = ls; l >= 1; --l) down(l, tid, 32, warp_sync);
      // coarsest: a single cell carries no information (multigrid.c:472-476)
      if (d.Nx[0] * d.Ny[0] == 1) {
        if (tid == 0) E[d.off[0]] = 0;
        __syncwarp();
      } else {
        smooth(0, d.pre + d.post, tid, 32, warp_sync);
      }
      for (int l = 1; l <= ls; ++l) up(l, tid, 32, warp_sync);
    }
  }
  __syncthreads();
  if (ls < 0) smooth(0, d.pre + d.post, tid, CT, block_sync);   // a coarsest level above CWARP_CELLS
  for (int l = (ls < 0 ? 1 : ls + 1); l < d.n; ++l) up(l, tid, CT, block_sync);
  int l = d.n - 1;
  for (int q = tid; q < d.Nx[l] * d.Ny[l]; q += CT) {
    int i = q % d.Nx[l], j = q / d.Nx[l];
    if (d.unit_out) ((T*)d.unit_out)[(size_t)q * d.unit_n + blockIdx.x] = E[d.off[l] + q];
    else ((T*)d.top_e)[(size_t)j * d.pitch[l] + i] = E[d.off[l] + q];
  }
}

// The coarse block started from a zero correction is a linear map of the top level's rhs
// (smoothing from zero, restriction and prolongation are linear): e_top = C rhs_top. C is
// tabulated once by running coarse_kernel on every unit rhs, then each V-cycle applies it
// as a matrix-vector product spread over the GPU (one warp per row, the rhs in shared
// memory), instead of one CTA walking the coarse levels phase by phase.
constexpr int CA_WARPS = 4;
template <typename T>
__device__ __forceinline__ void coarse_apply_body(const T* __restrict__ C, int n, int Nx, int pitch,
                                                  const T* __restrict__ rhs, T* __restrict__ e, int bx) {
  __shared__ T x[1024];
  for (int q = threadIdx.x; q < n; q += CA_WARPS * 32) x[q] = rhs[(size_t)(q / Nx) * pitch + q % Nx];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int row = bx * CA_WARPS + (threadIdx.x >> 5);
  if (row >= n) return;
  const T* c = C + (size_t)row * n;
  // four independent partial sums so that the loads of a row are all in flight at once
  T a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  int k = lane;
#pragma unroll 4
  for (; k + 96 < n; k += 128) {
    a0 += __ldg(c + k) * x[k];
    a1 += __ldg(c + k + 32) * x[k + 32];
    a2 += __ldg(c + k + 64) * x[k + 64];
    a3 += __ldg(c + k + 96) * x[k + 96];
  }
  for (; k < n; k += 32) a0 += __ldg(c + k) * x[k];
  T acc = (a0 + a1) + (a2 + a3);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) e[(size_t)(row / Nx) * pitch + row % Nx] = acc;
}

template <typename T>
__global__ void __launch_bounds__(CA_WARPS * 32) coarse_apply_kernel(const T* __restrict__ C, int n, int Nx, int pitch,
                                                                    const T* __restrict__ rhs, T* __restrict__ e) {
  coarse_apply_body<T>(C, n, Nx, pitch, rhs, e, blockIdx.x);
}

// ---------------------------------------------------------------- stopping test and loop control

struct LoopState {
  unsigned long long bits;   // max |pi - Jacobi(pi)| as an integer bit pattern
  int iters;
  int maxiters;
  double tol;
  double maxres;
  int* iters_out;            // nullable: receives iters and maxres after every cycle (the
  double* maxres_out;        // asynchronous solves' report slot)
};

// max |pi - Jacobi(pi)| on the fine level (multigrid.c:1123-1156); NaNs are ignored like fmax
__global__ void max_residual_kernel(LV<double> l, unsigned long long* bits) {
  double m = 0;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < l.Nx && j < l.Ny) {
    size_t c = IX(l, i, j);
    double r = l.e[c] - l.rOsum[c] * (neighbour_sum(l, l.e, i, j) - l.rhs[c]);
    m = fmax(m, fabs(r));
  }
  block_max_to(m, bits);
}

// the same measure for two fields sharing the operator and rhs (one read of them)
__global__ void max_residual2_kernel(LV<double> l, const double* pa, const double* pb, unsigned long long* bits) {
  double ma = 0, mb = 0;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < l.Nx && j < l.Ny) {
    size_t c = IX(l, i, j);
    ma = fmax(ma, fabs(pa[c] - l.rOsum[c] * (neighbour_sum(l, pa, i, j) - l.rhs[c])));
    mb = fmax(mb, fabs(pb[c] - l.rOsum[c] * (neighbour_sum(l, pb, i, j) - l.rhs[c])));
  }
  block_max_to(ma, &bits[0]);
  __syncthreads();
  block_max_to(mb, &bits[1]);
}

__global__ void loop_reset_kernel(LoopState* st, int maxiters, double tol, int* iters_out, double* maxres_out) {
  st->iters_out = iters_out;
  st->maxres_out = maxres_out;
  st->bits = 0;
  st->iters = 0;
  st->maxiters = maxiters;
  st->tol = tol;
  st->maxres = tol + 1;
}

// the loop condition of iterate_MG (multigrid.c:1185-1201)
__global__ void loop_finalize_kernel(LoopState* st, cudaGraphConditionalHandle h) {
  double m = __longlong_as_double((long long)st->bits);
  st->bits = 0;
  st->iters += 1;
  st->maxres = m;
  unsigned cont = (m > st->tol) && (st->iters < st->maxiters);
  if (st->iters_out) {
    *st->iters_out = st->iters;
    *st->maxres_out = m;
  }
  cudaGraphSetConditional(h, cont);
}

// FP64 defect step of the mixed-precision solve: pi_new = pi - e32 (when `correct`), the
// residual L(pi_new) - rhs stored as FP32 on the fine FP32 level, and the stopping measure
// of pi_new. pi ping-pongs between two arrays: cycle i reads `a` and writes `b` when i is
// even, the other way round when odd (i = *iter_dev, the device cycle count, or iter_host),
// so no copy-back pass is needed. Osum and 1/Osum are formed from the face coefficients
// already loaded (same sums and the same IEEE division as the stored arrays).
__global__ void defect_kernel(LV<double> l, double* a, double* b, const int* iter_dev, int iter_host,
                              const float* __restrict__ e32, int p32, float* r32, int correct,
                              unsigned long long* bits) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int it = iter_dev ? *iter_dev : iter_host;
  const double* pin = (it & 1) ? b : a;
  double* pout = (it & 1) ? a : b;
  double m = 0;
  if (i < l.Nx && j < l.Ny) {
    int ip1 = i + 1 == l.Nx ? 0 : i + 1, im1 = i == 0 ? l.Nx - 1 : i - 1;
    int jp1 = j + 1 == l.Ny ? 0 : j + 1, jm1 = j == 0 ? l.Ny - 1 : j - 1;
    auto P = [&](int x, int y) {
      double v = pin[IX(l, x, y)];
      if (correct) v -= (double)e32[(size_t)y * p32 + x];
      return v;
    };
    const size_t c = IX(l, i, j);
    const double ow = l.Ow[c], oe = l.Ow[IX(l, ip1, j)], os = l.Os[c], on = l.Os[IX(l, i, jp1)];
    const double osum = ow + oe + os + on;
    double ro = 1 / osum;
    if (!isfinite(ro)) ro = 0;
    double pc = P(i, j);
    double s = on * P(i, jp1) + os * P(i, jm1) + oe * P(ip1, j) + ow * P(im1, j);
    const double rh = l.rhs[c];
    m = fabs(pc - ro * (s - rh));
    if (m != m) m = 0;
    r32[(size_t)j * p32 + i] = (float)(s - osum * pc - rh);
    if (correct) pout[c] = pc;
  }
  block_max_to(m, bits);
}

// the asynchronous FP32 solve's end: when the last cycle (index iters - 1) was even it wrote pi
// to the scratch array, so copy it back; decided on the device from the loop state
__global__ void commit_if_even_kernel(const LoopState* st, double* dst, const double* src, int Nx, int Ny,
                                      int pitch) {
  const int it = st->iters;
  if (it <= 0 || ((it - 1) & 1) != 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  dst[(size_t)j * pitch + i] = src[(size_t)j * pitch + i];
}

__global__ void commit_kernel(double* dst, const double* src, int Nx, int Ny, int pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  dst[(size_t)j * pitch + i] = src[(size_t)j * pitch + i];
}

inline dim3 g2(int Nx, int Ny) { return dim3((Nx + 31) / 32, (Ny + 7) / 8); }
const dim3 B2(32, 8);

template <typename T> T* dalloc(size_t n) {
  T* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, n * sizeof(T));
  return p;
}

// host restriction with the reference's arithmetic (multigrid.c:651-740)
void host_restrict(int fnx, int fny, const std::vector<double>& f, int cnx, int cny, std::vector<double>& c,
                   bool power2) {
  c.assign((size_t)cnx * cny, 0.0);
  if (power2) {
    for (int i = 0; i < fnx / 2; ++i)
      for (int j = 0; j < fny / 2; ++j)
        c[(size_t)i * cny + j] = 0.25 * (f[(size_t)(2 * i) * fny + 2 * j] + f[(size_t)(2 * i + 1) * fny + 2 * j]
                                         + f[(size_t)(2 * i) * fny + 2 * j + 1] + f[(size_t)(2 * i + 1) * fny + 2 * j + 1]);
    return;
  }
  for (int ic = 0; ic < cnx; ++ic) {
    double x0 = ((double)ic) * fnx / cnx, x1 = ((double)(ic + 1)) * fnx / cnx;
    for (int jc = 0; jc < cny; ++jc) {
      double y0 = ((double)jc) * fny / cny, y1 = ((double)(jc + 1)) * fny / cny, wsum = 0;
      for (unsigned fi = (unsigned)floor(x0); fi < (unsigned)ceil(x1); ++fi) {
        double wx = fmin(x1, (double)(fi + 1)) - fmax(x0, (double)fi);
        if (wx <= 0) continue;
        for (unsigned fj = (unsigned)floor(y0); fj < (unsigned)ceil(y1); ++fj) {
          double wy = fmin(y1, (double)(fj + 1)) - fmax(y0, (double)fj);
          if (wy <= 0) continue;
          double w = wx * wy;
          c[(size_t)ic * cny + jc] += w * f[(size_t)fi * fny + fj];
          wsum += w;
        }
      }
      if (wsum > 0) c[(size_t)ic * cny + jc] /= wsum;
    }
  }
}


}  // namespace

struct Multigrid::Graphs {
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaGraphConditionalHandle handle[2];
  // options the graphs were captured with; any change rebuilds them
  int pre = -1, post = -1, inner = -1;
  double omega = -1;
};

Multigrid::Multigrid(int Nx, int Ny, double Lx, double Ly, bool wew, bool wns, const double* Hc_host,
                     const MGOptions& opt, cudaStream_t s)
    : Nx_(Nx), Ny_(Ny), wew_(wew), wns_(wns), opt_(opt), s_(s) {
  // level sizes, finest first (multigrid.c:224-263)
  std::vector<int> nxs, nys;
  int nx = Nx, ny = Ny;
  nxs.push_back(nx);
  nys.push_back(ny);
  while (nx > 1 || ny > 1) {
    nx = coarsen(nx);
    ny = coarsen(ny);
    nxs.push_back(nx);
    nys.push_back(ny);
  }
  int n = (int)nxs.size();
  lv_.resize(n);
  std::vector<std::vector<double>> Hc(n);
  Hc[n - 1].resize((size_t)Nx * Ny);
  for (int i = 0; i < Nx; ++i)
    for (int j = 0; j < Ny; ++j) Hc[n - 1][(size_t)i * Ny + j] = Hc_host[(size_t)j * Nx + i];
  for (int m = n - 1; m >= 0; --m) {
    Level& L = lv_[m];
    L.Nx = nxs[n - 1 - m];
    L.Ny = nys[n - 1 - m];
    L.pitch = round_up(L.Nx, 32);
    L.power2 = false;
    if (m > 0) {
      int cnx = nxs[n - m], cny = nys[n - m];
      L.power2 = (L.Nx == 2 * cnx) && (L.Ny == 2 * cny);
    }
  }
  for (int m = n - 2; m >= 0; --m)
    host_restrict(lv_[m + 1].Nx, lv_[m + 1].Ny, Hc[m + 1], lv_[m].Nx, lv_[m].Ny, Hc[m], lv_[m + 1].power2);
  bool good = true;
  for (int m = 0; m < n; ++m) {
    Level& L = lv_[m];
    int lx = L.Nx, ly = L.Ny;
    double dx = Lx / lx, dy = Ly / ly;
    std::vector<double> Ow((size_t)lx * ly), Os((size_t)lx * ly), Osum((size_t)lx * ly), rO((size_t)lx * ly);
    const std::vector<double>& H = Hc[m];
    auto at = [&](const std::vector<double>& a, int i, int j) { return a[(size_t)i * ly + j]; };
    for (int i = 0; i < lx; ++i) {
      int im1 = (i + lx - 1) % lx;
      for (int j = 0; j < ly; ++j) {
        int jm1 = (j + ly - 1) % ly;
        double Hw = 0.5 * (at(H, i, j) + at(H, im1, j));
        double Hs = 0.5 * (at(H, i, j) + at(H, i, jm1));
        Os[(size_t)i * ly + j] = Hs / (dy * dy);
        Ow[(size_t)i * ly + j] = Hw / (dx * dx);
      }
    }
    if (wns) for (int i = 0; i < lx; ++i) Os[(size_t)i * ly] = 0;
    if (wew) for (int j = 0; j < ly; ++j) Ow[(size_t)j] = 0;
    for (int i = 0; i < lx; ++i) {
      int ip1 = (i + lx + 1) % lx;
      for (int j = 0; j < ly; ++j) {
        int jp1 = (j + ly + 1) % ly;
        double s = at(Ow, i, j) + at(Ow, ip1, j) + at(Os, i, j) + at(Os, i, jp1);
        Osum[(size_t)i * ly + j] = s;
        rO[(size_t)i * ly + j] = 1 / s;
      }
    }
    size_t np = (size_t)L.pitch * ly;
    std::vector<double> buf(np, 0.0);
    std::vector<float> buf32(np, 0.f);
    double** dst64[4] = {&L.Ow, &L.Os, &L.Osum, &L.rOsum};
    float** dst32[4] = {&L.Ow32, &L.Os32, &L.Osum32, &L.rOsum32};
    const std::vector<double>* srcs[4] = {&Ow, &Os, &Osum, &rO};
    for (int a = 0; a < 4; ++a) {
      for (int i = 0; i < lx; ++i)
        for (int j = 0; j < ly; ++j) {
          double v = (*srcs[a])[(size_t)i * ly + j];
          if (a == 3 && !(isfinite(v))) v = 0;   // a 1x1 walled level has no operator
          buf[(size_t)j * L.pitch + i] = v;
          buf32[(size_t)j * L.pitch + i] = (float)v;
        }
      *dst64[a] = dalloc<double>(np);
      *dst32[a] = dalloc<float>(np);
      good = good && *dst64[a] && *dst32[a];
      if (!good) break;
      cudaMemcpy(*dst64[a], buf.data(), np * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(*dst32[a], buf32.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    }
    L.e = dalloc<double>(np); L.rhs = dalloc<double>(np); L.res = dalloc<double>(np);
    L.tmp = dalloc<double>(np); L.tmp32 = dalloc<float>(np);
    good = good && L.tmp && L.tmp32;
    L.e32 = dalloc<float>(np); L.rhs32 = dalloc<float>(np); L.res32 = dalloc<float>(np);
    good = good && L.e && L.rhs && L.res && L.e32 && L.rhs32 && L.res32;
  }
  own_e_ = lv_.back().e;
  own_rhs_ = lv_.back().rhs;
  // the top of the coarse block: the largest level with at most 1024 cells among the
  // CMAX_LEVELS coarsest (the block must fit one CTA's shared memory)
  ctop_ = 0;
  for (int m = 0; m < n && m < CMAX_LEVELS; ++m)
    if ((long long)lv_[m].Nx * lv_[m].Ny <= 1024) ctop_ = m;
  dstate_ = reinterpret_cast<void*>(dalloc<LoopState>(1));
  good = good && dstate_;
  cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking);
  g_ = new Graphs();
  ok_ = good;
  cudaFuncSetAttribute(coarse_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(coarse_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  set_all_tile_attrs<double>();
  set_all_tile_attrs<float>();
}

Multigrid::~Multigrid() {
  if (g_) {
    for (int p = 0; p < 2; ++p) {
      if (g_->exec[p]) cudaGraphExecDestroy(g_->exec[p]);
      if (g_->graph[p]) cudaGraphDestroy(g_->graph[p]);
    }
    delete g_;
  }
  if (cap_) cudaStreamDestroy(cap_);
  lv_.back().e = own_e_;
  lv_.back().rhs = own_rhs_;
  for (auto& L : lv_) {
    cudaFree(L.Ow); cudaFree(L.Os); cudaFree(L.Osum); cudaFree(L.rOsum);
    cudaFree(L.Ow32); cudaFree(L.Os32); cudaFree(L.Osum32); cudaFree(L.rOsum32);
    cudaFree(L.e); cudaFree(L.rhs); cudaFree(L.res); cudaFree(L.tmp); cudaFree(L.tmp32);
    cudaFree(L.e32); cudaFree(L.rhs32); cudaFree(L.res32);
  }
  cudaFree(dstate_);
  cudaFree(cmat_[0]);
  cudaFree(cmat_[1]);
}

template <typename T>
CoarseDesc Multigrid::coarse_desc(void* unit_out, int root) const {
  CoarseDesc dd;
  memset(&dd, 0, sizeof(dd));
  CoarseDesc* d = &dd;
  const int top = (int)lv_.size() - 1;
  const int btop = root >= 0 ? root : ctop_;
  d->n = btop + 1;
  int total = 0;
  for (int m = 0; m <= btop; ++m) {
    const Level& L = lv_[m];
    d->Nx[m] = L.Nx; d->Ny[m] = L.Ny; d->pitch[m] = L.pitch; d->power2[m] = L.power2 ? 1 : 0;
    d->lgx[m] = -1;
    for (int b = 0; b < 30; ++b)
      if (L.Nx == (1 << b)) d->lgx[m] = b;
    d->off[m] = total;
    total += L.Nx * L.Ny;
    if (sizeof(T) == 8) { d->Ow[m] = L.Ow; d->Os[m] = L.Os; d->rO[m] = L.rOsum; }
    else { d->Ow[m] = L.Ow32; d->Os[m] = L.Os32; d->rO[m] = L.rOsum32; }
  }
  d->total = total;
  const Level& Ltop = lv_[btop];
  d->top_rhs = sizeof(T) == 8 ? (const void*)Ltop.rhs : (const void*)Ltop.rhs32;
  d->top_e = sizeof(T) == 8 ? (void*)Ltop.e : (void*)Ltop.e32;
  // when the coarse block is the whole problem, the FP64 solve iterates on pi itself; a block
  // rooted at a lower level (the nested iteration) iterates on that level's solution
  d->top_from_e = ((btop == top || root >= 0) && sizeof(T) == 8) ? 1 : 0;
  d->wew = wew_; d->wns = wns_; d->pre = opt_.pre; d->post = opt_.post;
  d->unit_out = unit_out;
  d->unit_n = Ltop.Nx * Ltop.Ny;
  return dd;
}

template <typename T>
size_t Multigrid::coarse_smem(int root) const {
  const int btop = root >= 0 ? root : ctop_;
  int total = 0;
  for (int m = 0; m <= btop; ++m) total += lv_[m].Nx * lv_[m].Ny;
  return (size_t)(5 * total + lv_[btop].Nx * lv_[btop].Ny) * sizeof(T);
}

// tabulate the coarse block's linear map for the current smoother options (once per
// precision and option set; the tabulation runs the coarse kernel on every unit rhs)
template <typename T>
void Multigrid::tabulate_coarse(cudaStream_t s) {
  const int p = sizeof(T) == 8 ? 0 : 1;
  const int top = (int)lv_.size() - 1;
  if (ctop_ == top) return;   // the coarse block is the whole problem: iterate on pi itself
  if (cmat_[p] && cmat_pre_[p] == opt_.pre && cmat_post_[p] == opt_.post && cmat_omega_[p] == opt_.omega_rb)
    return;
  const int n = lv_[ctop_].Nx * lv_[ctop_].Ny;
  if (!cmat_[p] && cudaMalloc(&cmat_[p], (size_t)n * n * sizeof(T)) != cudaSuccess) {
    cmat_[p] = nullptr;
    return;
  }
  // a set-up launch, like the autotuner's, not counted as a step of the solve
  const CoarseDesc d = coarse_desc<T>(cmat_[p]);
  coarse_kernel<T><<<n, CT, coarse_smem<T>(), s>>>(d, (T)opt_.omega_rb);
  cmat_pre_[p] = opt_.pre;
  cmat_post_[p] = opt_.post;
  cmat_omega_[p] = opt_.omega_rb;
}

template <typename T>
void Multigrid::enqueue_vcycle(cudaStream_t s, unsigned long long* measure_bits, bool cont, int root) {
  const int finest = (int)lv_.size() - 1;
  const int top = root >= 0 ? root : finest;
  const T omega = (T)opt_.omega_rb;
  const int pre = opt_.pre, post = opt_.post;
  bool measured = false;
  if (top <= ctop_ && top < finest) {
    // a cycle rooted inside the coarse block (nested iteration): one CTA from the level's e
    CoarseDesc d = coarse_desc<T>(nullptr, top);
    coarse_kernel<T><<<1, CT, coarse_smem<T>(top), s>>>(d, omega);
    ++g_launches;
    if (measure_bits) {
      LV<double> f = view<double>(lv_[top]);
      max_residual_kernel<<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, measure_bits);
      ++g_launches;
    }
    return;
  }
  // down through the tiled levels
  for (int n = top; n > ctop_; --n) {
    Level& F = lv_[n];
    LV<T> f = view<T>(F), c = view<T>(lv_[n - 1]);
    // coarse corrections, and the FP32 correction of the defect loop, start from zero (a
    // continuing FP32 cycle starts from the correction of the previous one)
    bool zero_e = (n != top) || (sizeof(T) == 4 && !cont);
    if (tile_ok(F.Nx, F.Ny, F.power2, pre, post)) {
      launch_down<T>(sizeof(T) == 8 ? F.shape64 : F.shape32, f, c, omega, zero_e ? 1 : 0, f.tmp, s);
      ++g_launches;
    } else {
      if (zero_e) cudaMemsetAsync(f.e, 0, (size_t)F.pitch * F.Ny * sizeof(T), s);
      for (int q = 0; q < pre; ++q) {
        smooth_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, 0, omega);
        smooth_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, 1, omega);
      }
      residual_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f);
      restrict_general_kernel<T><<<g2(c.Nx, c.Ny), B2, 0, s>>>(f, c);
      g_launches += 2 * pre + 2;
    }
  }
  // coarse block: the tabulated linear map when available, else the one-CTA kernel
  {
    const Level& Ltop = lv_[ctop_];
    CoarseDesc d = coarse_desc<T>(nullptr);
    if (cont && ctop_ == top) d.top_from_e = 1;
    const T* C = static_cast<const T*>(cmat_[sizeof(T) == 8 ? 0 : 1]);
    if (C && !d.top_from_e) {
      const int n = Ltop.Nx * Ltop.Ny;
      coarse_apply_kernel<T><<<(n + CA_WARPS - 1) / CA_WARPS, CA_WARPS * 32, 0, s>>>(
          C, n, Ltop.Nx, Ltop.pitch, static_cast<const T*>(d.top_rhs), static_cast<T*>(d.top_e));
    } else {
      coarse_kernel<T><<<1, CT, coarse_smem<T>(), s>>>(d, omega);
    }
    ++g_launches;
  }
  // up through the tiled levels; the finest FP64 up kernel also forms the stopping measure
  for (int n = ctop_ + 1; n <= top; ++n) {
    Level& F = lv_[n];
    LV<T> f = view<T>(F), c = view<T>(lv_[n - 1]);
    if (tile_ok(F.Nx, F.Ny, F.power2, pre, post)) {
      unsigned long long* mb = (n == top && top == finest) ? measure_bits : nullptr;
      LV<T> fin = f;
      fin.e = f.tmp;   // the pre-smoothed correction written by the down kernel
      launch_up<T>(sizeof(T) == 8 ? F.shape64 : F.shape32, fin, c, omega, wew_, wns_, mb, f.e, s);
      ++g_launches;
      if (mb) measured = true;
    } else {
      prolong_correct_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, c, F.power2 ? 1 : 0, wew_, wns_);
      for (int q = 0; q < post; ++q) {
        smooth_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, 0, omega);
        smooth_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, 1, omega);
      }
      g_launches += 1 + 2 * post;
    }
  }
  if (measure_bits && !measured) {
    LV<double> f = view<double>(lv_[top]);
    max_residual_kernel<<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, measure_bits);
    ++g_launches;
  }
}

// Choose the tile shape of every tiled level by timing each shape's down and up kernels
// on that level. The runs read and write the level's scratch arrays only (the finest
// level's output goes to its `res` array), never the caller's pi. The choice only
// affects speed: every shape gives the same values.
template <typename T>
void Multigrid::tune(cudaStream_t s) {
  const int top = (int)lv_.size() - 1;
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  const long long counted = g_launches;
  for (int n = ctop_ + 1; n <= top; ++n) {
    Level& F = lv_[n];
    bool& tuned = sizeof(T) == 8 ? F.tuned64 : F.tuned32;
    int& shape = sizeof(T) == 8 ? F.shape64 : F.shape32;
    if (tuned) continue;
    tuned = true;
    if (opt_.tile_shape >= 0) {
      shape = opt_.tile_shape < kNumTileShapes ? opt_.tile_shape : kNumTileShapes - 1;
      continue;
    }
    if (const char* forced = getenv("PAWSIM_MG_SHAPES")) {
      // profiling recipes: the shapes of an unprofiled run, finest level first ("4,4,0,0")
      int k = top, v = 0;
      const char* c = forced;
      while (k > n && *c) {
        while (*c && *c != ',') ++c;
        if (*c) ++c;
        --k;
      }
      if (sscanf(c, "%d", &v) == 1 && v >= 0 && v < kNumTileShapes) {
        shape = v;
        continue;
      }
    }
    if (!tile_ok(F.Nx, F.Ny, F.power2, opt_.pre, opt_.post)) continue;
    LV<T> f = view<T>(F), c = view<T>(lv_[n - 1]);
    LV<T> fin = f;
    fin.e = f.tmp;
    T* out = f.res;
    unsigned long long* mb = (n == top && sizeof(T) == 8) ? &st->bits : nullptr;
    float best = 1e30f;
    for (int k = 0; k < kNumTileShapes; ++k) {
      if (k == kStripShape && !strip_ok(F.Nx, F.Ny)) continue;
      float ms = 0;
      for (int rep = 0; rep < 4; ++rep) {
        if (rep == 1) cudaEventRecord(ev[0], s);
        launch_down<T>(k, f, c, (T)opt_.omega_rb, 1, f.tmp, s);
        launch_up<T>(k, fin, c, (T)opt_.omega_rb, wew_, wns_, mb, out, s);
      }
      cudaEventRecord(ev[1], s);
      if (cudaEventSynchronize(ev[1]) != cudaSuccess) break;
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      if (ms < best) {
        best = ms;
        shape = k;
      }
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  g_launches = counted;   // tuning runs are not steps of the solve
  if (getenv("PAWSIM_MG_VERBOSE")) {
    // the shapes the tuner chose (0..3 tiles, kStripShape strips), for profiling recipes
    for (int n = ctop_ + 1; n <= top; ++n)
      fprintf(stderr, "pawsim mg: level %d (%d x %d) %s shape %d\n", n, lv_[n].Nx, lv_[n].Ny,
              sizeof(T) == 8 ? "fp64" : "fp32", sizeof(T) == 8 ? lv_[n].shape64 : lv_[n].shape32);
  }
}

void Multigrid::set_fine(double* pi, const double* rhs) {
  fine_pi_ = pi;
  fine_rhs_ = rhs;
  Level& F = lv_.back();
  F.e = pi;
  F.rhs = const_cast<double*>(rhs);
}

int Multigrid::build_graph(int prec) {
  cudaGraph_t& G = g_->graph[prec];
  if (cudaGraphCreate(&G, 0) != cudaSuccess) return -1;
  if (cudaGraphConditionalHandleCreate(&g_->handle[prec], G, 1, cudaGraphCondAssignDefault) != cudaSuccess) return -1;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = g_->handle[prec];
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, G, nullptr, 0, &cp) != cudaSuccess) return -1;
  if (capture_body(prec, cp.conditional.phGraph_out[0], g_->handle[prec]) != 0) return -1;
  if (cudaGraphInstantiate(&g_->exec[prec], G, 0) != cudaSuccess) return -1;
  return 0;
}

// The loop body (one V-cycle, or the FP32 cycles and the FP64 defect step, then the loop
// test that sets the conditional handle h) captured into `body`.
int Multigrid::capture_body(int prec, cudaGraph_t body, cudaGraphConditionalHandle h) {
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  const long long counted = g_launches;   // captured launches are counted per executed cycle
  if (cudaStreamBeginCaptureToGraph(cap_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return -1;
  Level& F = lv_.back();
  if (prec == 0) {
    enqueue_vcycle<double>(cap_, &st->bits);
  } else {
    enqueue_vcycle<float>(cap_, nullptr);
    for (int q = 1; q < opt_.fp32_inner; ++q) enqueue_vcycle<float>(cap_, nullptr, true);
    LV<double> f = view<double>(F);
    defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, cap_>>>(f, F.e, F.res, &st->iters, 0, F.e32, F.pitch, F.rhs32, 1,
                                                   &st->bits);
  }
  loop_finalize_kernel<<<1, 1, 0, cap_>>>(st, h);
  body_launches_[prec] = (int)(g_launches - counted) + (prec ? 2 : 1);   // + defect, finalize
  g_launches = counted;
  if (cudaStreamEndCapture(cap_, &body) != cudaSuccess) return -1;
  return 0;
}

// The V-cycle loop as a conditional node of the graph that s_ is being captured into (a handle
// of that graph, the body captured afresh), so that a larger captured graph holds whole solves.
// The same pattern as the loop graph's own; the outer capture continues after the node.
int Multigrid::add_loop_node(int prec) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t G = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s_, &cs, nullptr, &G, &deps, &nd) != cudaSuccess || cs != cudaStreamCaptureStatusActive)
    return -1;
  std::vector<cudaGraphNode_t> dv(deps, deps + nd);
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, G, 1, cudaGraphCondAssignDefault) != cudaSuccess) return -1;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, G, dv.data(), nd, &cp) != cudaSuccess) return -1;
  if (capture_body(prec, cp.conditional.phGraph_out[0], h) != 0) return -1;
  if (cudaStreamUpdateCaptureDependencies(s_, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return -1;
  return 0;
}

void Multigrid::measure_async(const double* pi, const double* rhs, unsigned long long* bits, cudaStream_t s) {
  LV<double> f = view<double>(lv_.back());
  f.e = const_cast<double*>(pi);
  f.rhs = const_cast<double*>(rhs);
  cudaMemsetAsync(bits, 0, sizeof(unsigned long long), s);
  max_residual_kernel<<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, bits);
  ++g_launches;
}

void Multigrid::measure2_async(const double* pa, const double* pb, const double* rhs, unsigned long long* bits,
                               cudaStream_t s) {
  LV<double> f = view<double>(lv_.back());
  f.rhs = const_cast<double*>(rhs);
  cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned long long), s);
  max_residual2_kernel<<<g2(f.Nx, f.Ny), B2, 0, s>>>(f, pa, pb, bits);
  ++g_launches;
}

double Multigrid::max_residual(const double* pi, int pitch, const double* rhs, int rhs_pitch) {
  Level& F = lv_.back();
  LV<double> f = view<double>(F);
  f.e = const_cast<double*>(pi);
  f.rhs = const_cast<double*>(rhs);
  (void)pitch; (void)rhs_pitch;
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
  max_residual_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, &st->bits);
  ++g_launches;
  unsigned long long b = 0;
  cudaMemcpyAsync(&b, &st->bits, sizeof(b), cudaMemcpyDeviceToHost, s_);
  cudaStreamSynchronize(s_);
  double m;
  memcpy(&m, &b, sizeof(m));
  return m;
}

int Multigrid::solve(double* pi, int pitch, const double* rhs, int rhs_pitch, double tol, int maxiters,
                     double* maxres_out) {
  (void)pitch; (void)rhs_pitch;
  if (opt_.omega_auto && !omega_tuned_ && nsolves_ >= 1) {
    omega_tuned_ = true;
    const Level& F = lv_.back();
    const size_t bytes = (size_t)F.pitch * F.Ny * sizeof(double);
    double* backup = nullptr;
    if (cudaMalloc(&backup, bytes) == cudaSuccess) {
      cudaMemcpyAsync(backup, pi, bytes, cudaMemcpyDeviceToDevice, s_);
      double best = 1.0;
      int best_it = -1;
      for (double w : kOmegaCandidates) {
        opt_.omega_rb = w;
        cudaMemcpyAsync(pi, backup, bytes, cudaMemcpyDeviceToDevice, s_);
        const int it = solve_once(pi, rhs, tol, maxiters, nullptr);
        if (it >= 0 && (best_it < 0 || it < best_it)) {
          best_it = it;
          best = w;
        }
      }
      opt_.omega_rb = best;
      cudaMemcpyAsync(pi, backup, bytes, cudaMemcpyDeviceToDevice, s_);
      cudaStreamSynchronize(s_);
      cudaFree(backup);
    }
  }
  ++nsolves_;
  return solve_once(pi, rhs, tol, maxiters, maxres_out);
}

// The nested iteration of full_MG (multigrid.c:1236-1270) below the finest level: the rhs is
// restricted to every level, the 1 x 1 level holds zero (exactSolve_MG), and each finer level
// starts from the interpolated coarser solution and runs FP64 V-cycles rooted at itself until
// its own stopping measure is within tol (or maxiters). The finest level's start is left in pi;
// its iteration is the regular solve. Host-sequenced: one measure read per coarse cycle.
int Multigrid::full_mg_start(double tol, int maxiters) {
  const int top = (int)lv_.size() - 1;
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  for (int n = top; n > 0; --n) {
    restrict_rhs_kernel<<<g2(lv_[n - 1].Nx, lv_[n - 1].Ny), B2, 0, s_>>>(view<double>(lv_[n]), view<double>(lv_[n - 1]),
                                                                       lv_[n].power2 ? 1 : 0);
    ++g_launches;
  }
  cudaMemsetAsync(lv_[0].e, 0, (size_t)lv_[0].pitch * lv_[0].Ny * sizeof(double), s_);
  for (int n = 1; n <= top; ++n) {
    LV<double> f = view<double>(lv_[n]), c = view<double>(lv_[n - 1]);
    prolong_set_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, c, lv_[n].power2 ? 1 : 0, wew_, wns_);
    ++g_launches;
    if (n == top) break;
    double mres = tol + 1;
    for (int it = 0; mres > tol && it < maxiters; ++it) {
      cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
      enqueue_vcycle<double>(s_, &st->bits, false, n);
      unsigned long long b = 0;
      cudaMemcpyAsync(&b, &st->bits, sizeof(b), cudaMemcpyDeviceToHost, s_);
      if (cudaStreamSynchronize(s_) != cudaSuccess) return -1;
      memcpy(&mres, &b, sizeof(mres));
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int Multigrid::solve_once(double* pi, const double* rhs, double tol, int maxiters, double* maxres_out) {
  const int prec = opt_.fp32_cycles ? 1 : 0;
  if (fine_pi_ != pi || fine_rhs_ != rhs || g_->pre != opt_.pre || g_->post != opt_.post ||
      g_->omega != opt_.omega_rb || g_->inner != opt_.fp32_inner) {
    for (int p = 0; p < 2; ++p) {
      if (g_->exec[p]) cudaGraphExecDestroy(g_->exec[p]);
      if (g_->graph[p]) cudaGraphDestroy(g_->graph[p]);
      g_->exec[p] = nullptr;
      g_->graph[p] = nullptr;
    }
    g_->pre = opt_.pre;
    g_->post = opt_.post;
    g_->inner = opt_.fp32_inner;
    g_->omega = opt_.omega_rb;
  }
  set_fine(pi, rhs);
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  if (prec == 0) {
    tune<double>(s_);
    tabulate_coarse<double>(s_);
  } else {
    tune<float>(s_);
    tabulate_coarse<float>(s_);
  }
  if (opt_.full_mg) {
    // the nested cycles below the finest level run in FP64 with its tile shapes and map
    if (prec == 1) {
      tune<double>(s_);
      tabulate_coarse<double>(s_);
    }
    if (full_mg_start(tol, maxiters) != 0) return -1;
  }
  if (getenv("PAWSIM_MG_HOST_LOOP")) {
    // host-driven loop with the same kernels (for profilers that do not see inside the
    // conditional graph node)
    Level& F = lv_.back();
    LV<double> f = view<double>(F);
    int it = 0;
    double mres = tol + 1;
    if (prec == 1) {
      cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
      defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e, F.res, nullptr, 0, F.e32, F.pitch, F.rhs32, 0, &st->bits);
    }
    while (mres > tol && it < maxiters) {
      cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
      if (prec == 0) {
        enqueue_vcycle<double>(s_, &st->bits);
      } else {
        enqueue_vcycle<float>(s_, nullptr);
        for (int q = 1; q < opt_.fp32_inner; ++q) enqueue_vcycle<float>(s_, nullptr, true);
        defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e, F.res, nullptr, it, F.e32, F.pitch, F.rhs32, 1,
                                                     &st->bits);
      }
      unsigned long long b = 0;
      cudaMemcpyAsync(&b, &st->bits, sizeof(b), cudaMemcpyDeviceToHost, s_);
      if (cudaStreamSynchronize(s_) != cudaSuccess) return -1;
      memcpy(&mres, &b, sizeof(mres));
      ++it;
    }
    // the last cycle wrote pi to the scratch array when its index was even
    if (prec == 1 && it > 0 && ((it - 1) & 1) == 0)
      commit_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(F.e, F.res, F.Nx, F.Ny, F.pitch);
    if (maxres_out) *maxres_out = mres;
    return it;
  }
  if (!g_->exec[prec] && build_graph(prec) != 0) return -1;
  loop_reset_kernel<<<1, 1, 0, s_>>>(st, maxiters, tol, nullptr, nullptr);
  ++g_launches;
  if (prec == 1) {
    Level& F = lv_.back();
    LV<double> f = view<double>(F);
    defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e, F.res, nullptr, 0, F.e32, F.pitch, F.rhs32, 0, &st->bits);
    cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
    ++g_launches;
  }
  if (cudaGraphLaunch(g_->exec[prec], s_) != cudaSuccess) return -1;
  LoopState h;
  cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s_);
  if (cudaStreamSynchronize(s_) != cudaSuccess) return -1;
  if (prec == 1 && h.iters > 0 && ((h.iters - 1) & 1) == 0) {
    // the last cycle wrote pi to the scratch array
    Level& F = lv_.back();
    commit_kernel<<<g2(F.Nx, F.Ny), B2, 0, s_>>>(F.e, F.res, F.Nx, F.Ny, F.pitch);
    ++g_launches;
    if (cudaStreamSynchronize(s_) != cudaSuccess) return -1;
  }
  // kernels of the graph body, counted once per executed V-cycle
  g_launches += (long long)h.iters * body_launches_[prec];
  if (maxres_out) *maxres_out = h.maxres;
  return h.iters;
}

bool Multigrid::async_ready() const {
  const int prec = opt_.fp32_cycles ? 1 : 0;
  return g_->exec[prec] != nullptr && !opt_.full_mg && (!opt_.omega_auto || omega_tuned_) &&
         fine_pi_ != nullptr;
}

int Multigrid::solve_async(double* pi, const double* rhs, double tol, int maxiters, int* iters_out,
                           double* maxres_out, long long* launches) {
  const int prec = opt_.fp32_cycles ? 1 : 0;
  if (fine_pi_ != pi || fine_rhs_ != rhs || !g_->exec[prec]) return -1;
  LoopState* st = reinterpret_cast<LoopState*>(dstate_);
  ++nsolves_;
  loop_reset_kernel<<<1, 1, 0, s_>>>(st, maxiters, tol, iters_out, maxres_out);
  *launches = 1;
  Level& F = lv_.back();
  if (prec == 1) {
    LV<double> f = view<double>(F);
    defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e, F.res, nullptr, 0, F.e32, F.pitch, F.rhs32, 0, &st->bits);
    cudaMemsetAsync(&st->bits, 0, sizeof(unsigned long long), s_);
    ++*launches;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s_, &cs) != cudaSuccess) return -1;
  if (cs == cudaStreamCaptureStatusActive) {
    // the caller captures a larger graph: the loop becomes one of its nodes
    if (add_loop_node(prec) != 0) return -1;
  } else if (cudaGraphLaunch(g_->exec[prec], s_) != cudaSuccess) {
    return -1;
  }
  if (prec == 1) {
    commit_if_even_kernel<<<g2(F.Nx, F.Ny), B2, 0, s_>>>(st, F.e, F.res, F.Nx, F.Ny, F.pitch);
    ++*launches;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------- batched solves (MGBatch)

namespace {

struct BatchLevel {   // one member's arrays for a level kernel of the batched V-cycle
  LV<double> f, c;
  double omega;
  double* out;
  int zero_e;
};

struct BatchCoarse {  // one member's tabulated coarse map and its top-level arrays
  const double* C;
  const double* rhs;
  double* e;
};

struct BatchLoop {    // one member's loop state (the batched LoopState)
  unsigned long long bits;   // max |pi - Jacobi(pi)| of the cycle, as an integer bit pattern
  int iters;
  int active;                // still iterating
  int maxiters;
  double tol;
  double maxres;
};

// the batched level kernels' tile shapes: 64 x 16 tiles (less halo per owned cell) where a
// level holds at least kBigLevel cells over all members, 32 x 8 tiles below (more CTAs);
// every shape gives the same values
constexpr long long kBigLevel = 1 << 20;

template <int OX, int OY, int NT>
__global__ void __launch_bounds__(NT) down_batch_kernel(const BatchLevel* __restrict__ d,
                                                         const BatchLoop* __restrict__ st) {
  const int m = blockIdx.z;
  if (!st[m].active) return;
  const BatchLevel L = d[m];
  down_tile_body<double, OX, OY, NT, 1>(L.f, L.c, L.omega, L.zero_e, L.out, blockIdx.x, blockIdx.y);
}

template <int OX, int OY, int NT, bool MEASURE>
__global__ void __launch_bounds__(NT) up_batch_kernel(const BatchLevel* __restrict__ d, BatchLoop* st, int wew,
                                                       int wns) {
  const int m = blockIdx.z;
  if (!st[m].active) return;
  const BatchLevel L = d[m];
  up_tile_body<double, OX, OY, NT, 1, MEASURE>(L.f, L.c, L.omega, wew, wns, &st[m].bits, L.out, blockIdx.x,
                                               blockIdx.y);
}

// the streamed strip kernels over every member (blockIdx.y = member) on the big levels
__global__ void __launch_bounds__(SP_WARPS * 32, SP_CTAS_DOWN)
down_strip_batch_kernel(const BatchLevel* __restrict__ d, const BatchLoop* __restrict__ st, int S, int nstrips,
                        int nsegs) {
  const int m = blockIdx.y;
  if (!st[m].active) return;
  const BatchLevel L = d[m];
  down_strip_body<double>(L.f, L.c, L.omega, L.zero_e, L.out, S, nstrips, nsegs, blockIdx.x);
}

template <bool MEASURE>
__global__ void __launch_bounds__(SP_WARPS * 32, SP_CTAS_UP)
up_strip_batch_kernel(const BatchLevel* __restrict__ d, BatchLoop* st, int wew, int wns, int S, int nstrips,
                      int nsegs) {
  const int m = blockIdx.y;
  if (!st[m].active) return;
  const BatchLevel L = d[m];
  up_strip_body<double, MEASURE>(L.f, L.c, L.omega, wew, wns, &st[m].bits, L.out, S, nstrips, nsegs, blockIdx.x);
}

// strips of one member's level when `count` members share the GPU: longer segments than a
// single grid takes, so that the members' strips together fill it once
inline StripGrid strip_grid_batch(int Nx, int Ny, int count) {
  StripGrid g;
  const int sms = num_sms() / count;
  g.S = strip_rows(Nx, Ny, sms < 1 ? 1 : sms);
  g.nstrips = (Nx + SP_OWN - 1) / SP_OWN;
  g.nsegs = (Ny + g.S - 1) / g.S;
  g.blocks = (unsigned)((g.nstrips * g.nsegs + SP_WARPS - 1) / SP_WARPS);
  return g;
}

template <int OX, int OY, int NT>
void set_batch_attrs() {
  cudaFuncSetAttribute(down_batch_kernel<OX, OY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<double, OX, OY, 3>());
  cudaFuncSetAttribute(up_batch_kernel<OX, OY, NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<double, OX, OY, 3>());
  cudaFuncSetAttribute(up_batch_kernel<OX, OY, NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)tile_bytes<double, OX, OY, 2>());
}

template <int OX, int OY, int NT>
void launch_down_batch(int nx, int ny, int count, const BatchLevel* d, const BatchLoop* st, cudaStream_t s) {
  const dim3 grid((nx + OX - 1) / OX, (ny + OY - 1) / OY, count);
  down_batch_kernel<OX, OY, NT><<<grid, NT, tile_bytes<double, OX, OY, 3>(), s>>>(d, st);
}

template <int OX, int OY, int NT>
void launch_up_batch(int nx, int ny, int count, bool measure, const BatchLevel* d, BatchLoop* st, int wew, int wns,
                     cudaStream_t s) {
  const dim3 grid((nx + OX - 1) / OX, (ny + OY - 1) / OY, count);
  if (measure)
    up_batch_kernel<OX, OY, NT, true><<<grid, NT, tile_bytes<double, OX, OY, 3>(), s>>>(d, st, wew, wns);
  else
    up_batch_kernel<OX, OY, NT, false><<<grid, NT, tile_bytes<double, OX, OY, 2>(), s>>>(d, st, wew, wns);
}

__global__ void __launch_bounds__(CA_WARPS * 32) coarse_batch_kernel(const BatchCoarse* __restrict__ d,
                                                                      const BatchLoop* __restrict__ st, int n, int Nx,
                                                                      int pitch) {
  const int m = blockIdx.y;
  if (!st[m].active) return;
  const BatchCoarse B = d[m];
  coarse_apply_body<double>(B.C, n, Nx, pitch, B.rhs, B.e, blockIdx.x);
}

// flag = 1 when the two arrays differ in any bit (the members' coarse maps are shared when equal)
__global__ void differ_kernel(const unsigned long long* __restrict__ a, const unsigned long long* __restrict__ b,
                              size_t n, int* flag) {
  int d = 0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    d |= a[q] != b[q];
  if (__syncthreads_or(d) && threadIdx.x == 0) *flag = 1;
}

__global__ void batch_reset_kernel(BatchLoop* st, int n) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    st[m].bits = 0;
    st[m].iters = 0;
    st[m].active = 1;
    st[m].maxres = st[m].tol + 1;
  }
}

// the loop test of every member still iterating (loop_finalize_kernel per member); the loop
// continues while any member does. One block.
__global__ void batch_finalize_kernel(BatchLoop* st, int n, int* const* it_out, double* const* meas_out,
                                      cudaGraphConditionalHandle h) {
  int any = 0;
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    BatchLoop& s = st[m];
    if (s.active) {
      const double v = __longlong_as_double((long long)s.bits);
      s.bits = 0;
      s.iters += 1;
      s.maxres = v;
      *it_out[m] = s.iters;
      *meas_out[m] = v;
      s.active = (v > s.tol) && (s.iters < s.maxiters);
    }
    any |= s.active;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

}  // namespace

struct MGBatch::Group {
  int off = 0, count = 0;        // members [off, off + count) of the loop state
  int top = 0, ctop = 0;         // level indices of the finest level and the coarse block's top
  int wew = 0, wns = 0;
  std::vector<int> nx, ny;       // per level
  std::vector<BatchLevel*> down, up;   // per level (device arrays of count entries)
  BatchCoarse* coarse = nullptr;
  int cn = 0, cnx = 0, cpitch = 0;     // the coarse block's top level
  ~Group() {
    for (BatchLevel* p : down) cudaFree(p);
    for (BatchLevel* p : up) cudaFree(p);
    cudaFree(coarse);
  }
};

MGBatch::MGBatch(const std::vector<Multigrid*>& members, const std::vector<double>& tol,
                 const std::vector<int>& maxiters, const std::vector<int*>& it_out,
                 const std::vector<double*>& meas_out) {
  n_ = (int)members.size();
  if (n_ < 1 || tol.size() != members.size() || maxiters.size() != members.size() ||
      it_out.size() != members.size() || meas_out.size() != members.size())
    return;
  for (const Multigrid* g : members) {
    const int top = (int)g->lv_.size() - 1;
    if (!g->async_ready() || g->opt_.fp32_cycles || g->opt_.pre != 1 || g->opt_.post != 1 || g->opt_.full_mg ||
        !g->cmat_[0] || top <= g->ctop_ || g->lv_[g->ctop_].Nx * g->lv_[g->ctop_].Ny > 1024)
      return;
    for (int n = g->ctop_ + 1; n <= top; ++n)
      if (!tile_ok(g->lv_[n].Nx, g->lv_[n].Ny, g->lv_[n].power2, 1, 1)) return;
  }
  // group the members by level hierarchy (finest size and walls), keeping their order
  std::vector<int> order;
  std::vector<std::vector<int>> sets;
  for (int i = 0; i < n_; ++i) {
    const Multigrid* g = members[i];
    int found = -1;
    for (size_t k = 0; k < sets.size(); ++k) {
      const Multigrid* r = members[sets[k][0]];
      if (r->Nx_ == g->Nx_ && r->Ny_ == g->Ny_ && r->wew_ == g->wew_ && r->wns_ == g->wns_ &&
          r->lv_.size() == g->lv_.size() && r->ctop_ == g->ctop_)
        found = (int)k;
    }
    if (found < 0) {
      sets.emplace_back();
      found = (int)sets.size() - 1;
    }
    sets[found].push_back(i);
  }
  // loop state and report slots in group order
  std::vector<BatchLoop> hl;
  std::vector<int*> hit;
  std::vector<double*> hmeas;
  bool good = true;
  body_launches_ = 1;   // the loop test
  for (const std::vector<int>& set : sets) {
    Group* G = new Group();
    groups_.push_back(G);
    const Multigrid* r = members[set[0]];
    G->off = (int)hl.size();
    G->count = (int)set.size();
    G->top = (int)r->lv_.size() - 1;
    G->ctop = r->ctop_;
    G->wew = r->wew_ ? 1 : 0;
    G->wns = r->wns_ ? 1 : 0;
    G->nx.resize(G->top + 1);
    G->ny.resize(G->top + 1);
    G->down.assign(G->top + 1, nullptr);
    G->up.assign(G->top + 1, nullptr);
    for (int n = 0; n <= G->top; ++n) {
      G->nx[n] = r->lv_[n].Nx;
      G->ny[n] = r->lv_[n].Ny;
    }
    for (int n = G->ctop + 1; n <= G->top; ++n) {
      std::vector<BatchLevel> dn(G->count), upv(G->count);
      for (int q = 0; q < G->count; ++q) {
        Multigrid* g = members[set[q]];
        const LV<double> f = view<double>(g->lv_[n]), c = view<double>(g->lv_[n - 1]);
        dn[q] = BatchLevel{f, c, g->opt_.omega_rb, f.tmp, n != G->top ? 1 : 0};
        LV<double> fin = f;
        fin.e = f.tmp;   // the pre-smoothed correction written by the down kernel
        upv[q] = BatchLevel{fin, c, g->opt_.omega_rb, f.e, 0};
      }
      good = good && cudaMalloc(&G->down[n], G->count * sizeof(BatchLevel)) == cudaSuccess &&
             cudaMalloc(&G->up[n], G->count * sizeof(BatchLevel)) == cudaSuccess &&
             cudaMemcpy(G->down[n], dn.data(), G->count * sizeof(BatchLevel), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(G->up[n], upv.data(), G->count * sizeof(BatchLevel), cudaMemcpyHostToDevice) == cudaSuccess;
      body_launches_ += 2;
    }
    std::vector<BatchCoarse> cv(G->count);
    const Multigrid::Level& Lt = r->lv_[G->ctop];
    G->cn = Lt.Nx * Lt.Ny;
    G->cnx = Lt.Nx;
    G->cpitch = Lt.pitch;
    // members whose coarse maps are bit-identical (same depth field and smoother weight, as in
    // an ensemble over one basin) read one copy, which then stays in L2 across the group
    int* flags = nullptr;
    good = good && cudaMalloc(&flags, G->count * sizeof(int)) == cudaSuccess &&
           cudaMemset(flags, 0, G->count * sizeof(int)) == cudaSuccess;
    const size_t cwords = (size_t)G->cn * G->cn;
    const double* C0 = static_cast<const double*>(members[set[0]]->cmat_[0]);
    for (int q = 1; good && q < G->count; ++q)
      differ_kernel<<<64, 256>>>(static_cast<const unsigned long long*>(members[set[q]]->cmat_[0]),
                                 reinterpret_cast<const unsigned long long*>(C0), cwords, flags + q);
    std::vector<int> differs(G->count, 1);
    good = good && cudaMemcpy(differs.data(), flags, G->count * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(flags);
    for (int q = 0; q < G->count; ++q) {
      Multigrid* g = members[set[q]];
      const Multigrid::Level& L = g->lv_[g->ctop_];
      const double* C = (q > 0 && !differs[q]) ? C0 : static_cast<const double*>(g->cmat_[0]);
      cv[q] = BatchCoarse{C, L.rhs, L.e};
    }
    good = good && cudaMalloc(&G->coarse, G->count * sizeof(BatchCoarse)) == cudaSuccess &&
           cudaMemcpy(G->coarse, cv.data(), G->count * sizeof(BatchCoarse), cudaMemcpyHostToDevice) == cudaSuccess;
    body_launches_ += 1;
    for (int q = 0; q < G->count; ++q) {
      const int i = set[q];
      BatchLoop b;
      memset(&b, 0, sizeof(b));
      b.tol = tol[i];
      b.maxiters = maxiters[i];
      hl.push_back(b);
      hit.push_back(it_out[i]);
      hmeas.push_back(meas_out[i]);
    }
  }
  good = good && cudaMalloc(&loop_, n_ * sizeof(BatchLoop)) == cudaSuccess &&
         cudaMalloc(&it_out_, n_ * sizeof(int*)) == cudaSuccess &&
         cudaMalloc(&meas_out_, n_ * sizeof(double*)) == cudaSuccess &&
         cudaMemcpy(loop_, hl.data(), n_ * sizeof(BatchLoop), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(it_out_, hit.data(), n_ * sizeof(int*), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(meas_out_, hmeas.data(), n_ * sizeof(double*), cudaMemcpyHostToDevice) == cudaSuccess;
  if (good) {
    set_batch_attrs<32, 8, 256>();
    set_batch_attrs<64, 16, 512>();
    cudaFuncSetAttribute(down_strip_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)strip_smem_bytes<double>(false));
    cudaFuncSetAttribute(up_strip_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)strip_smem_bytes<double>(true));
    cudaFuncSetAttribute(up_strip_batch_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)strip_smem_bytes<double>(true));
  }
  ok_ = good && cudaGetLastError() == cudaSuccess;
}

MGBatch::~MGBatch() {
  for (Group* g : groups_) delete g;
  cudaFree(loop_);
  cudaFree(it_out_);
  cudaFree(meas_out_);
}

int MGBatch::capture(cudaStream_t s, cudaStream_t cap) {
  if (!ok_) return -1;
  BatchLoop* st = static_cast<BatchLoop*>(loop_);
  batch_reset_kernel<<<(n_ + 255) / 256, 256, 0, s>>>(st, n_);
  ++g_launches;
  cudaStreamCaptureStatus cs;
  cudaGraph_t G = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &G, &deps, &nd) != cudaSuccess || cs != cudaStreamCaptureStatusActive)
    return -1;
  std::vector<cudaGraphNode_t> dv(deps, deps + nd);
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, G, 1, cudaGraphCondAssignDefault) != cudaSuccess) return -1;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, G, dv.data(), nd, &cp) != cudaSuccess) return -1;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return -1;
  for (const Group* g : groups_) {
    BatchLoop* gs = st + g->off;
    auto big = [&](int n) { return (long long)g->count * g->nx[n] * g->ny[n] >= kBigLevel; };
    auto strips = [&](int n) { return big(n) && strip_ok(g->nx[n], g->ny[n]); };
    for (int n = g->top; n > g->ctop; --n) {
      if (strips(n)) {
        const StripGrid sg = strip_grid_batch(g->nx[n], g->ny[n], g->count);
        down_strip_batch_kernel<<<dim3(sg.blocks, g->count), SP_WARPS * 32, strip_smem_bytes<double>(false), cap>>>(
            g->down[n], gs, sg.S, sg.nstrips, sg.nsegs);
      } else if (big(n)) {
        launch_down_batch<64, 16, 512>(g->nx[n], g->ny[n], g->count, g->down[n], gs, cap);
      } else {
        launch_down_batch<32, 8, 256>(g->nx[n], g->ny[n], g->count, g->down[n], gs, cap);
      }
    }
    coarse_batch_kernel<<<dim3((g->cn + CA_WARPS - 1) / CA_WARPS, g->count), CA_WARPS * 32, 0, cap>>>(
        g->coarse, gs, g->cn, g->cnx, g->cpitch);
    for (int n = g->ctop + 1; n <= g->top; ++n) {
      if (strips(n)) {
        const StripGrid sg = strip_grid_batch(g->nx[n], g->ny[n], g->count);
        const dim3 grid(sg.blocks, g->count);
        if (n == g->top)
          up_strip_batch_kernel<true><<<grid, SP_WARPS * 32, strip_smem_bytes<double>(true), cap>>>(
              g->up[n], gs, g->wew, g->wns, sg.S, sg.nstrips, sg.nsegs);
        else
          up_strip_batch_kernel<false><<<grid, SP_WARPS * 32, strip_smem_bytes<double>(true), cap>>>(
              g->up[n], gs, g->wew, g->wns, sg.S, sg.nstrips, sg.nsegs);
      } else if (big(n)) {
        launch_up_batch<64, 16, 512>(g->nx[n], g->ny[n], g->count, n == g->top, g->up[n], gs, g->wew, g->wns, cap);
      } else {
        launch_up_batch<32, 8, 256>(g->nx[n], g->ny[n], g->count, n == g->top, g->up[n], gs, g->wew, g->wns, cap);
      }
    }
  }
  batch_finalize_kernel<<<1, 256, 0, cap>>>(st, n_, it_out_, meas_out_, h);
  if (cudaStreamEndCapture(cap, &body) != cudaSuccess) return -1;
  if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template void Multigrid::enqueue_vcycle<double>(cudaStream_t, unsigned long long*, bool, int);
template void Multigrid::enqueue_vcycle<float>(cudaStream_t, unsigned long long*, bool, int);

}  // namespace pawsim
