// common.cuh -- device-side layout, boundary mapping and launch helpers.
//
// Layout: every 2-D field is FP64 (or FP32 inside the multigrid preconditioner), x fastest
// (the AWSIM disk order), rows of `pitch` elements (a multiple of 32, so every row starts on
// a 256-byte boundary), layers `lstride = Ny*pitch` apart. Only owned cells are stored; the
// reference's 3-cell ghost ring (model_code/pawsim.c:28) and its halo exchanges
// (model_code/field.c:121-241) are replaced by the index maps below, applied at load time.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace pawsim {

// Boundary behaviour of a field along one axis (model_code/field.c:158-241):
//   MAP_S  scalar and wall-parallel velocity: mirror about the wall (F(-1) = F(0))
//   MAP_N  wall-normal velocity: zero on the wall face, odd mirror beyond it
//          (F(0) = +0, F(-i) = -F(i), F(N) = -0, F(N+i) = -F(N-i))
//   MAP_Q  q-grid: nearest of the N+1 stored lines
enum MapKind { MAP_S = 0, MAP_N = 1, MAP_Q = 2 };

struct AxisMap {
  int idx;      // source index in [0, N) (or [0, N] for MAP_Q)
  double sgn;   // +1 or -1
  bool zero;    // value is a signed zero (sgn carries the sign)
};

// i mod n for the few-cells-out-of-range indices of stencils; no integer division unless
// the index is more than one period away
__host__ __device__ inline int wrap_index(int i, int n) {
  if (i < 0) i += n;
  if (i >= n) i -= n;
  if (i < 0 || i >= n) {
    i %= n;
    if (i < 0) i += n;
  }
  return i;
}

// Map a raw coordinate i (any integer within a few cells of [0, N)) to storage.
__host__ __device__ inline AxisMap map_axis(int i, int n, bool wall, int kind) {
  AxisMap m;
  m.sgn = 1.0;
  m.zero = false;
  if (!wall) {
    m.idx = wrap_index(i, n);
    return m;
  }
  if (kind == MAP_Q) {
    m.idx = i < 0 ? 0 : (i > n ? n : i);
    return m;
  }
  if (kind == MAP_S) {
    if (i < 0) m.idx = -i - 1;
    else if (i >= n) m.idx = 2 * n - i - 1;
    else m.idx = i;
    return m;
  }
  // MAP_N
  if (i == 0) { m.idx = 0; m.zero = true; return m; }
  if (i == n) { m.idx = 0; m.zero = true; m.sgn = -1.0; return m; }
  if (i < 0) { m.idx = -i; m.sgn = -1.0; return m; }
  if (i > n) { m.idx = 2 * n - i; m.sgn = -1.0; return m; }
  m.idx = i;
  return m;
}

// Read a field at raw (i, j) with the x and y boundary kinds of that field. The sign of
// a wall zero follows the reference exactly (+0 on the west/south face, -0 on east/north).
__host__ __device__ inline double load_mapped(const double* __restrict__ f, int pitch, int i, int j,
                                              int nx, int ny, bool wx, bool wy, int kx, int ky) {
  AxisMap ax = map_axis(i, nx, wx, kx);
  if (ax.zero) return ax.sgn * 0.0;
  AxisMap ay = map_axis(j, ny, wy, ky);
  if (ay.zero) return ay.sgn * 0.0;
  double v = f[(size_t)ay.idx * pitch + ax.idx];
  return (ax.sgn * ay.sgn < 0) ? -v : v;
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// ---- corner ghosts of the reference's serial build on x-periodic, y-walled grids.
// There a halo fill copies whole columns periodically in x first, ghost rows included, and
// only then fills the wall ghost rows of the owned columns (model_code/field.c:353-532), so
// the four corner blocks receive what the ghost rows of the periodic image columns held
// before this fill. For the copied work arrays (u, v, h, b: pawsim_work_load_state,
// work.c:538-559) that is the previous fill's wall mirror. The library keeps those values in a
// small "corner shadow": per field and layer the owned values of the previous fill at the 3
// columns next to each side of the periodic seam and the 4 rows next to each wall. A load at a
// corner position reads the shadow through the wall mirror instead of the current field.
// (Fields computed over the ghosted array before their fill, such as the face thickness, get
// at a corner the value computed at the periodic image: corner_face below.)
constexpr int CORNER_F = 4;        // u, v, h and the tracer b of the work arrays
constexpr int CORNER_R = 4;        // rows from each wall
constexpr int CORNER_C = 6;        // columns: x = 0, 1, 2 and Nx-3, Nx-2, Nx-1
enum { CF_U, CF_V, CF_H, CF_B };

__host__ __device__ inline size_t corner_elems(int L) {
  return (size_t)CORNER_F * L * 2 * CORNER_R * CORNER_C;
}
// slot of field f, layer k, wall side (0 south, 1 north), row r from that wall, column c
__host__ __device__ inline size_t corner_slot(int f, int k, int L, int side, int r, int c) {
  return ((((size_t)f * L + k) * 2 + side) * CORNER_R + r) * CORNER_C + c;
}
// owned source position of a slot
__host__ __device__ inline int corner_x(int c, int Nx) { return c < 3 ? c : Nx - CORNER_C + c; }
__host__ __device__ inline int corner_y(int side, int r, int Ny) { return side == 0 ? r : Ny - 1 - r; }
// is raw (x, y) a corner ghost (x outside [0, Nx) and y outside [0, Ny))
__host__ __device__ inline bool is_corner(int x, int y, int Nx, int Ny) {
  return (x < 0 || x >= Nx) && (y < 0 || y >= Ny);
}
// the value of a corner ghost (x within 3 columns, y within 3 rows of the grid) of field f,
// layer k; kind_y is the field's wall kind along y (MAP_S, or MAP_N for v)
__host__ __device__ inline double corner_load(const double* buf, int f, int k, int L, int x, int y, int Nx, int Ny,
                                              int kind_y) {
  const int xs = wrap_index(x, Nx);
  const int c = xs < 3 ? xs : xs - Nx + CORNER_C;
  if (kind_y == MAP_N) {
    if (y == Ny) return -0.0;                          // the north wall face
    if (y < 0) return -buf[corner_slot(f, k, L, 0, -y, c)];
    return -buf[corner_slot(f, k, L, 1, y - Ny - 1, c)];
  }
  if (y < 0) return buf[corner_slot(f, k, L, 0, -y - 1, c)];
  return buf[corner_slot(f, k, L, 1, y - Ny, c)];
}

// The face thickness h_west (west) or h_south of one layer at a corner ghost (x, y) of an
// x-periodic, y-walled grid in the serial build: calc_face_thickness_layer (work.c:566-684)
// evaluates its formula over the ghosted array, then the fill copies into the corner the value
// at the periodic image (wrap(x), y), computed from the work copy of h whose own corner ghosts
// hold the previous fill (the shadow `sh`). uv is the layer's u (west) or v, read for the sign
// of the upwind schemes. ts: 0 AL81, 1 HK83, 2 UP3, 3 KT00 (the same expression order as the
// tile kernels' face_west / face_south). At an owned (x, y) it is the cell's own face thickness
// with the corner ghosts of its stencil taken from the shadow.
__device__ inline double corner_minmod3(double a, double b, double c) {
  if ((a > 0) && (b > 0) && (c > 0)) return fmin(a, fmin(b, c));
  if ((a < 0) && (b < 0) && (c < 0)) return fmax(a, fmax(b, c));
  return 0;
}
template <bool WEST>
__device__ inline double corner_face(const double* h, const double* uv, int pitch, int Nx, int Ny, int ts, double sig,
                                     const double* sh, int k, int L, int x, int y) {
  const int i = wrap_index(x, Nx), j = y;
  auto H = [&](int a, int b) {
    if (is_corner(a, b, Nx, Ny)) return corner_load(sh, CF_H, k, L, a, b, Nx, Ny, MAP_S);
    return load_mapped(h, pitch, a, b, Nx, Ny, false, true, MAP_S, MAP_S);
  };
  if (WEST) {
    if (ts == 1)
      return (1.0 / 3) * (H(i, j) + H(i - 1, j) + 0.25 * (H(i, j + 1) + H(i - 1, j + 1) + H(i, j - 1) + H(i - 1, j - 1)));
    if (ts == 2 || ts == 3) {
      const double uc = load_mapped(uv, pitch, i, j, Nx, Ny, false, true, MAP_N, MAP_S);
      if (ts == 2) {
        const double d2m = H(i, j) - 2 * H(i - 1, j) + H(i - 2, j);
        const double d2c = H(i + 1, j) - 2 * H(i, j) + H(i - 1, j);
        return 0.5 * (H(i, j) + H(i - 1, j)) - (1 / 6.0) * ((uc > 0) ? d2m : d2c);
      }
      const double dm = corner_minmod3(sig * (H(i, j) - H(i - 1, j)), 0.5 * (H(i, j) - H(i - 2, j)),
                                       sig * (H(i - 1, j) - H(i - 2, j)));
      const double dc = corner_minmod3(sig * (H(i + 1, j) - H(i, j)), 0.5 * (H(i + 1, j) - H(i - 1, j)),
                                       sig * (H(i, j) - H(i - 1, j)));
      const double xm = H(i - 1, j) + 0.5 * dm;
      const double xp = H(i, j) - 0.5 * dc;
      return (uc > 0) ? xm : xp;
    }
    return 0.5 * (H(i, j) + H(i - 1, j));
  }
  if (ts == 1)
    return (1.0 / 3) * (H(i, j) + H(i, j - 1) + 0.25 * (H(i + 1, j) + H(i - 1, j) + H(i + 1, j - 1) + H(i - 1, j - 1)));
  if (ts == 2 || ts == 3) {
    const double vc = load_mapped(uv, pitch, i, j, Nx, Ny, false, true, MAP_S, MAP_N);
    if (ts == 2) {
      const double d2m = H(i, j) - 2 * H(i, j - 1) + H(i, j - 2);
      const double d2c = H(i, j + 1) - 2 * H(i, j) + H(i, j - 1);
      return 0.5 * (H(i, j) + H(i, j - 1)) - (1 / 6.0) * ((vc > 0) ? d2m : d2c);
    }
    const double dm = corner_minmod3(sig * (H(i, j) - H(i, j - 1)), 0.5 * (H(i, j) - H(i, j - 2)),
                                     sig * (H(i, j - 1) - H(i, j - 2)));
    const double dc = corner_minmod3(sig * (H(i, j + 1) - H(i, j)), 0.5 * (H(i, j + 1) - H(i, j - 1)),
                                     sig * (H(i, j) - H(i, j - 1)));
    const double ym = H(i, j - 1) + 0.5 * dm;
    const double yp = H(i, j) + 0.5 * dc;
    return (vc > 0) ? ym : yp;
  }
  return 0.5 * (H(i, j) + H(i, j - 1));
}

// x / d rounded to nearest, given r = 1/d rounded to nearest. Markstein's theorem: when q
// is within one ulp of x/d and r is the correctly rounded reciprocal, the remainder
// x - q*d is exact and q + (x - q*d)*r rounds to x/d. The first correction makes q = x*r
// faithful, the second rounds it. Zeros keep their sign; tiny, huge and non-finite
// operands take the IEEE division. The range test reads the biased exponent of x from its
// high word (integer instructions): 2^-899 <= |x| < 2^900, exponents 124..1922, take the
// corrections. Checked against the hardware division bit for bit by
// pawsim_gpu_check_division (tests/test_gpu_division.py).
__device__ __forceinline__ double div_rn(double x, double d, double r) {
  double q = x * r;
  const unsigned be = ((unsigned)__double2hiint(x) >> 20) & 0x7ffu;
  if (be - 124u > 1922u - 124u) return (x == 0) ? q : x / d;
  double e = fma(-q, d, x);
  q = fma(e, r, q);
  e = fma(-q, d, x);
  return fma(e, r, q);
}

// div_rn without a branch, for the fast path of a tile: the same corrections applied to every
// operand, zeros keeping their sign by a select. An operand outside the corrections' range
// (tiny, huge, infinite or NaN) raises `oor`; the caller then recomputes what used the quotient
// with div_rn, so every result still equals the IEEE division's.
__device__ __forceinline__ double div_rn_fast(double x, double d, double r, bool& oor) {
  // the exponent field outside [124, 1922], tested on the high word without extracting it:
  // |hi| < 124 << 20 or |hi| >= 1923 << 20
  const unsigned ahi = (unsigned)__double2hiint(x) & 0x7fffffffu;
  oor |= (ahi - (124u << 20) > (1923u << 20) - 1u - (124u << 20)) & (x != 0);
  const double q = x * r;
  double e = fma(-q, d, x);
  const double q1 = fma(e, r, q);
  e = fma(-q1, d, x);
  const double res = fma(e, r, q1);
  return (x == 0) ? q : res;
}

}  // namespace pawsim

#define PAWSIM_CUDA_OK(call)                                     \
  do {                                                           \
    cudaError_t _e = (call);                                     \
    if (_e != cudaSuccess) return ::pawsim::set_cuda_error(_e, #call, __FILE__, __LINE__); \
  } while (0)

namespace pawsim {
int set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
// kernels launched by this library since load (reported by pawsim_gpu_launch_count); atomic
// because entry points without a model handle may be called from several host threads
extern std::atomic<long long> g_launches;
}
