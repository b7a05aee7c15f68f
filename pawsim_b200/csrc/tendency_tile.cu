// tendency_tile.cu -- fused layer tendency + Adams-Bashforth step (the K-tend kernel).
//
// Compiled for three tile heights, PAWSIM_TEND_TY = 8, 12 and 16 (256, 384 and 512 threads):
// a taller tile computes fewer halo cells per owned cell but needs more shared memory, and
// tendency.cu picks the height by how many CTAs then share an SM.
//
// One CTA owns a TX x TY tile of cells for every layer. It replaces, for that tile, the
// reference's whole derivative evaluation and state update:
//   model_code/tendency.c:81-115 (pawsim_tendency_eval) with the stages of work.c
//   (face thickness :566-684, eta :1173-1203, PV :1231-1288, PV coefficients :1294-1404,
//   Bernoulli :1410-1512, momentum :1520-1857, thickness :1864-1941), restoring.c:29-220,
//   diapycnal.c:72-291, forcing.c:30-395, and the AB1/AB2/AB3 update of
//   integrator.c:15-198, plus the rigid-lid column correction of pressure.c:525-561.
// Every intermediate lives in shared memory over exactly the region later stages read.
// The halo exchanges of field.c become index maps at load time (common.cuh), and each
// derived field is evaluated either directly at a ghost position (fields the reference
// computes over its ghost ring) or at the mirrored owned position (fields the reference
// re-fills after computing them), so results equal the reference's bit for bit. This
// file is compiled with -fmad=false: no multiply-add is contracted, as in the reference's
// x86-64 build.
#include "common.cuh"
#include "tendency.cuh"

namespace pawsim {

namespace {

#ifndef PAWSIM_TEND_TY
#define PAWSIM_TEND_TY 8
#endif
// PAWSIM_TEND_BUD = 1 builds the budget variant (every enabled budget family accumulated)
#ifndef PAWSIM_TEND_BUD
#define PAWSIM_TEND_BUD 0
#endif
constexpr bool BUD = PAWSIM_TEND_BUD != 0;
constexpr int TX = 32;
constexpr int TY = PAWSIM_TEND_TY;
constexpr int NT = TX * TY;
// tile halo: 2 cells cover TW81 + A2 + A4; the upwind thickness schemes (UP3, KT00) and the
// Smagorinsky biharmonic coefficient reach one cell further
template <int H>
struct Geo {
  static constexpr int RW = TX + 2 * H, RH = TY + 2 * H, RN = RW * RH;
};
enum { F_U, F_V, F_H, F_HW, F_HS, F_QQ, F_HQ, F_KE, F_HUU, F_HVV, F_DT, F_DS, F_U4, F_V4, F_NUM };
// Smagorinsky coefficients (allocated only when used): A2 and sqrt(A4) at cells and q points
enum { S_A2H, S_A2Q, S_A4H, S_A4Q, S_NUM };

template <int HALO>
struct Tile {
  int X0, Y0;
  int Nx, Ny;
  bool wx, wy;
  // raw coordinate of local index
  __device__ int gx(int lx) const { return X0 - HALO + lx; }
  __device__ int gy(int ly) const { return Y0 - HALO + ly; }
  // raw position within the band that owned cells can reach (mirrors stay in the tile)
  __device__ bool near(int lx, int ly) const {
    int x = gx(lx), y = gy(ly);
    return x >= -HALO && x < Nx + HALO && y >= -HALO && y < Ny + HALO;
  }
  // local index of the owned cell that a filled (mirror-symmetric) field copies at raw x
  __device__ int mlx(int lx) const {
    if (!wx) return lx;
    int g = gx(lx);
    if (g < 0) g = -g - 1;
    else if (g >= Nx) g = 2 * Nx - g - 1;
    return g - X0 + HALO;
  }
  __device__ int mly(int ly) const {
    if (!wy) return ly;
    int g = gy(ly);
    if (g < 0) g = -g - 1;
    else if (g >= Ny) g = 2 * Ny - g - 1;
    return g - Y0 + HALO;
  }
};

// tile accessor; RW is the row length of the instantiation in scope
#define AT(arr, lx, ly) (arr)[(ly) * RW + (lx)]

__device__ inline double sq(double x) { return x * x; }

// PV interpolation coefficients (work.c:1294-1404) evaluated from qq in shared memory
template <int MS, int RW, typename DV> struct Coef {
  const double* q;
  double r24;
  DV div;   // the quotient x / d given 1/d (div_rn, or its branch-free pass)
  __device__ double D(double x) const { return div(x, 24.0, r24); }
  __device__ double Q(int x, int y) const { return AT(q, x, y); }
  __device__ double alpha(int i, int j) const {
    if (MS == 3)
      return D(2 * Q(i + 1, j + 1) + 3 * Q(i, j + 1) + 2 * Q(i, j) + Q(i + 1, j) - Q(i, j + 2) - Q(i - 1, j + 1));
    return D(2 * Q(i + 1, j + 1) + Q(i, j + 1) + 2 * Q(i, j) + Q(i + 1, j));
  }
  __device__ double beta(int i, int j) const {
    if (MS == 3)
      return D(3 * Q(i, j + 1) + 2 * Q(i - 1, j + 1) + Q(i - 1, j) + 2 * Q(i, j) - Q(i + 1, j + 1) - Q(i, j + 2));
    return D(Q(i, j + 1) + 2 * Q(i - 1, j + 1) + Q(i - 1, j) + 2 * Q(i, j));
  }
  __device__ double gamma(int i, int j) const {
    if (MS == 3)
      return D(2 * Q(i, j + 1) + Q(i - 1, j + 1) + 2 * Q(i - 1, j) + 3 * Q(i, j) - Q(i, j - 1) - Q(i + 1, j));
    return D(2 * Q(i, j + 1) + Q(i - 1, j + 1) + 2 * Q(i - 1, j) + Q(i, j));
  }
  __device__ double delta(int i, int j) const {
    if (MS == 3)
      return D(Q(i + 1, j + 1) + 2 * Q(i, j + 1) + 3 * Q(i, j) + 2 * Q(i + 1, j) - Q(i - 1, j) - Q(i, j - 1));
    return D(Q(i + 1, j + 1) + 2 * Q(i, j + 1) + Q(i, j) + 2 * Q(i + 1, j));
  }
  __device__ double epsilon(int i, int j) const {
    return D(Q(i + 1, j + 1) + Q(i, j + 1) - Q(i, j) - Q(i + 1, j));
  }
  __device__ double phi(int i, int j) const {
    return D(-Q(i + 1, j + 1) + Q(i, j + 1) + Q(i, j) - Q(i + 1, j));
  }
  __device__ double lambda(int i, int j) const { return D(Q(i + 1, j) - Q(i - 1, j)); }
  __device__ double mu(int i, int j) const { return D(Q(i, j - 1) - Q(i, j + 1)); }
};

__device__ inline double minmod3(double a, double b, double c) {
  // defs.c:1000-1014: zero unless all three share a sign, else the smallest magnitude
  if ((a > 0) && (b > 0) && (c > 0)) return fmin(a, fmin(b, c));
  if ((a < 0) && (b < 0) && (c < 0)) return fmax(a, fmax(b, c));
  return 0;
}

// face thickness of one layer at a local position (work.c:566-684): AL81 centred mean, HK83
// weighted mean, UP3 mean minus a sixth of the upwind second difference, KT00 limited
// reconstruction from the upwind side (the velocity's sign is read at the face)
template <int TS, int RW>
__device__ inline double face_west(const double* h, const double* u, double sig, int i, int j) {
  if (TS == 1)
    return (1.0 / 3) * (AT(h, i, j) + AT(h, i - 1, j)
                        + 0.25 * (AT(h, i, j + 1) + AT(h, i - 1, j + 1) + AT(h, i, j - 1) + AT(h, i - 1, j - 1)));
  if (TS == 2) {
    const double d2m = AT(h, i, j) - 2 * AT(h, i - 1, j) + AT(h, i - 2, j);
    const double d2c = AT(h, i + 1, j) - 2 * AT(h, i, j) + AT(h, i - 1, j);
    return 0.5 * (AT(h, i, j) + AT(h, i - 1, j)) - (1 / 6.0) * ((AT(u, i, j) > 0) ? d2m : d2c);
  }
  if (TS == 3) {
    const double dm = minmod3(sig * (AT(h, i, j) - AT(h, i - 1, j)), 0.5 * (AT(h, i, j) - AT(h, i - 2, j)),
                              sig * (AT(h, i - 1, j) - AT(h, i - 2, j)));
    const double dc = minmod3(sig * (AT(h, i + 1, j) - AT(h, i, j)), 0.5 * (AT(h, i + 1, j) - AT(h, i - 1, j)),
                              sig * (AT(h, i, j) - AT(h, i - 1, j)));
    const double xm = AT(h, i - 1, j) + 0.5 * dm;
    const double xp = AT(h, i, j) - 0.5 * dc;
    return (AT(u, i, j) > 0) ? xm : xp;
  }
  return 0.5 * (AT(h, i, j) + AT(h, i - 1, j));
}
template <int TS, int RW>
__device__ inline double face_south(const double* h, const double* v, double sig, int i, int j) {
  if (TS == 1)
    return (1.0 / 3) * (AT(h, i, j) + AT(h, i, j - 1)
                        + 0.25 * (AT(h, i + 1, j) + AT(h, i - 1, j) + AT(h, i + 1, j - 1) + AT(h, i - 1, j - 1)));
  if (TS == 2) {
    const double d2m = AT(h, i, j) - 2 * AT(h, i, j - 1) + AT(h, i, j - 2);
    const double d2c = AT(h, i, j + 1) - 2 * AT(h, i, j) + AT(h, i, j - 1);
    return 0.5 * (AT(h, i, j) + AT(h, i, j - 1)) - (1 / 6.0) * ((AT(v, i, j) > 0) ? d2m : d2c);
  }
  if (TS == 3) {
    const double dm = minmod3(sig * (AT(h, i, j) - AT(h, i, j - 1)), 0.5 * (AT(h, i, j) - AT(h, i, j - 2)),
                              sig * (AT(h, i, j - 1) - AT(h, i, j - 2)));
    const double dc = minmod3(sig * (AT(h, i, j + 1) - AT(h, i, j)), 0.5 * (AT(h, i, j + 1) - AT(h, i, j - 1)),
                              sig * (AT(h, i, j) - AT(h, i, j - 1)));
    const double ym = AT(h, i, j - 1) + 0.5 * dm;
    const double yp = AT(h, i, j) + 0.5 * dc;   // the reference adds the half slope on this side too
    return (AT(v, i, j) > 0) ? ym : yp;
  }
  return 0.5 * (AT(h, i, j) + AT(h, i, j - 1));
}

// kinetic energy of the Bernoulli function (work.c:1437-1499); U(a, b), V(a, b) read the
// layer's velocities
template <int MS, typename UF, typename VF>
__device__ inline double kinetic_f(UF U, VF V, int i, int j) {
  if (MS == 1) {
    return (sq(U(i + 1, j)) + sq(U(i, j))
            + 0.25 * (sq(U(i + 1, j + 1)) + sq(U(i, j + 1)) + sq(U(i + 1, j - 1)) + sq(U(i, j - 1)))
            + sq(V(i, j + 1)) + sq(V(i, j))
            + 0.25 * (sq(V(i + 1, j + 1)) + sq(V(i + 1, j)) + sq(V(i - 1, j + 1)) + sq(V(i - 1, j)))) / 6;
  }
  if (MS == 3) {
    return 0.25 * ((2.0 / 3.0) * sq(U(i, j))
                   + (1.0 / 3.0) * sq(0.5 * (U(i - 1, j) + U(i + 1, j)))
                   + (2.0 / 3.0) * sq(U(i + 1, j))
                   + (1.0 / 3.0) * sq(0.5 * (U(i, j) + U(i + 2, j)))
                   + (2.0 / 3.0) * sq(V(i, j))
                   + (1.0 / 3.0) * sq(0.5 * (V(i, j - 1) + V(i, j + 1)))
                   + (2.0 / 3.0) * sq(V(i, j + 1))
                   + (1.0 / 3.0) * sq(0.5 * (V(i, j) + V(i, j + 2))));
  }
  return (sq(U(i + 1, j)) + sq(U(i, j))) / 4 + (sq(V(i, j + 1)) + sq(V(i, j))) / 4;
}
template <int MS, int RW>
__device__ inline double kinetic(const double* u, const double* v, int i, int j) {
  return kinetic_f<MS>([&](int a, int b) { return AT(u, a, b); }, [&](int a, int b) { return AT(v, a, b); }, i, j);
}
// The work arrays u, v, h of one layer as the serial build holds them around a periodic image
// column (x-periodic, y-walled grids): the copied values, except the corner ghosts relative to
// that column, which come from the corner shadow. A field the reference computes and then
// copies into the seam's ghost columns by its periodic exchange is evaluated with these at the
// image column wrap(x) (field.c:353-427; common.cuh).
struct ImageW {
  const double *u, *v, *h, *sh;
  int pitch, Nx, Ny, k, L;
  __device__ double U(int a, int b) const {
    return is_corner(a, b, Nx, Ny) ? corner_load(sh, CF_U, k, L, a, b, Nx, Ny, MAP_S)
                                   : load_mapped(u, pitch, a, b, Nx, Ny, false, true, MAP_N, MAP_S);
  }
  __device__ double V(int a, int b) const {
    return is_corner(a, b, Nx, Ny) ? corner_load(sh, CF_V, k, L, a, b, Nx, Ny, MAP_N)
                                   : load_mapped(v, pitch, a, b, Nx, Ny, false, true, MAP_S, MAP_N);
  }
  __device__ double H(int a, int b) const {
    return is_corner(a, b, Nx, Ny) ? corner_load(sh, CF_H, k, L, a, b, Nx, Ny, MAP_S)
                                   : load_mapped(h, pitch, a, b, Nx, Ny, false, true, MAP_S, MAP_S);
  }
};

// the same at raw (x, y) of the serial build's work arrays on an x-periodic, y-walled grid,
// evaluated at the periodic image of x, with the corner ghosts of the stencil from the shadow
// (the value the fill copies into a periodic ghost column, common.cuh)
template <int MS>
__device__ inline double kinetic_image(const double* uk, const double* vk, int pitch, int Nx, int Ny, const double* sh,
                                       int k, int L, int x, int y) {
  auto U = [&](int a, int b) {
    if (is_corner(a, b, Nx, Ny)) return corner_load(sh, CF_U, k, L, a, b, Nx, Ny, MAP_S);
    return load_mapped(uk, pitch, a, b, Nx, Ny, false, true, MAP_N, MAP_S);
  };
  auto V = [&](int a, int b) {
    if (is_corner(a, b, Nx, Ny)) return corner_load(sh, CF_V, k, L, a, b, Nx, Ny, MAP_N);
    return load_mapped(vk, pitch, a, b, Nx, Ny, false, true, MAP_S, MAP_N);
  };
  return kinetic_f<MS>(U, V, wrap_index(x, Nx), y);
}

__device__ inline double gload(const double* f, const TendParams& p, int gi, int gj, int kx, int ky) {
  return load_mapped(f, p.pitch, gi, gj, p.Nx, p.Ny, p.wall_ew, p.wall_ns, kx, ky);
}

// hz = h (eta_k + eta_k+1) / 2 of layer k at raw (x, y) (work.c:205-208), interface heights
// built upward from the bottom as work.c:1184-1199 does; ghost positions through the maps
__device__ inline double buoy_hz(const TendParams& p, int k, int x, int y) {
  double e1 = gload(p.hhb, p, x, y, MAP_S, MAP_S);
  for (int m = p.L - 1; m > k; --m) e1 = e1 + gload(p.h + m * p.lstride, p, x, y, MAP_S, MAP_S);
  const double hk = gload(p.h + k * p.lstride, p, x, y, MAP_S, MAP_S);
  const double e0 = e1 + hk;
  return hk * 0.5 * (e0 + e1);
}

// face thickness of a layer at an owned cell, read from global memory (h, u, v of that layer;
// ghost positions through the scalar / velocity maps)
template <int TS>
__device__ inline double gface_west(const TendParams& p, const double* h, const double* u, int i, int j) {
  auto H = [&](int a, int b) { return gload(h, p, a, b, MAP_S, MAP_S); };
  if (TS == 1)
    return (1.0 / 3) * (H(i, j) + H(i - 1, j) + 0.25 * (H(i, j + 1) + H(i - 1, j + 1) + H(i, j - 1) + H(i - 1, j - 1)));
  if (TS == 2 || TS == 3) {
    const double uc = gload(u, p, i, j, MAP_N, MAP_S);
    if (TS == 2) {
      const double d2m = H(i, j) - 2 * H(i - 1, j) + H(i - 2, j);
      const double d2c = H(i + 1, j) - 2 * H(i, j) + H(i - 1, j);
      return 0.5 * (H(i, j) + H(i - 1, j)) - (1 / 6.0) * ((uc > 0) ? d2m : d2c);
    }
    const double sg = p.kt00_sigma;
    const double dm = minmod3(sg * (H(i, j) - H(i - 1, j)), 0.5 * (H(i, j) - H(i - 2, j)), sg * (H(i - 1, j) - H(i - 2, j)));
    const double dc = minmod3(sg * (H(i + 1, j) - H(i, j)), 0.5 * (H(i + 1, j) - H(i - 1, j)), sg * (H(i, j) - H(i - 1, j)));
    return (uc > 0) ? H(i - 1, j) + 0.5 * dm : H(i, j) - 0.5 * dc;
  }
  return 0.5 * (H(i, j) + H(i - 1, j));
}
template <int TS>
__device__ inline double gface_south(const TendParams& p, const double* h, const double* v, int i, int j) {
  auto H = [&](int a, int b) { return gload(h, p, a, b, MAP_S, MAP_S); };
  if (TS == 1)
    return (1.0 / 3) * (H(i, j) + H(i, j - 1) + 0.25 * (H(i + 1, j) + H(i - 1, j) + H(i + 1, j - 1) + H(i - 1, j - 1)));
  if (TS == 2 || TS == 3) {
    const double vc = gload(v, p, i, j, MAP_S, MAP_N);
    if (TS == 2) {
      const double d2m = H(i, j) - 2 * H(i, j - 1) + H(i, j - 2);
      const double d2c = H(i, j + 1) - 2 * H(i, j) + H(i, j - 1);
      return 0.5 * (H(i, j) + H(i, j - 1)) - (1 / 6.0) * ((vc > 0) ? d2m : d2c);
    }
    const double sg = p.kt00_sigma;
    const double dm = minmod3(sg * (H(i, j) - H(i, j - 1)), 0.5 * (H(i, j) - H(i, j - 2)), sg * (H(i, j - 1) - H(i, j - 2)));
    const double dc = minmod3(sg * (H(i, j + 1) - H(i, j)), 0.5 * (H(i, j + 1) - H(i, j - 1)), sg * (H(i, j) - H(i, j - 1)));
    return (vc > 0) ? H(i, j - 1) + 0.5 * dm : H(i, j) + 0.5 * dc;
  }
  return 0.5 * (H(i, j) + H(i, j - 1));
}

// face thickness of layer k at an owned cell from global memory; on x-periodic, y-walled grids
// with the serial build's corners the stencil's corner ghosts come from the corner shadow
template <int TS>
__device__ inline double face_west_cell(const TendParams& p, int k, int i, int j) {
  if (p.corners)
    return corner_face<true>(p.h + k * p.lstride, p.u + k * p.lstride, p.pitch, p.Nx, p.Ny, TS, p.kt00_sigma,
                             p.corners, k, p.L, i, j);
  return gface_west<TS>(p, p.h + k * p.lstride, p.u + k * p.lstride, i, j);
}
template <int TS>
__device__ inline double face_south_cell(const TendParams& p, int k, int i, int j) {
  if (p.corners)
    return corner_face<false>(p.h + k * p.lstride, p.v + k * p.lstride, p.pitch, p.Nx, p.Ny, TS, p.kt00_sigma,
                              p.corners, k, p.L, i, j);
  return gface_south<TS>(p, p.h + k * p.lstride, p.v + k * p.lstride, i, j);
}

// Surface and bottom layer fractions of every layer at owned cell (gi, gj) (work.c:2151-2340):
// out(f, k, value) receives f = 0 hFsurf_west, 1 hFsurf_south, 2 hFbot_west, 3 hFbot_south,
// zeros included. hsml <= 0 puts the whole surface forcing in the top layer, hbbl <= 0 the
// whole bottom forcing in the bottom layer.
template <int TS, typename Out>
__device__ inline void cell_fractions(const TendParams& p, int gi, int gj, Out out) {
  const int L = p.L;
  double hwk[LMAX], hsk[LMAX];
  for (int k = 0; k < L; ++k) {
    hwk[k] = face_west_cell<TS>(p, k, gi, gj);
    hsk[k] = face_south_cell<TS>(p, k, gi, gj);
  }
  for (int f = 0; f < 4; ++f)
    for (int k = 0; k < L; ++k) out(f, k, 0.0);
  if (p.hsml <= 0) {
    out(0, 0, 1.0);
    out(1, 0, 1.0);
  } else {
    const double hsw = 0.5 * (gload(p.hhs, p, gi, gj, MAP_S, MAP_S) + gload(p.hhs, p, gi - 1, gj, MAP_S, MAP_S));
    const double hss = 0.5 * (gload(p.hhs, p, gi, gj, MAP_S, MAP_S) + gload(p.hhs, p, gi, gj - 1, MAP_S, MAP_S));
    double zw = hsw - p.hsml, zs = hss - p.hsml, ew = hsw, es = hss, sw = 0, ss = 0;
    for (int k = 0; k < L; ++k) {
      const double ewl = ew - hwk[k], esl = es - hsk[k];
      if (sw < 1.0) {
        zw -= fmin(p.hmin_surf, hwk[k]);
        double he = fmax(ew, zw) - fmax(ewl, zw);
        he = fmax(he - p.hmin_surf, 0.0);
        const double fr = he / p.hsml;
        out(0, k, fr);
        sw += fr;
      }
      if (ss < 1.0) {
        zs -= fmin(p.hmin_surf, hsk[k]);
        double he = fmax(es, zs) - fmax(esl, zs);
        he = fmax(he - p.hmin_surf, 0.0);
        const double fr = he / p.hsml;
        out(1, k, fr);
        ss += fr;
      }
      ew = ewl;
      es = esl;
    }
  }
  if (p.hbbl <= 0) {
    out(2, L - 1, 1.0);
    out(3, L - 1, 1.0);
  } else {
    const double hbw = 0.5 * (gload(p.hhb, p, gi, gj, MAP_S, MAP_S) + gload(p.hhb, p, gi - 1, gj, MAP_S, MAP_S));
    const double hbs = 0.5 * (gload(p.hhb, p, gi, gj, MAP_S, MAP_S) + gload(p.hhb, p, gi, gj - 1, MAP_S, MAP_S));
    double zw = hbw + p.hbbl, zs = hbs + p.hbbl, ewl = hbw, esl = hbs, sw = 0, ss = 0;
    for (int k = L; k > 0; --k) {
      const int kk = k - 1;
      const double ewu = ewl + hwk[kk], esu = esl + hsk[kk];
      if (sw < 1.0) {
        zw += fmin(p.hmin_bot, hwk[kk]);
        double he = fmin(ewu, zw) - fmin(ewl, zw);
        he = fmax(he - p.hmin_bot, 0.0);
        const double fr = he / p.hbbl;
        out(2, kk, fr);
        sw += fr;
      }
      if (ss < 1.0) {
        zs += fmin(p.hmin_bot, hsk[kk]);
        double he = fmin(esu, zs) - fmin(esl, zs);
        he = fmax(he - p.hmin_bot, 0.0);
        const double fr = he / p.hbbl;
        out(3, kk, fr);
        ss += fr;
      }
      ewl = ewu;
      esl = esu;
    }
  }
}

// Pre-pass of the quadratic drags whose boundary layer spreads over several layers
// (forcing.c:95-143, 181-223): at every owned cell the fraction-weighted sums of the layer
// velocities, u_bot = sum_k u_k hFbot_west_k and v_bot (hbbl > 0), u_surf and v_surf (hsml > 0),
// in layer order from zero as the reference sums them. Planes of p.dragv: 0 u_bot, 1 v_bot,
// 2 u_surf, 3 v_surf.
template <int TS>
__global__ void drag_speed_kernel(const __grid_constant__ TendParams p) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  const int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= p.Nx || gj >= p.Ny) return;
  const size_t c = (size_t)gj * p.pitch + gi;
  double fr[4][LMAX];
  cell_fractions<TS>(p, gi, gj, [&](int f, int k, double v) { fr[f][k] = v; });
  double ub = 0, vb = 0, us = 0, vs = 0;
  for (int k = 0; k < p.L; ++k) {
    const size_t o = k * p.lstride + c;
    us += p.u[o] * fr[0][k];
    vs += p.v[o] * fr[1][k];
    ub += p.u[o] * fr[2][k];
    vb += p.v[o] * fr[3][k];
  }
  if (p.drag_bot) {
    p.dragv[c] = ub;
    p.dragv[p.lstride + c] = vb;
  }
  if (p.drag_surf) {
    p.dragv[2 * p.lstride + c] = us;
    p.dragv[3 * p.lstride + c] = vs;
  }
}

// a drag velocity plane at raw (x, y): a product of two fields of the same wall parity, so
// ghosts take the mirrored value without a sign change and the wall face holds +0
__device__ inline double drag_load(const double* f, const TendParams& p, int x, int y, int kx, int ky) {
  AxisMap ax = map_axis(x, p.Nx, p.wall_ew, kx);
  if (ax.zero) return 0.0;
  AxisMap ay = map_axis(y, p.Ny, p.wall_ns, ky);
  if (ay.zero) return 0.0;
  return f[(size_t)ay.idx * p.pitch + ax.idx];
}

// 64 registers per thread: four 256-thread or two 512-thread CTAs per SM
#ifndef PAWSIM_TEND_MINB
#define PAWSIM_TEND_MINB (1024 / NT)
#endif

// One tile (bx, by) of the fused step; the fused kernel runs one per CTA, the exact pass the
// tiles listed by it.
// an L2 prefetch of the line holding *ptr (no register result, nothing to wait for)
__device__ __forceinline__ void prefetch_l2(const void* ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

template <int MS, int TS, int H, bool LEAN, bool EXACT>
__device__ __forceinline__ void tendency_tile(const TendParams& p, int bx, int by) {
  // LEAN instantiations serve set-ups without w_dia, Smagorinsky, layer fractions, restoring,
  // diapycnal viscosity, surface or quadratic drag, Fbaro, biharmonic viscosity and corner
  // shadow: those paths compile away
  const bool use_wdia = !LEAN && p.use_wdia, use_relax = !LEAN && p.use_relax;
  const bool use_diavisc = !LEAN && p.use_diavisc, use_fractions = !LEAN && p.use_fractions;
  const bool use_fbaro = !LEAN && p.use_fbaro, useA4 = !LEAN && p.useA4;
  const int use_smag = LEAN ? 0 : p.use_smag;
  const double* const corners = LEAN ? nullptr : p.corners;
  // Stencil quotients. The plain build's first pass divides without a branch (div_rn_fast) and
  // flags its tile when an operand fell outside the corrections' range; the EXACT pass then
  // recomputes only the flagged tiles with div_rn (the budget build always uses div_rn, as it
  // adds to running sums on the way).
  constexpr bool SLOWDIV = EXACT || BUD;
  bool oor = false;
  auto DIV = [&](double x, double d, double r) {
    if constexpr (SLOWDIV) return div_rn(x, d, r);
    else return div_rn_fast(x, d, r, oor);
  };
  constexpr int RW = Geo<H>::RW, RH = Geo<H>::RH, RN = Geo<H>::RN;
  extern __shared__ double smem[];
  // the lean build has no biharmonic intermediates (U4, V4): their planes are not allocated
  constexpr int FP = LEAN ? F_U4 : F_NUM;
  double* F[F_NUM];
#pragma unroll
  for (int f = 0; f < F_NUM; ++f) F[f] = smem + (f < FP ? f : 0) * RN;
  double* MMall = smem + FP * RN;               // [L][RN]
  double* WDall = MMall + p.L * RN;             // [L+1][RN] when use_wdia
  double* SM = WDall + (use_wdia ? (p.L + 1) * RN : 0);   // [S_NUM][RN] when use_smag
  double* FR = SM + (use_smag ? S_NUM * RN : 0);          // [4][L][NT] when use_fractions

  const int tid = threadIdx.x;
  Tile<H> t;
  t.X0 = bx * TX;
  t.Y0 = by * TY;
  t.Nx = p.Nx;
  t.Ny = p.Ny;
  t.wx = p.wall_ew;
  t.wy = p.wall_ns;
  const int L = p.L;
  const double dx = p.dx, dy = p.dy, rdx = p.rdx, rdy = p.rdy, r24 = p.r24;
  // tiles whose halo lies inside the domain read global memory without boundary maps
  const bool inner = t.X0 - H >= 0 && t.X0 + TX + H <= p.Nx && t.Y0 - H >= 0 && t.Y0 + TY + H <= p.Ny;

  if (!EXACT) {
    // the first layer's velocities at this thread's cell, read after the column prologue
    const int gi0 = t.X0 + tid % TX, gj0 = t.Y0 + tid / TX;
    if (gi0 < p.Nx && gj0 < p.Ny) {
      const size_t c0 = (size_t)gj0 * p.pitch + gi0;
      prefetch_l2(p.u + c0);
      prefetch_l2(p.v + c0);
    }
  }
  // ---- column prologue over the Bernoulli region: eta, pp, Montgomery MM, wdia ----
  for (int q = tid; q < RN; q += NT) {
    int lx = q % RW, ly = q / RW;
    if (lx < H - 1 || lx > TX + H - 1 || ly < H - 1 || ly > TY + H - 1) continue;
    if (!t.near(lx, ly)) {
      for (int k = 0; k < L; ++k) MMall[k * RN + q] = 0;
      if (use_wdia)
        for (int k = 0; k <= L; ++k) WDall[k * RN + q] = 0;
      continue;
    }
    int gi = t.gx(lx), gj = t.gy(ly);
    // the layer loops run over the LMAX bound with a guard, so the per-layer arrays stay
    // in registers
    double hk[LMAX], eta[LMAX];
    const size_t gc = (size_t)gj * p.pitch + gi;
    double hb = inner ? p.hhb[gc] : gload(p.hhb, p, gi, gj, MAP_S, MAP_S);
    double e_acc = hb;
#pragma unroll
    for (int k = LMAX - 1; k >= 0; --k) {
      if (k < L) {
        hk[k] = inner ? p.h[k * p.lstride + gc] : gload(p.h + k * p.lstride, p, gi, gj, MAP_S, MAP_S);
        e_acc = e_acc + hk[k];
        eta[k] = e_acc;
      }
    }
    double pp = 0;
    double bprev = 0;   // tracer of the layer above (buoyancy build)
#pragma unroll
    for (int k = 0; k < LMAX; ++k) {
      if (k < L) {
        if (k == 0) pp = p.use_rl ? 0 : p.gg[0] * eta[0];
        else pp = pp + p.gg[k] * eta[k];
        if constexpr (BUD) {
          // the buoyancy anomaly in the Bernoulli pressure (work.c:1438-1452)
          if (p.use_buoy) {
            const double bk = inner ? p.b[k * p.lstride + gc] : gload(p.b + k * p.lstride, p, gi, gj, MAP_S, MAP_S);
            if (k == 0) {
              if (!p.use_rl) pp -= bk * eta[0];
            } else {
              pp += eta[k] * (bprev - bk);
            }
            bprev = bk;
          }
        }
        double mm = pp;
        if (p.h0 != 0) {
          double h0 = p.h0, hc = hk[k];
          mm -= p.geff[k] * (h0 * h0 * h0 * h0) / (hc * hc * hc) / 3;
        }
        MMall[k * RN + q] = mm;
      }
    }
    if (use_wdia) {
      double* wd = WDall + q;   // interface k at wd[k * RN]
      for (int k = 0; k <= L; ++k) {
        if (p.use_wdia_file) {
          wd[k * RN] = p.ww0 * gload(p.wd0 + k * p.lstride, p, gi, gj, MAP_S, MAP_S)
                     + p.ww1 * gload(p.wd1 + k * p.lstride, p, gi, gj, MAP_S, MAP_S);
        } else {
          wd[k * RN] = 0;
        }
      }
      if (use_relax) {
        double acc = 0;
        double ht = gload(p.hTime, p, gi, gj, MAP_S, MAP_S);
#pragma unroll
        for (int k = LMAX - 1; k >= 0; --k) {
          if (k < L) {
            if (ht > 0) {
              acc += (hk[k] - gload(p.hRelax + k * p.lstride, p, gi, gj, MAP_S, MAP_S)) / ht;
              wd[k * RN] += acc;
            }
            double et = gload(p.eTime + k * p.lstride, p, gi, gj, MAP_S, MAP_S);
            if (et > 0) wd[k * RN] += (eta[k] - gload(p.eRelax + k * p.lstride, p, gi, gj, MAP_S, MAP_S)) / et;
          }
        }
      }
      if (p.wdia_out && lx >= H && lx < H + TX && ly >= H && ly < H + TY && gi < p.Nx && gj < p.Ny) {
        for (int k = 0; k <= L; ++k) p.wdia_out[k * p.lstride + (size_t)gj * p.pitch + gi] = wd[k * RN];
      }
    }
  }

  // per-thread output cell
  const int tx = tid % TX, ty = tid / TX;
  const int ox = tx + H, oy = ty + H;
  const int gi = t.X0 + tx, gj = t.Y0 + ty;
  const bool valid = gi < p.Nx && gj < p.Ny;
  const size_t cell = (size_t)gj * p.pitch + gi;
  double htot = 0;   // sum of the new layer thicknesses, in layer order

  // ---- surface and bottom layer fractions at the owned cell (work.c:2151-2340) ----
  // FR[(f * L + k) * NT + tid], f = 0 hFsw, 1 hFss, 2 hFbw, 3 hFbs
  if (use_fractions && valid)
    cell_fractions<TS>(p, gi, gj, [&](int f, int k, double v) { FR[(f * L + k) * NT + tid] = v; });

  for (int k = 0; k < L; ++k) {
    const double* uk = p.u + k * p.lstride;
    const double* vk = p.v + k * p.lstride;
    const double* hkp = p.h + k * p.lstride;
    if (!EXACT && valid) {
      // this layer's AB history (read in the epilogue) and the next layer's state at this
      // thread's cell start towards L2 while the layer is computed
      const size_t o = k * p.lstride + cell;
      if (p.ab_mode >= 2) {
        prefetch_l2(p.f1u + o);
        prefetch_l2(p.f1v + o);
        prefetch_l2(p.f1h + o);
      }
      if (p.ab_mode >= 3) {
        prefetch_l2(p.f2u + o);
        prefetch_l2(p.f2v + o);
        prefetch_l2(p.f2h + o);
      }
      if (k + 1 < L) {
        prefetch_l2(p.u + o + p.lstride);
        prefetch_l2(p.v + o + p.lstride);
        prefetch_l2(p.h + o + p.lstride);
      }
    }
    __syncthreads();
    // ---- load the layer's u, v, h with the reference's ghost semantics ----
    if (inner) {
      for (int q = tid; q < RN; q += NT) {
        int lx = q % RW, ly = q / RW;
        size_t g = (size_t)t.gy(ly) * p.pitch + t.gx(lx);
        F[F_U][q] = uk[g];
        F[F_V][q] = vk[g];
        F[F_H][q] = hkp[g];
      }
    } else {
      for (int q = tid; q < RN; q += NT) {
        int lx = q % RW, ly = q / RW;
        int gx = t.gx(lx), gy = t.gy(ly);
        bool in = gx >= -H && gx < p.Nx + H && gy >= -H && gy < p.Ny + H;
        if (in && corners && is_corner(gx, gy, p.Nx, p.Ny)) {
          F[F_U][q] = corner_load(corners, CF_U, k, L, gx, gy, p.Nx, p.Ny, MAP_S);
          F[F_V][q] = corner_load(corners, CF_V, k, L, gx, gy, p.Nx, p.Ny, MAP_N);
          F[F_H][q] = corner_load(corners, CF_H, k, L, gx, gy, p.Nx, p.Ny, MAP_S);
          continue;
        }
        F[F_U][q] = in ? gload(uk, p, gx, gy, MAP_N, MAP_S) : 0.0;
        F[F_V][q] = in ? gload(vk, p, gx, gy, MAP_S, MAP_N) : 0.0;
        F[F_H][q] = in ? gload(hkp, p, gx, gy, MAP_S, MAP_S) : 0.0;
      }
    }
    __syncthreads();
    const double* su = F[F_U];
    const double* sv = F[F_V];
    const double* sh = F[F_H];
    // ---- face thickness, PV, kinetic energy, deformation rates ----
    for (int q = tid; q < RN; q += NT) {
      int lx = q % RW, ly = q / RW;
      const bool nr = t.near(lx, ly);
      if (lx >= H - 1 && lx <= TX + H && ly >= H - 1 && ly <= TY + H && nr) {
        // a periodic ghost column (its corners included) receives the values computed at the
        // image column, whose stencil reads the corner shadow (serial build, common.cuh)
        if (corners && !inner && (t.gx(lx) < 0 || t.gx(lx) >= p.Nx)) {
          F[F_HW][q] = corner_face<true>(hkp, uk, p.pitch, p.Nx, p.Ny, TS, p.kt00_sigma, corners, k, L, t.gx(lx),
                                         t.gy(ly));
          F[F_HS][q] = corner_face<false>(hkp, vk, p.pitch, p.Nx, p.Ny, TS, p.kt00_sigma, corners, k, L, t.gx(lx),
                                          t.gy(ly));
        } else {
          int mx = t.mlx(lx), my = t.mly(ly);
          F[F_HW][q] = face_west<TS, RW>(sh, su, p.kt00_sigma, mx, my);
          F[F_HS][q] = face_south<TS, RW>(sh, sv, p.kt00_sigma, mx, my);
        }
      }
      // at the seam's ghost columns (serial build's corners) zeta, h_q and q are periodic copies
      // of the image column's (work.c:1231-1288 then an internal exchange); the deformation
      // rates are computed in place over the ghosted arrays
      const bool seam = corners && !inner && (t.gx(lx) < 0 || t.gx(lx) >= p.Nx);
      const ImageW iw{uk, vk, hkp, corners, p.pitch, p.Nx, p.Ny, k, L};
      const int ix = wrap_index(t.gx(lx), p.Nx), iy = t.gy(ly);
      if (lx >= H - 1 && ly >= H - 1 && lx <= TX + H + 1 && ly <= TY + H + 1) {
        // zeta, h on the q grid and q itself (work.c:1261-1270)
        double z, hq;
        if (seam) {
          z = DIV(iw.U(ix, iy - 1) - iw.U(ix, iy), dy, rdy) + DIV(iw.V(ix, iy) - iw.V(ix - 1, iy), dx, rdx);
          hq = 0.25 * (iw.H(ix, iy) + iw.H(ix - 1, iy - 1) + iw.H(ix - 1, iy) + iw.H(ix, iy - 1));
        } else {
          z = DIV(AT(su, lx, ly - 1) - AT(su, lx, ly), dy, rdy) + DIV(AT(sv, lx, ly) - AT(sv, lx - 1, ly), dx, rdx);
          hq = 0.25 * (AT(sh, lx, ly) + AT(sh, lx - 1, ly - 1) + AT(sh, lx - 1, ly) + AT(sh, lx, ly - 1));
        }
        double om = inner ? p.omz[(size_t)t.gy(ly) * p.qpitch + t.gx(lx)]
                          : load_mapped(p.omz, p.qpitch, t.gx(lx), t.gy(ly), p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_Q, MAP_Q);
        F[F_QQ][q] = (2 * om + z) / hq;
        F[F_HQ][q] = hq;
      }
      if (lx >= H - 1 && lx <= TX + H - 1 && ly >= H - 1 && ly <= TY + H - 1) {
        if (nr && corners && !inner && (t.gx(lx) < 0 || t.gx(lx) >= p.Nx) && t.gy(ly) >= 0 && t.gy(ly) < p.Ny)
          F[F_KE][q] = kinetic_image<MS>(uk, vk, p.pitch, p.Nx, p.Ny, corners, k, L, t.gx(lx), t.gy(ly));
        else
          F[F_KE][q] = nr ? kinetic<MS, RW>(su, sv, t.mlx(lx), t.mly(ly)) : 0.0;
      }
      if (p.useA2 || useA4) {
        if (lx >= H - 2 && lx <= RW - 2 && ly >= H - 2 && ly <= RH - 2)
          F[F_DT][q] = DIV(AT(su, lx + 1, ly) - AT(su, lx, ly), dx, rdx)
                     - DIV(AT(sv, lx, ly + 1) - AT(sv, lx, ly), dy, rdy);
        if (lx >= 1 && ly >= 1 && lx >= H - 2 && ly >= H - 2)
          F[F_DS][q] = DIV(AT(su, lx, ly) - AT(su, lx, ly - 1), dy, rdy)
                     + DIV(AT(sv, lx, ly) - AT(sv, lx - 1, ly), dx, rdx);
      }
    }
    __syncthreads();
    const double* hw = F[F_HW];
    const double* hs = F[F_HS];
    const double* hq = F[F_HQ];
    const double* DT = F[F_DT];
    const double* DS = F[F_DS];
    // ---- Smagorinsky coefficients from the deformation rates (work.c:1587-1610) ----
    const double* A2h = SM + S_A2H * RN;
    const double* A2q = SM + S_A2Q * RN;
    const double* A4h = SM + S_A4H * RN;
    const double* A4q = SM + S_A4Q * RN;
    if (use_smag) {
      for (int q = tid; q < RN; q += NT) {
        int lx = q % RW, ly = q / RW;
        // cells: A2 and sqrt(A4) from |D| at the cell centre
        if (lx >= H - 2 && lx <= TX + H && ly >= H - 2 && ly <= TY + H && lx >= 1 && ly >= 1) {
          const double DDh = sqrt(sq(AT(DT, lx, ly))
                                  + sq(0.25 * (AT(DS, lx, ly) + AT(DS, lx + 1, ly) + AT(DS, lx, ly + 1) + AT(DS, lx + 1, ly + 1))));
          SM[S_A2H * RN + q] = fmax(p.A2, p.A2f * DDh);
          SM[S_A4H * RN + q] = sqrt(fmax(p.A4, p.A4f * DDh));
        }
        // q points
        if (lx >= H - 1 && lx <= TX + H + 1 && ly >= H - 1 && ly <= TY + H + 1 && lx <= RW - 2 && ly <= RH - 2) {
          const double DDq = sqrt(sq(0.25 * (AT(DT, lx, ly) + AT(DT, lx - 1, ly) + AT(DT, lx, ly - 1) + AT(DT, lx - 1, ly - 1)))
                                  + sq(AT(DS, lx, ly)));
          SM[S_A2Q * RN + q] = fmax(p.A2, p.A2f * DDq);
          SM[S_A4Q * RN + q] = sqrt(fmax(p.A4, p.A4f * DDq));
        }
      }
      __syncthreads();
    }
    // without its Smagorinsky term a coefficient is the constant itself (fmax(A, 0) = A and
    // sqrt(fmax(A4, 0)) = sqrt(A4) in the reference)
    const bool smag2 = (use_smag & 1) != 0, smag4 = (use_smag & 2) != 0;
    auto A2H = [&](int x, int y) { return smag2 ? AT(A2h, x, y) : p.A2; };
    auto A2Q = [&](int x, int y) { return smag2 ? AT(A2q, x, y) : p.A2; };
    auto A4H = [&](int x, int y) { return smag4 ? AT(A4h, x, y) : p.A4sqrt; };
    auto A4Q = [&](int x, int y) { return smag4 ? AT(A4q, x, y) : p.A4sqrt; };
    // ---- mass fluxes and the biharmonic intermediate velocities ----
    for (int q = tid; q < RN; q += NT) {
      int lx = q % RW, ly = q / RW;
      // seam ghost columns (serial build's corners): the mass fluxes are periodic copies of the
      // image column's (work.c:162-186 then an internal exchange); the biharmonic terms are
      // computed in place over the ghosted arrays
      const bool seam = corners && !inner && (t.gx(lx) < 0 || t.gx(lx) >= p.Nx);
      const ImageW iw{uk, vk, hkp, corners, p.pitch, p.Nx, p.Ny, k, L};
      const int ix = wrap_index(t.gx(lx), p.Nx), iy = t.gy(ly);
      auto SU = [&](int a, int b) { return seam ? iw.U(ix + a - lx, iy + b - ly) : AT(su, a, b); };
      auto SV = [&](int a, int b) { return seam ? iw.V(ix + a - lx, iy + b - ly) : AT(sv, a, b); };
      if (lx >= H - 1 && lx <= TX + H && ly >= H - 1 && ly <= TY + H - 1) F[F_HUU][q] = SU(lx, ly) * hw[q];
      if (lx >= H - 1 && lx <= TX + H - 1 && ly >= H - 1 && ly <= TY + H) F[F_HVV][q] = SV(lx, ly) * hs[q];
      if (useA4 && lx >= H - 1 && lx <= TX + H && ly >= H - 1 && ly <= TY + H) {
        F[F_U4][q] = (DIV(A4H(lx, ly) * AT(sh, lx, ly) * AT(DT, lx, ly) - A4H(lx - 1, ly) * AT(sh, lx - 1, ly) * AT(DT, lx - 1, ly), dx, rdx)
                      + DIV(A4Q(lx, ly + 1) * AT(hq, lx, ly + 1) * AT(DS, lx, ly + 1) - A4Q(lx, ly) * AT(hq, lx, ly) * AT(DS, lx, ly), dy, rdy))
                     / AT(hw, lx, ly);
        F[F_V4][q] = (DIV(A4Q(lx + 1, ly) * AT(hq, lx + 1, ly) * AT(DS, lx + 1, ly) - A4Q(lx, ly) * AT(hq, lx, ly) * AT(DS, lx, ly), dx, rdx)
                      - DIV(A4H(lx, ly) * AT(sh, lx, ly) * AT(DT, lx, ly) - A4H(lx, ly - 1) * AT(sh, lx, ly - 1) * AT(DT, lx, ly - 1), dy, rdy))
                     / AT(hs, lx, ly);
      }
    }
    __syncthreads();
    if (!valid) continue;

    const double* huu = F[F_HUU];
    const double* hvv = F[F_HVV];
    const double* KE = F[F_KE];
    const double* MM = MMall + k * RN;
    const double* U4 = F[F_U4];
    const double* V4 = F[F_V4];
    Coef<MS, RW, decltype(DIV)> c{F[F_QQ], r24, DIV};
    const double* qq = F[F_QQ];
    const int i = ox, j = oy;
    const double hwest = AT(hw, i, j), hsouth = AT(hs, i, j);
    const double rhw = 1.0 / hwest, rhs = 1.0 / hsouth;   // reciprocals for div_rn
    const double uc = AT(su, i, j), vc = AT(sv, i, j);

    // ---- u momentum (work.c:1667-1752) ----
    double ru;
    {
      double gM = DIV(-(AT(MM, i, j) - AT(MM, i - 1, j)), dx, rdx);
      double gK = DIV(-(AT(KE, i, j) - AT(KE, i - 1, j)), dx, rdx);
      double rq = 0;
      if (MS == 0 || MS == 1) {
        rq += c.alpha(i, j) * AT(hvv, i, j + 1) + c.beta(i, j) * AT(hvv, i - 1, j + 1)
            + c.gamma(i, j) * AT(hvv, i - 1, j) + c.delta(i, j) * AT(hvv, i, j)
            - c.epsilon(i, j) * AT(huu, i + 1, j) + c.epsilon(i - 1, j) * AT(huu, i - 1, j);
      } else if (MS == 3) {
        rq += c.alpha(i, j) * AT(hvv, i, j + 1) + c.beta(i, j) * AT(hvv, i - 1, j + 1)
            + c.gamma(i, j) * AT(hvv, i - 1, j) + c.delta(i, j) * AT(hvv, i, j)
            - c.epsilon(i, j) * AT(huu, i + 1, j) + c.epsilon(i - 1, j) * AT(huu, i - 1, j)
            - c.lambda(i, j + 1) * AT(huu, i, j) + c.lambda(i, j) * AT(huu, i, j - 1);
      } else {
        rq += 0.25 * AT(qq, i, j) * (AT(hvv, i, j) + AT(hvv, i - 1, j))
            + 0.25 * AT(qq, i, j + 1) * (AT(hvv, i, j + 1) + AT(hvv, i - 1, j + 1));
      }
      double a2 = 0, a4 = 0;
      if (p.useA2) {
        a2 = (DIV(A2H(i, j) * AT(sh, i, j) * AT(DT, i, j) - A2H(i - 1, j) * AT(sh, i - 1, j) * AT(DT, i - 1, j), dx, rdx)
              + DIV(A2Q(i, j + 1) * AT(hq, i, j + 1) * AT(DS, i, j + 1) - A2Q(i, j) * AT(hq, i, j) * AT(DS, i, j), dy, rdy));
      }
      if (useA4) {
        double d4t0 = DIV(AT(U4, i + 1, j) - AT(U4, i, j), dx, rdx) - DIV(AT(V4, i, j + 1) - AT(V4, i, j), dy, rdy);
        double d4tm = DIV(AT(U4, i, j) - AT(U4, i - 1, j), dx, rdx) - DIV(AT(V4, i - 1, j + 1) - AT(V4, i - 1, j), dy, rdy);
        double d4s1 = DIV(AT(U4, i, j + 1) - AT(U4, i, j), dy, rdy) + DIV(AT(V4, i, j + 1) - AT(V4, i - 1, j + 1), dx, rdx);
        double d4s0 = DIV(AT(U4, i, j) - AT(U4, i, j - 1), dy, rdy) + DIV(AT(V4, i, j) - AT(V4, i - 1, j), dx, rdx);
        a4 = -(DIV(A4H(i, j) * AT(sh, i, j) * d4t0 - A4H(i - 1, j) * AT(sh, i - 1, j) * d4tm, dx, rdx)
               + DIV(A4Q(i, j + 1) * AT(hq, i, j + 1) * d4s1 - A4Q(i, j) * AT(hq, i, j) * d4s0, dy, rdy));
      }
      double buoy = 0;
      if constexpr (BUD) {
        // -0.5 (hz(i) + hz(i-1)) db/dx (work.c:1745-1748)
        if (p.use_buoy && hwest != 0)
          buoy = -0.5 * (buoy_hz(p, k, gi, gj) + buoy_hz(p, k, gi - 1, gj))
               * DIV(gload(p.b + k * p.lstride, p, gi, gj, MAP_S, MAP_S)
                        - gload(p.b + k * p.lstride, p, gi - 1, gj, MAP_S, MAP_S), dx, rdx);
      }
      ru = gM + gK + rq + ((hwest != 0) ? DIV(a2 + a4 + buoy, hwest, rhw) : 0);
      if constexpr (BUD) {
        // work.c:1753-1763
        const bool active = !(p.wall_ew && gi == 0);
        budget_add(p.bud_u, BU_GRADM, k, L, p.lstride, cell, hwest * gM * p.dt);
        budget_add(p.bud_u, BU_GRADKE, k, L, p.lstride, cell, hwest * gK * p.dt);
        budget_add(p.bud_u, BU_Q, k, L, p.lstride, cell, hwest * rq * p.dt);
        budget_add(p.bud_u, BU_A2, k, L, p.lstride, cell, active ? a2 * p.dt : 0);
        budget_add(p.bud_u, BU_A4, k, L, p.lstride, cell, active ? a4 * p.dt : 0);
        budget_add(p.bud_e, BE_GRADM, k, L, p.lstride, cell, hwest * gM * uc * p.dt);
        budget_add(p.bud_e, BE_ADV, k, L, p.lstride, cell, hwest * (gK + rq) * uc * p.dt);
        budget_add(p.bud_e, BE_A2, k, L, p.lstride, cell, a2 * uc * p.dt);
        budget_add(p.bud_e, BE_A4, k, L, p.lstride, cell, a4 * uc * p.dt);
        budget_add(p.bud_u, BU_BUOY, k, L, p.lstride, cell, buoy * p.dt);
        budget_add(p.bud_e, BE_BUOY, k, L, p.lstride, cell, buoy * uc * p.dt);
      }
    }
    // ---- v momentum (work.c:1759-1852) ----
    double rv;
    {
      double gM = DIV(-(AT(MM, i, j) - AT(MM, i, j - 1)), dy, rdy);
      double gK = DIV(-(AT(KE, i, j) - AT(KE, i, j - 1)), dy, rdy);
      double rq = 0;
      if (MS == 0 || MS == 1) {
        rq += c.phi(i, j - 1) * AT(hvv, i, j - 1) - c.phi(i, j) * AT(hvv, i, j + 1)
            - c.gamma(i + 1, j) * AT(huu, i + 1, j) - c.delta(i, j) * AT(huu, i, j)
            - c.alpha(i, j - 1) * AT(huu, i, j - 1) - c.beta(i + 1, j - 1) * AT(huu, i + 1, j - 1);
      } else if (MS == 3) {
        rq += c.phi(i, j - 1) * AT(hvv, i, j - 1) - c.phi(i, j) * AT(hvv, i, j + 1)
            - c.gamma(i + 1, j) * AT(huu, i + 1, j) - c.delta(i, j) * AT(huu, i, j)
            - c.alpha(i, j - 1) * AT(huu, i, j - 1) - c.beta(i + 1, j - 1) * AT(huu, i + 1, j - 1)
            - c.mu(i + 1, j) * AT(hvv, i, j) + c.mu(i, j) * AT(hvv, i - 1, j);
      } else {
        rq -= 0.25 * AT(qq, i, j) * (AT(huu, i, j) + AT(huu, i, j - 1))
            + 0.25 * AT(qq, i + 1, j) * (AT(huu, i + 1, j) + AT(huu, i + 1, j - 1));
      }
      double a2 = 0, a4 = 0;
      if (p.useA2) {
        a2 = (DIV(A2Q(i + 1, j) * AT(hq, i + 1, j) * AT(DS, i + 1, j) - A2Q(i, j) * AT(hq, i, j) * AT(DS, i, j), dx, rdx)
              - DIV(A2H(i, j) * AT(sh, i, j) * AT(DT, i, j) - A2H(i, j - 1) * AT(sh, i, j - 1) * AT(DT, i, j - 1), dy, rdy));
      }
      if (useA4) {
        double d4s1 = DIV(AT(U4, i + 1, j) - AT(U4, i + 1, j - 1), dy, rdy) + DIV(AT(V4, i + 1, j) - AT(V4, i, j), dx, rdx);
        double d4s0 = DIV(AT(U4, i, j) - AT(U4, i, j - 1), dy, rdy) + DIV(AT(V4, i, j) - AT(V4, i - 1, j), dx, rdx);
        double d4t0 = DIV(AT(U4, i + 1, j) - AT(U4, i, j), dx, rdx) - DIV(AT(V4, i, j + 1) - AT(V4, i, j), dy, rdy);
        double d4tm = DIV(AT(U4, i + 1, j - 1) - AT(U4, i, j - 1), dx, rdx) - DIV(AT(V4, i, j) - AT(V4, i, j - 1), dy, rdy);
        a4 = -(DIV(A4Q(i + 1, j) * AT(hq, i + 1, j) * d4s1 - A4Q(i, j) * AT(hq, i, j) * d4s0, dx, rdx)
               - DIV(A4H(i, j) * AT(sh, i, j) * d4t0 - A4H(i, j - 1) * AT(sh, i, j - 1) * d4tm, dy, rdy));
      }
      double buoy = 0;
      if constexpr (BUD) {
        // work.c:1829-1832
        if (p.use_buoy && hsouth != 0)
          buoy = -0.5 * (buoy_hz(p, k, gi, gj) + buoy_hz(p, k, gi, gj - 1))
               * DIV(gload(p.b + k * p.lstride, p, gi, gj, MAP_S, MAP_S)
                        - gload(p.b + k * p.lstride, p, gi, gj - 1, MAP_S, MAP_S), dy, rdy);
      }
      rv = gM + gK + rq + ((hsouth != 0) ? DIV(a2 + a4 + buoy, hsouth, rhs) : 0);
      if constexpr (BUD) {
        // work.c:1837-1847
        const bool active = !(p.wall_ns && gj == 0);
        budget_add(p.bud_v, BU_GRADM, k, L, p.lstride, cell, hsouth * gM * p.dt);
        budget_add(p.bud_v, BU_GRADKE, k, L, p.lstride, cell, hsouth * gK * p.dt);
        budget_add(p.bud_v, BU_Q, k, L, p.lstride, cell, hsouth * rq * p.dt);
        budget_add(p.bud_v, BU_A2, k, L, p.lstride, cell, active ? a2 * p.dt : 0);
        budget_add(p.bud_v, BU_A4, k, L, p.lstride, cell, active ? a4 * p.dt : 0);
        budget_add(p.bud_e, BE_GRADM, k, L, p.lstride, cell, hsouth * gM * vc * p.dt);
        budget_add(p.bud_e, BE_ADV, k, L, p.lstride, cell, hsouth * (gK + rq) * vc * p.dt);
        budget_add(p.bud_e, BE_A2, k, L, p.lstride, cell, a2 * vc * p.dt);
        budget_add(p.bud_e, BE_A4, k, L, p.lstride, cell, a4 * vc * p.dt);
        budget_add(p.bud_v, BU_BUOY, k, L, p.lstride, cell, buoy * p.dt);
        budget_add(p.bud_e, BE_BUOY, k, L, p.lstride, cell, buoy * vc * p.dt);
      }
    }
    // ---- diapycnal advection and viscosity (diapycnal.c:203-291) ----
    if (use_wdia || use_diavisc) {
      if (use_wdia) {
        const double* W0 = WDall + k * RN;
        const double* W1 = WDall + (k + 1) * RN;
        double wu0 = 0.5 * (AT(W0, i, j) + AT(W0, i - 1, j));
        double wu1 = 0.5 * (AT(W1, i, j) + AT(W1, i - 1, j));
        double wv0 = 0.5 * (AT(W0, i, j) + AT(W0, i, j - 1));
        double wv1 = 0.5 * (AT(W1, i, j) + AT(W1, i, j - 1));
        double up = (k == 0) ? 0 : p.u[(k - 1) * p.lstride + cell];
        double um = (k == L - 1) ? 0 : p.u[(k + 1) * p.lstride + cell];
        double vp = (k == 0) ? 0 : p.v[(k - 1) * p.lstride + cell];
        double vm = (k == L - 1) ? 0 : p.v[(k + 1) * p.lstride + cell];
        // the wall face carries a zero tendency at the end, whatever is accumulated here
        double dup = (wu0 > 0) ? 0 : up - uc;
        double dum = (wu1 > 0) ? uc - um : 0;
        double dvp = (wv0 > 0) ? 0 : vp - vc;
        double dvm = (wv1 > 0) ? vc - vm : 0;
        if (hwest != 0) {
          const double r = -(wu0 * dup + wu1 * dum);
          ru += DIV(r, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_WDIA, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_WDIAKE, k, L, p.lstride, cell, r * uc * p.dt);
          }
        }
        if (hsouth != 0) {
          const double r = -(wv0 * dvp + wv1 * dvm);
          rv += DIV(r, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_WDIA, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_WDIAKE, k, L, p.lstride, cell, r * vc * p.dt);
          }
        }
      }
      if (use_diavisc && L >= 2) {
        double Fu[2] = {0, 0}, Fv[2] = {0, 0};
        for (int s = 0; s < 2; ++s) {
          int kk = k + s;                    // interface kk between layers kk-1 and kk
          if (kk < 1 || kk > L - 1) continue;
          double hwa = face_west_cell<TS>(p, kk - 1, gi, gj);
          double hwb = face_west_cell<TS>(p, kk, gi, gj);
          double hsa = face_south_cell<TS>(p, kk - 1, gi, gj);
          double hsb = face_south_cell<TS>(p, kk, gi, gj);
          double dzu = 0.5 * (hwb + hwa);
          double dzv = 0.5 * (hsb + hsa);
          double nuu = gload(p.nu_u + kk * p.lstride, p, gi, gj, MAP_N, MAP_S);
          double nuv = gload(p.nu_v + kk * p.lstride, p, gi, gj, MAP_S, MAP_N);
          if constexpr (BUD) {
            // convective viscosity where the local reduced gravity g' = gg + b(k-1) - b(k) is
            // negative (diapycnal.c:40-66, 104-114); without buoyancy g' = gg >= 0
            if (p.use_buoy && p.conv_diff != 0) {
              auto gp = [&](int x, int y) {
                return p.gg[kk] + (gload(p.b + (kk - 1) * p.lstride, p, x, y, MAP_S, MAP_S)
                                   - gload(p.b + kk * p.lstride, p, x, y, MAP_S, MAP_S));
              };
              const double g0 = gp(gi, gj);
              if (g0 < 0 || gp(gi - 1, gj) < 0) nuu += p.conv_diff;
              if (g0 < 0 || gp(gi, gj - 1) < 0) nuv += p.conv_diff;
            }
          }
          double ua = gload(p.u + (kk - 1) * p.lstride, p, gi, gj, MAP_N, MAP_S);
          double ub = gload(p.u + kk * p.lstride, p, gi, gj, MAP_N, MAP_S);
          double va = gload(p.v + (kk - 1) * p.lstride, p, gi, gj, MAP_S, MAP_N);
          double vb = gload(p.v + kk * p.lstride, p, gi, gj, MAP_S, MAP_N);
          if (dzu != 0) Fu[s] = nuu * (ua - ub) / dzu;
          if (dzv != 0) Fv[s] = nuv * (va - vb) / dzv;
        }
        if (hwest != 0) {
          const double r = Fu[0] - Fu[1];
          ru += DIV(r, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_DIAVISC, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_DIAVISC, k, L, p.lstride, cell, r * uc * p.dt);
          }
        }
        if (hsouth != 0) {
          const double r = Fv[0] - Fv[1];
          rv += DIV(r, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_DIAVISC, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_DIAVISC, k, L, p.lstride, cell, r * vc * p.dt);
          }
        }
      }
    }
    // ---- forcing and drag (forcing.c:149-395) ----
    {
      const bool wface_u = p.wall_ew && gi == 0;
      const bool wface_v = p.wall_ns && gj == 0;
      // layer fractions: computed ones, or all to the top / bottom layer; zero on a wall face
      double fsw, fss, fbw, fbs;
      if (use_fractions) {
        fsw = FR[(0 * L + k) * NT + tid];
        fss = FR[(1 * L + k) * NT + tid];
        fbw = FR[(2 * L + k) * NT + tid];
        fbs = FR[(3 * L + k) * NT + tid];
      } else {
        fsw = fss = (k == 0) ? 1.0 : 0.0;
        fbw = fbs = (k == L - 1) ? 1.0 : 0.0;
      }
      if (wface_u) fsw = fbw = 0.0;
      if (wface_v) fss = fbs = 0.0;
      if (p.use_wind) {
        double tx_ = p.tw0 * p.taux0[cell] + p.tw1 * p.taux1[cell];
        double ty_ = p.tw0 * p.tauy0[cell] + p.tw1 * p.tauy1[cell];
        double r = tx_ * fsw;
        if (hwest != 0) ru += DIV(r, hwest, rhw);
        if constexpr (BUD) {
          budget_add(p.bud_u, BU_WIND, k, L, p.lstride, cell, r * p.dt);
          budget_add(p.bud_e, BE_WIND, k, L, p.lstride, cell, r * uc * p.dt);
        }
        r = ty_ * fss;
        if (hsouth != 0) rv += DIV(r, hsouth, rhs);
        if constexpr (BUD) {
          budget_add(p.bud_v, BU_WIND, k, L, p.lstride, cell, r * p.dt);
          budget_add(p.bud_e, BE_WIND, k, L, p.lstride, cell, r * vc * p.dt);
        }
      }
      if (use_fbaro) {
        const double fx = gload(p.fbx, p, gi, gj, MAP_N, MAP_S), fy = gload(p.fby, p, gi, gj, MAP_S, MAP_N);
        ru += fx;
        rv += fy;
        if constexpr (BUD) {
          budget_add(p.bud_u, BU_FBARO, k, L, p.lstride, cell, hwest * fx * p.dt);
          budget_add(p.bud_v, BU_FBARO, k, L, p.lstride, cell, hsouth * fy * p.dt);
          budget_add(p.bud_e, BE_FBARO, k, L, p.lstride, cell, (hwest * fx * uc + hsouth * fy * vc) * p.dt);
        }
      }
      if (p.lin_drag > 0) {
        if (hwest != 0) {
          const double r = -p.lin_drag * uc * fbw;
          ru += DIV(r, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_RDRAG, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_RDRAG, k, L, p.lstride, cell, r * uc * p.dt);
          }
        }
        if (hsouth != 0) {
          const double r = -p.lin_drag * vc * fbs;
          rv += DIV(r, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_RDRAG, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_RDRAG, k, L, p.lstride, cell, r * vc * p.dt);
          }
        }
      }
      // the surface drag is off under a rigid lid over land unless oceanSurfDrag
      auto surf_mask_u = [&]() {
        double hsw = 0.5 * (gload(p.hhs, p, gi, gj, MAP_S, MAP_S) + gload(p.hhs, p, gi - 1, gj, MAP_S, MAP_S));
        return !p.ocean_surf_drag && p.use_rl && hsw >= 0;
      };
      auto surf_mask_v = [&]() {
        double hss = 0.5 * (gload(p.hhs, p, gi, gj, MAP_S, MAP_S) + gload(p.hhs, p, gi, gj - 1, MAP_S, MAP_S));
        return !p.ocean_surf_drag && p.use_rl && hss >= 0;
      };
      if ((!LEAN && p.lin_drag_surf > 0)) {
        if (hwest != 0) {
          double r = -p.lin_drag_surf * (uc - gload(p.uLid, p, gi, gj, MAP_N, MAP_S)) * fsw;
          if (surf_mask_u()) r = 0;
          ru += DIV(r, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_RSURF, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_RSURF, k, L, p.lstride, cell, r * uc * p.dt);
          }
        }
        if (hsouth != 0) {
          double r = -p.lin_drag_surf * (vc - gload(p.vLid, p, gi, gj, MAP_S, MAP_N)) * fss;
          if (surf_mask_v()) r = 0;
          rv += DIV(r, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_RSURF, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_RSURF, k, L, p.lstride, cell, r * vc * p.dt);
          }
        }
      }
      // quadratic drag (forcing.c:95-143, 330-393): the speed at the cell centre from the
      // squared bottom (surface) velocities of the neighbouring faces. Without a fraction
      // depth it acts on the bottom (top) layer alone, whose tile is in shared memory; with one
      // it acts on every layer the fractions reach, from the pre-pass's weighted velocities.
      if ((!LEAN && p.quad_drag > 0) && (p.drag_bot || k == L - 1)) {
        auto uab = [&](int a, int b) {
          if (p.drag_bot) {
            const double* UB = p.dragv;
            const double* VB = p.dragv + p.lstride;
            const int x = t.gx(a), y = t.gy(b);
            return sqrt(0.5 * (sq(drag_load(UB, p, x, y, MAP_N, MAP_S)) + sq(drag_load(UB, p, x + 1, y, MAP_N, MAP_S)))
                        + 0.5 * (sq(drag_load(VB, p, x, y, MAP_S, MAP_N)) + sq(drag_load(VB, p, x, y + 1, MAP_S, MAP_N))));
          }
          return sqrt(0.5 * (sq(AT(su, a, b)) + sq(AT(su, a + 1, b))) + 0.5 * (sq(AT(sv, a, b)) + sq(AT(sv, a, b + 1))));
        };
        if (hwest != 0) {
          const double ua = 0.5 * (uab(i, j) + uab(i - 1, j));
          ru -= DIV(p.quad_drag * ua * uc * fbw, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_CDBOT, k, L, p.lstride, cell, -p.quad_drag * ua * uc * fbw * p.dt);
            budget_add(p.bud_e, BE_CDBOT, k, L, p.lstride, cell, -p.quad_drag * ua * sq(uc) * fbw * p.dt);
          }
        }
        if (hsouth != 0) {
          const double ua = 0.5 * (uab(i, j) + uab(i, j - 1));
          rv -= DIV(p.quad_drag * ua * vc * fbs, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_CDBOT, k, L, p.lstride, cell, -p.quad_drag * ua * vc * fbs * p.dt);
            budget_add(p.bud_e, BE_CDBOT, k, L, p.lstride, cell, -p.quad_drag * ua * sq(vc) * fbs * p.dt);
          }
        }
      }
      if ((!LEAN && p.quad_drag_surf > 0) && (p.drag_surf || k == 0)) {
        const double wf = 1.0 - p.wfb;
        auto lidu = [&](int a, int b) { return gload(p.uLid, p, t.gx(a), t.gy(b), MAP_N, MAP_S); };
        auto lidv = [&](int a, int b) { return gload(p.vLid, p, t.gx(a), t.gy(b), MAP_S, MAP_N); };
        // the surface velocity: the top layer's, or the mixed-layer average of the pre-pass
        auto sfu = [&](int a, int b) {
          return p.drag_surf ? drag_load(p.dragv + 2 * p.lstride, p, t.gx(a), t.gy(b), MAP_N, MAP_S) : AT(su, a, b);
        };
        auto sfv = [&](int a, int b) {
          return p.drag_surf ? drag_load(p.dragv + 3 * p.lstride, p, t.gx(a), t.gy(b), MAP_S, MAP_N) : AT(sv, a, b);
        };
        auto usq = [&](int a, int b) { const double r = wf * sfu(a, b) - lidu(a, b); return r * r; };
        auto vsq = [&](int a, int b) { const double r = wf * sfv(a, b) - lidv(a, b); return r * r; };
        auto uab = [&](int a, int b) { return sqrt(0.5 * (usq(a, b) + usq(a + 1, b)) + 0.5 * (vsq(a, b) + vsq(a, b + 1))); };
        if (hwest != 0) {
          const double ua = 0.5 * (uab(i, j) + uab(i - 1, j));
          double r = -p.quad_drag_surf * ua * (wf * uc - gload(p.uLid, p, gi, gj, MAP_N, MAP_S)) * fsw;
          if (surf_mask_u()) r = 0;
          ru += DIV(r, hwest, rhw);
          if constexpr (BUD) {
            budget_add(p.bud_u, BU_CDSURF, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_CDSURF, k, L, p.lstride, cell, r * uc * p.dt);
          }
        }
        if (hsouth != 0) {
          const double ua = 0.5 * (uab(i, j) + uab(i, j - 1));
          double r = -p.quad_drag_surf * ua * (wf * vc - gload(p.vLid, p, gi, gj, MAP_S, MAP_N)) * fss;
          if (surf_mask_v()) r = 0;
          rv += DIV(r, hsouth, rhs);
          if constexpr (BUD) {
            budget_add(p.bud_v, BU_CDSURF, k, L, p.lstride, cell, r * p.dt);
            budget_add(p.bud_e, BE_CDSURF, k, L, p.lstride, cell, r * vc * p.dt);
          }
        }
      }
    }
    // ---- Newtonian velocity restoring (restoring.c:172-220) ----
    if (use_relax) {
      double ut = gload(p.uTime + k * p.lstride, p, gi, gj, MAP_N, MAP_S);
      if (ut > 0) {
        const double r = (-(uc - gload(p.uRelax + k * p.lstride, p, gi, gj, MAP_N, MAP_S))) / ut;
        ru += r;
        if constexpr (BUD) {
          budget_add(p.bud_u, BU_RELAX, k, L, p.lstride, cell, hwest * r * p.dt);
          budget_add(p.bud_e, BE_RELAX, k, L, p.lstride, cell, hwest * r * uc * p.dt);
        }
      }
      double vt = gload(p.vTime + k * p.lstride, p, gi, gj, MAP_S, MAP_N);
      if (vt > 0) {
        const double r = (-(vc - gload(p.vRelax + k * p.lstride, p, gi, gj, MAP_S, MAP_N))) / vt;
        rv += r;
        if constexpr (BUD) {
          budget_add(p.bud_v, BU_RELAX, k, L, p.lstride, cell, hsouth * r * p.dt);
          budget_add(p.bud_e, BE_RELAX, k, L, p.lstride, cell, hsouth * r * vc * p.dt);
        }
      }
    }
    // the wall-normal tendency is zero on the wall face (field.c:173-176, 216-220)
    if (p.wall_ew && gi == 0) ru = 0.0;
    if (p.wall_ns && gj == 0) rv = 0.0;
    // ---- thickness tendency (work.c:1875-1885) ----
    double rh;
    {
      double adv = DIV(AT(huu, i, j) - AT(huu, i + 1, j), dx, rdx) + DIV(AT(hvv, i, j) - AT(hvv, i, j + 1), dy, rdy);
      double rel = 0;
      if (use_wdia) {
        const double* W0 = WDall + k * RN;
        const double* W1 = WDall + (k + 1) * RN;
        rel = -(AT(W0, i, j) - AT(W1, i, j));
      } else {
        rel = -(0.0 - 0.0);
      }
      rh = adv + rel;
      if constexpr (BUD) {
        // work.c:1891-1906 and the second loop of work.c:1913-1937
        const double hc0 = AT(sh, i, j);
        const double ke2 = 0.5 * (sq(uc) + sq(vc));
        const double w0 = use_wdia ? AT(WDall + k * RN, i, j) : 0.0;
        const double w1 = use_wdia ? AT(WDall + (k + 1) * RN, i, j) : 0.0;
        double eta1 = p.hhb[cell];   // eta_w[k+1] and eta_w[k], built upward as in work.c:1184-1199
        for (int m = L - 1; m > k; --m) eta1 = eta1 + p.h[m * p.lstride + cell];
        const double eta0 = eta1 + hc0;
        const double g = p.geff[k], h0 = p.h0;
        budget_add(p.bud_h, BH_ADV, k, L, p.lstride, cell, adv * p.dt);
        budget_add(p.bud_h, BH_RELAX, k, L, p.lstride, cell, rel * p.dt);
        budget_add(p.bud_e, BE_ADV, k, L, p.lstride, cell, ke2 * adv * p.dt);
        budget_add(p.bud_e, BE_WDIAKE, k, L, p.lstride, cell, ke2 * rel * p.dt);
        budget_add(p.bud_e, BE_WDIAPE, k, L, p.lstride, cell,
                   -g * (eta0 * w0 - eta1 * w1) * p.dt
                   - (-g * (h0 * h0 * h0 * h0) / (hc0 * hc0 * hc0) / 3) * (-rel) * p.dt);
        if (p.b) {
          const double bc = p.b[k * p.lstride + cell];
          budget_add(p.bud_b, BB_ADV, k, L, p.lstride, cell, bc * adv * p.dt);
          budget_add(p.bud_b, BB_WDIA, k, L, p.lstride, cell, bc * rel * p.dt);
        }
        if (p.bud_u || p.bud_v) {
          const double adv_w = DIV(AT(huu, i - 1, j) - AT(huu, i, j), dx, rdx)
                             + DIV(AT(hvv, i - 1, j) - AT(hvv, i - 1, j + 1), dy, rdy);
          const double adv_s = DIV(AT(huu, i, j - 1) - AT(huu, i + 1, j - 1), dx, rdx)
                             + DIV(AT(hvv, i, j - 1) - AT(hvv, i, j), dy, rdy);
          double rel_w = -(0.0 - 0.0), rel_s = -(0.0 - 0.0);
          if (use_wdia) {
            rel_w = -(AT(WDall + k * RN, i - 1, j) - AT(WDall + (k + 1) * RN, i - 1, j));
            rel_s = -(AT(WDall + k * RN, i, j - 1) - AT(WDall + (k + 1) * RN, i, j - 1));
          }
          budget_add(p.bud_u, BU_DHDT, k, L, p.lstride, cell, 0.5 * uc * (adv + adv_w) * p.dt);
          budget_add(p.bud_u, BU_WDIA, k, L, p.lstride, cell, 0.5 * uc * (rel + rel_w) * p.dt);
          budget_add(p.bud_v, BU_DHDT, k, L, p.lstride, cell, 0.5 * vc * (adv + adv_s) * p.dt);
          budget_add(p.bud_v, BU_WDIA, k, L, p.lstride, cell, 0.5 * vc * (rel + rel_s) * p.dt);
        }
      }
    }
    // ---- Adams-Bashforth epilogue (integrator.c:15-69) ----
    const size_t o = k * p.lstride + cell;
    if (p.ab_mode == 0) {
      p.fu_out[o] = ru;
      p.fv_out[o] = rv;
      p.fh_out[o] = rh;
      continue;
    }
    double un, vn, hn;
    const double hc = sh[j * RW + i];
    if (p.ab_mode == 1) {
      un = uc + p.c0 * ru;
      vn = vc + p.c0 * rv;
      hn = hc + p.c0 * rh;
    } else if (p.ab_mode == 2) {
      un = uc + (p.c0 * ru - p.c1 * p.f1u[o]);
      vn = vc + (p.c0 * rv - p.c1 * p.f1v[o]);
      hn = hc + (p.c0 * rh - p.c1 * p.f1h[o]);
    } else {
      un = uc + (p.c0 * ru - p.c1 * p.f1u[o] + p.c2 * p.f2u[o]);
      vn = vc + (p.c0 * rv - p.c1 * p.f1v[o] + p.c2 * p.f2v[o]);
      hn = hc + (p.c0 * rh - p.c1 * p.f1h[o] + p.c2 * p.f2h[o]);
    }
    // after the update the reference re-imposes the wall face (field.c:173-176, 216-220)
    if (p.wall_ew && gi == 0) un = 0.0;
    if (p.wall_ns && gj == 0) vn = 0.0;
    if (p.nonfinite && !(isfinite(un) && isfinite(vn) && isfinite(hn))) *p.nonfinite = 1;
    if (p.write_hist) {
      p.fu_out[o] = ru;
      p.fv_out[o] = rv;
      p.fh_out[o] = rh;
    }
    p.u_out[o] = un;
    p.v_out[o] = vn;
    p.h_out[o] = hn;
    htot += hn;
  }

  // ---- rigid-lid column thickness constraint (pressure.c:525-561) ----
  if (p.ab_mode != 0 && p.fuse_thickness_fix && valid && htot != 0) {
    // the new thicknesses are read back from h_out (this thread's own writes, in L2)
    const double err = htot - p.Hc[cell];
    for (int k = 0; k < L; ++k) {
      const size_t o = k * p.lstride + cell;
      p.h_out[o] = p.h_out[o] * (1 - err / htot);
    }
  }
  // a tile whose quotients met an operand outside the branch-free division's range is listed
  // for the exact pass (tile_list: count, done counter, tile indices)
  if constexpr (!SLOWDIV) {
    if (__syncthreads_or(oor) && tid == 0) {
      const int e = atomicAdd(&p.tile_list[0], 1);
      p.tile_list[2 + e] = by * ((p.Nx + TX - 1) / TX) + bx;
    }
  }
}

template <int MS, int TS, int H, bool LEAN>
__global__ void __launch_bounds__(NT, PAWSIM_TEND_MINB) tendency_kernel(const __grid_constant__ TendParams p) {
  tendency_tile<MS, TS, H, LEAN, false>(p, blockIdx.x, blockIdx.y);
}

// The exact pass: the tiles the fused kernel listed, recomputed with div_rn (normally none).
// The last CTA to finish empties the list for the next launch.
template <int MS, int TS, int H>
__global__ void __launch_bounds__(NT, PAWSIM_TEND_MINB) tendency_exact_kernel(const __grid_constant__ TendParams p) {
  const int n = p.tile_list[0];
  const int gx = (p.Nx + TX - 1) / TX;
  for (int e = blockIdx.x; e < n; e += gridDim.x) {
    const int id = p.tile_list[2 + e];
    tendency_tile<MS, TS, H, false, true>(p, id % gx, id / gx);
    __syncthreads();
  }
  __shared__ int last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&p.tile_list[1], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    p.tile_list[0] = 0;
    p.tile_list[1] = 0;
    __threadfence();
  }
}

// Batched ensemble: one launch over a work-list of (member, tile) pairs, member << 20 | tile,
// with each member's parameters staged in shared memory. Every tile computes exactly what
// the member's own launch computes.
template <int MS, int TS, int H, bool LEAN>
__global__ void __launch_bounds__(NT, PAWSIM_TEND_MINB)
tendency_batch_kernel(const TendParams* __restrict__ ps, const int* __restrict__ work) {
  __shared__ TendParams sp;
  const int w = work[blockIdx.x];
  const int member = w >> 20, tile = w & 0xfffff;
  for (int q = threadIdx.x; q < (int)(sizeof(TendParams) / sizeof(int)); q += NT)
    reinterpret_cast<int*>(&sp)[q] = reinterpret_cast<const int*>(ps + member)[q];
  __syncthreads();
  const int gx = (sp.Nx + TX - 1) / TX;
  tendency_tile<MS, TS, H, LEAN, false>(sp, tile % gx, tile / gx);
}

// the exact pass of every member's tile list (see tendency_exact_kernel); the last CTA empties
// all lists
template <int MS, int TS, int H>
__global__ void __launch_bounds__(NT, PAWSIM_TEND_MINB)
tendency_batch_exact_kernel(const TendParams* __restrict__ ps, int members, int* done) {
  __shared__ TendParams sp;
  for (int mb = 0; mb < members; ++mb) {
    for (int q = threadIdx.x; q < (int)(sizeof(TendParams) / sizeof(int)); q += NT)
      reinterpret_cast<int*>(&sp)[q] = reinterpret_cast<const int*>(ps + mb)[q];
    __syncthreads();
    const int n = sp.tile_list[0];
    const int gx = (sp.Nx + TX - 1) / TX;
    for (int e = blockIdx.x; e < n; e += gridDim.x) {
      const int id = sp.tile_list[2 + e];
      tendency_tile<MS, TS, H, false, true>(sp, id % gx, id / gx);
      __syncthreads();
    }
    __syncthreads();
  }
  __shared__ int last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    for (int mb = threadIdx.x; mb < members; mb += NT) {
      ps[mb].tile_list[0] = 0;
      ps[mb].tile_list[1] = 0;
    }
    if (threadIdx.x == 0) *done = 0;
    __threadfence();
  }
}

// dynamic shared memory of a tile (lean: the lean instantiation's, without the U4, V4 planes)
template <int H>
size_t smem_bytes(const TendParams& p, bool lean = false) {
  constexpr int RN = Geo<H>::RN;
  const int planes = lean ? F_U4 : F_NUM;
  return (size_t)(planes + p.L + (p.use_wdia ? p.L + 1 : 0) + (p.use_smag ? S_NUM : 0)) * RN * sizeof(double)
       + (p.use_fractions ? (size_t)4 * p.L * NT * sizeof(double) : 0);
}

constexpr int EXACT_CTAS = 148;   // the exact pass's grid: one CTA per SM

inline bool lean_params(const TendParams& p) { return tendency_lean(p); }

// Launches the step (the drag pre-pass when needed, the fused kernel and, in the plain build,
// the exact pass over flagged tiles); returns the number of launches, or -1.
template <int MS, int TS, int H>
int launch_t(const TendParams& p, cudaStream_t s) {
  const size_t shm = smem_bytes<H>(p);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(tendency_kernel<MS, TS, H, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if constexpr (!BUD) {
      cudaFuncSetAttribute(tendency_kernel<MS, TS, H, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      cudaFuncSetAttribute(tendency_exact_kernel<MS, TS, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           200 * 1024);
    }
    attr_done = true;
  }
  if (shm > 200 * 1024) return -1;
  int pre = 0;
  if (p.drag_bot || p.drag_surf) {
    dim3 b(32, 8), g((p.Nx + 31) / 32, (p.Ny + 7) / 8);
    drag_speed_kernel<TS><<<g, b, 0, s>>>(p);
    pre = 1;
  }
  dim3 grid((p.Nx + TX - 1) / TX, (p.Ny + TY - 1) / TY);
  if constexpr (BUD) {
    tendency_kernel<MS, TS, H, false><<<grid, NT, shm, s>>>(p);
    return pre + 1;
  } else {
    if (lean_params(p)) tendency_kernel<MS, TS, H, true><<<grid, NT, smem_bytes<H>(p, true), s>>>(p);
    else tendency_kernel<MS, TS, H, false><<<grid, NT, shm, s>>>(p);
    // the exact recomputation of the listed tiles (one CTA per SM walks the list; the full
    // build, so the full shared memory)
    tendency_exact_kernel<MS, TS, H><<<EXACT_CTAS, NT, shm, s>>>(p);
    return pre + 2;
  }
}

// the batched launch for members sharing p0's scheme, halo, feature set and layer count
template <int MS, int TS, int H>
int launch_batch_t(const TendParams& p0, const TendParams* ps, const int* work, int nwork, int members, int* done,
                   cudaStream_t s) {
  if constexpr (BUD) {
    return -1;
  } else {
    const size_t shm = smem_bytes<H>(p0);
    if (shm > 200 * 1024 || p0.drag_bot || p0.drag_surf) return -1;
    static bool attr_done = false;
    if (!attr_done) {
      cudaFuncSetAttribute(tendency_batch_kernel<MS, TS, H, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           200 * 1024);
      cudaFuncSetAttribute(tendency_batch_kernel<MS, TS, H, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           200 * 1024);
      cudaFuncSetAttribute(tendency_batch_exact_kernel<MS, TS, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           200 * 1024);
      attr_done = true;
    }
    if (lean_params(p0)) tendency_batch_kernel<MS, TS, H, true><<<nwork, NT, smem_bytes<H>(p0, true), s>>>(ps, work);
    else tendency_batch_kernel<MS, TS, H, false><<<nwork, NT, shm, s>>>(ps, work);
    tendency_batch_exact_kernel<MS, TS, H><<<EXACT_CTAS, NT, shm, s>>>(ps, members, done);
    return 2;
  }
}

template <int TS, int H>
int launch_ms(const TendParams& p, int ms, cudaStream_t s) {
#ifdef PAWSIM_TEND_MS
  // this translation unit holds one momentum scheme (the build splits the instantiations)
  if (ms != PAWSIM_TEND_MS) return -1;
  return launch_t<PAWSIM_TEND_MS, TS, H>(p, s);
#else
  switch (ms) {
    case 0: return launch_t<0, TS, H>(p, s);
    case 1: return launch_t<1, TS, H>(p, s);
    case 2: return launch_t<2, TS, H>(p, s);
    case 3: return launch_t<3, TS, H>(p, s);
  }
  return -1;
#endif
}

// the upwind thickness schemes and the Smagorinsky biharmonic reach a third halo cell
inline bool wide_halo(const TendParams& p, int ts) { return ts >= 2 || (p.use_smag & 2); }

}  // namespace

#define PAWSIM_TEND_CAT2(a, b) a##b
#define PAWSIM_TEND_CAT(a, b) PAWSIM_TEND_CAT2(a, b)

#if PAWSIM_TEND_BUD
#define PAWSIM_TEND_SMEM_FN tendency_smem_budget
#define PAWSIM_TEND_LAUNCH_FN launch_tendency_budget_tile
#else
#define PAWSIM_TEND_SMEM_FN PAWSIM_TEND_CAT(tendency_smem_ty, PAWSIM_TEND_TY)
#define PAWSIM_TEND_LAUNCH_FN PAWSIM_TEND_CAT(PAWSIM_TEND_CAT(launch_tendency_ty, PAWSIM_TEND_TY), \
                                              PAWSIM_TEND_CAT(_m, PAWSIM_TEND_MS))
#endif

#if PAWSIM_TEND_BUD || PAWSIM_TEND_MS == 0
size_t PAWSIM_TEND_SMEM_FN(const TendParams& p, int ts) {
  return wide_halo(p, ts) ? smem_bytes<3>(p) : smem_bytes<2>(p);
}
#endif

#if !PAWSIM_TEND_BUD
// batched ensemble launch (tendency.cu dispatches on the momentum scheme and tile height)
int PAWSIM_TEND_CAT(batch_, PAWSIM_TEND_LAUNCH_FN)(const TendParams& p0, const TendParams* ps, const int* work,
                                                    int nwork, int members, int* done, int ms, int ts,
                                                    cudaStream_t s) {
#ifdef PAWSIM_TEND_MS
  if (ms != PAWSIM_TEND_MS) return -1;
#endif
  if (p0.L < 1 || p0.L > LMAX) return -1;
  if (!wide_halo(p0, ts)) {
    if (ts == 0) return launch_batch_t<PAWSIM_TEND_MS, 0, 2>(p0, ps, work, nwork, members, done, s);
    if (ts == 1) return launch_batch_t<PAWSIM_TEND_MS, 1, 2>(p0, ps, work, nwork, members, done, s);
    return -1;
  }
  switch (ts) {
    case 0: return launch_batch_t<PAWSIM_TEND_MS, 0, 3>(p0, ps, work, nwork, members, done, s);
    case 1: return launch_batch_t<PAWSIM_TEND_MS, 1, 3>(p0, ps, work, nwork, members, done, s);
    case 2: return launch_batch_t<PAWSIM_TEND_MS, 2, 3>(p0, ps, work, nwork, members, done, s);
    case 3: return launch_batch_t<PAWSIM_TEND_MS, 3, 3>(p0, ps, work, nwork, members, done, s);
  }
  return -1;
}
#endif

int PAWSIM_TEND_LAUNCH_FN(const TendParams& p, int ms, int ts, cudaStream_t s) {
  if (p.L < 1 || p.L > LMAX) return -1;
  if (!wide_halo(p, ts)) {
    if (ts == 0) return launch_ms<0, 2>(p, ms, s);
    if (ts == 1) return launch_ms<1, 2>(p, ms, s);
    return -1;
  }
  switch (ts) {
    case 0: return launch_ms<0, 3>(p, ms, s);
    case 1: return launch_ms<1, 3>(p, ms, s);
    case 2: return launch_ms<2, 3>(p, ms, s);
    case 3: return launch_ms<3, 3>(p, ms, s);
  }
  return -1;
}

}  // namespace pawsim
