// tracer.cu -- passive tracer tendency and Adams-Bashforth update (see tracer.cuh).
//
// One thread per owned cell and layer, reading its stencil through the boundary maps of
// common.cuh (cached loads; the tracer is a small share of a step). The ghost semantics are
// those of the fused tendency kernel: b is a scalar mirrored at walls; the face thickness
// h_west / h_south, which the reference re-fills after computing it, is evaluated at the
// mirrored owned position; the fields the reference computes over its ghost ring and never
// re-fills (h u, h v, the tracer gradients and fluxes, BB4) are evaluated directly at the
// ghost position. Expression order follows work.c:1947-2144 so that the results are those
// of the reference bit for bit (this file is compiled with -fmad=false).
#include "common.cuh"
#include "tracer.cuh"

namespace pawsim {

namespace {

struct TView {
  const TracerParams& p;
  const double *u, *v, *h, *b;
  __device__ double B(int a, int c) const {
    return load_mapped(b, p.pitch, a, c, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_S);
  }
  __device__ double Hc(int a, int c) const {
    return load_mapped(h, p.pitch, a, c, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_S);
  }
  __device__ double U(int a, int c) const {
    return load_mapped(u, p.pitch, a, c, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_N, MAP_S);
  }
  __device__ double V(int a, int c) const {
    return load_mapped(v, p.pitch, a, c, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_N);
  }
  __device__ int mx(int a) const { return map_axis(a, p.Nx, p.wall_ew, MAP_S).idx; }
  __device__ int my(int c) const { return map_axis(c, p.Ny, p.wall_ns, MAP_S).idx; }

  // face thickness of work.c:566-684 at an owned cell (i, j)
  __device__ double face_w_owned(int i, int j) const {
    auto H = [&](int a, int c) { return Hc(a, c); };
    const int TS = p.thick_scheme;
    if (TS == 1)
      return (1.0 / 3) * (H(i, j) + H(i - 1, j) + 0.25 * (H(i, j + 1) + H(i - 1, j + 1) + H(i, j - 1) + H(i - 1, j - 1)));
    if (TS == 2 || TS == 3) {
      const double uc = U(i, j);
      if (TS == 2) {
        const double d2m = H(i, j) - 2 * H(i - 1, j) + H(i - 2, j);
        const double d2c = H(i + 1, j) - 2 * H(i, j) + H(i - 1, j);
        return 0.5 * (H(i, j) + H(i - 1, j)) - (1 / 6.0) * ((uc > 0) ? d2m : d2c);
      }
      const double sg = p.kt00_sigma;
      const double dm = mm3(sg * (H(i, j) - H(i - 1, j)), 0.5 * (H(i, j) - H(i - 2, j)), sg * (H(i - 1, j) - H(i - 2, j)));
      const double dc = mm3(sg * (H(i + 1, j) - H(i, j)), 0.5 * (H(i + 1, j) - H(i - 1, j)), sg * (H(i, j) - H(i - 1, j)));
      return (uc > 0) ? H(i - 1, j) + 0.5 * dm : H(i, j) - 0.5 * dc;
    }
    return 0.5 * (H(i, j) + H(i - 1, j));
  }
  __device__ double face_s_owned(int i, int j) const {
    auto H = [&](int a, int c) { return Hc(a, c); };
    const int TS = p.thick_scheme;
    if (TS == 1)
      return (1.0 / 3) * (H(i, j) + H(i, j - 1) + 0.25 * (H(i + 1, j) + H(i - 1, j) + H(i + 1, j - 1) + H(i - 1, j - 1)));
    if (TS == 2 || TS == 3) {
      const double vc = V(i, j);
      if (TS == 2) {
        const double d2m = H(i, j) - 2 * H(i, j - 1) + H(i, j - 2);
        const double d2c = H(i, j + 1) - 2 * H(i, j) + H(i, j - 1);
        return 0.5 * (H(i, j) + H(i, j - 1)) - (1 / 6.0) * ((vc > 0) ? d2m : d2c);
      }
      const double sg = p.kt00_sigma;
      const double dm = mm3(sg * (H(i, j) - H(i, j - 1)), 0.5 * (H(i, j) - H(i, j - 2)), sg * (H(i, j - 1) - H(i, j - 2)));
      const double dc = mm3(sg * (H(i, j + 1) - H(i, j)), 0.5 * (H(i, j + 1) - H(i, j - 1)), sg * (H(i, j) - H(i, j - 1)));
      return (vc > 0) ? H(i, j - 1) + 0.5 * dm : H(i, j) + 0.5 * dc;
    }
    return 0.5 * (H(i, j) + H(i, j - 1));
  }
  // re-filled fields: the value of the mirrored owned position
  __device__ double Hw(int a, int c) const { return face_w_owned(mx(a), my(c)); }
  __device__ double Hs(int a, int c) const { return face_s_owned(mx(a), my(c)); }
  // layer mass fluxes (work.c:162-186), at the raw position
  __device__ double huu(int a, int c) const { return U(a, c) * Hw(a, c); }
  __device__ double hvv(int a, int c) const { return V(a, c) * Hs(a, c); }

  // minmod of three slopes (defs.c:1000-1014)
  __device__ static double mm3(double x, double y, double z) {
    if ((x > 0) && (y > 0) && (z > 0)) return fmin(x, fmin(y, z));
    if ((x < 0) && (y < 0) && (z < 0)) return fmax(x, fmax(y, z));
    return 0;
  }

  // tracer gradients and fluxes (work.c:1967-2053), at the raw position
  __device__ double db_dx(int a, int c) const { return (B(a, c) - B(a - 1, c)) / p.dx; }
  __device__ double db_dy(int a, int c) const { return (B(a, c) - B(a, c - 1)) / p.dy; }
  __device__ double d2bx(int a, int c) const { return B(a + 1, c) - 2 * B(a, c) + B(a - 1, c); }
  __device__ double d2by(int a, int c) const { return B(a, c + 1) - 2 * B(a, c) + B(a, c - 1); }
  __device__ double kt_dx(int a, int c) const {
    const double s = p.kt00_sigma;
    return mm3(s * (B(a + 1, c) - B(a, c)), 0.5 * (B(a + 1, c) - B(a - 1, c)), s * (B(a, c) - B(a - 1, c))) / p.dx;
  }
  __device__ double kt_dy(int a, int c) const {
    const double s = p.kt00_sigma;
    return mm3(s * (B(a, c + 1) - B(a, c)), 0.5 * (B(a, c + 1) - B(a, c - 1)), s * (B(a, c) - B(a, c - 1))) / p.dy;
  }
  __device__ double hub(int a, int c) const {
    if (p.scheme == 1) {
      double r = 0.5 * (B(a, c) + B(a - 1, c)) - (1 / 6.0) * ((U(a, c) > 0) ? d2bx(a - 1, c) : d2bx(a, c));
      return r * huu(a, c);
    }
    const double b_xm = B(a - 1, c) + 0.5 * kt_dx(a - 1, c) * p.dx;
    const double b_xp = B(a, c) - 0.5 * kt_dx(a, c) * p.dx;
    return ((U(a, c) > 0) ? b_xm : b_xp) * huu(a, c);
  }
  __device__ double hvb(int a, int c) const {
    if (p.scheme == 1) {
      double r = 0.5 * (B(a, c) + B(a, c - 1)) - (1 / 6.0) * ((V(a, c) > 0) ? d2by(a, c - 1) : d2by(a, c));
      return r * hvv(a, c);
    }
    const double b_ym = B(a, c - 1) + 0.5 * kt_dy(a, c - 1) * p.dy;
    const double b_yp = B(a, c) + 0.5 * kt_dy(a, c) * p.dy;
    return ((V(a, c) > 0) ? b_ym : b_yp) * hvv(a, c);
  }
  // thickness-weighted Laplacian of f over the face thickness (the K2 bracket and BB4's)
  template <typename F>
  __device__ double lap(F f, int a, int c) const {
    const double dxsq = p.dx * p.dx, dysq = p.dy * p.dy;
    return (Hw(a + 1, c) * (f(a + 1, c) - f(a, c)) - Hw(a, c) * (f(a, c) - f(a - 1, c))) / dxsq
         + (Hs(a, c + 1) * (f(a, c + 1) - f(a, c)) - Hs(a, c) * (f(a, c) - f(a, c - 1))) / dysq;
  }
  __device__ double BB4(int a, int c) const {
    return lap([&](int x, int y) { return B(x, y); }, a, c) / Hc(a, c);
  }
};

__global__ void tracer_kernel(const TracerParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.Nx || j >= p.Ny) return;
  const size_t lk = (size_t)k * p.lstride;
  const TView t{p, p.u + lk, p.v + lk, p.h + lk, p.b + lk};
  const size_t cell = (size_t)j * p.pitch + i;
  const double h = t.h[cell];
  const double bc = t.b[cell];
  double rhs_b = 0;
  double rhs_adv = 0;
  if (p.scheme == 0) {
    rhs_adv = -0.5 * (t.U(i + 1, j) * t.db_dx(i + 1, j) + t.U(i, j) * t.db_dx(i, j)
                      + t.V(i, j + 1) * t.db_dy(i, j + 1) + t.V(i, j) * t.db_dy(i, j));
  } else if (h != 0) {
    rhs_adv = -((t.hub(i + 1, j) - t.hub(i, j)) / p.dx + (t.hvb(i, j + 1) - t.hvb(i, j)) / p.dy) / h
            + bc * ((t.huu(i + 1, j) - t.huu(i, j)) / p.dx + (t.hvv(i, j + 1) - t.hvv(i, j)) / p.dy) / h;
  }
  rhs_b += rhs_adv;
  if (p.use_wdia && h != 0) {
    const double w0 = p.wdia[lk + cell], w1 = p.wdia[lk + p.lstride + cell];
    const double b_p = (k == 0) ? 0 : p.b[lk - p.lstride + cell];
    const double b_m = (k == p.L - 1) ? 0 : p.b[lk + p.lstride + cell];
    const double db_p = (w0 > 0) ? 0 : b_p - bc;
    const double db_m = (w1 > 0) ? bc - b_m : 0;
    const double rhs_wdia = -(w0 * db_p + w1 * db_m);
    rhs_b += rhs_wdia / h;
  }
  if (p.K2 > 0 && h != 0) {
    const double rhs_K2 = p.K2 * t.lap([&](int x, int y) { return t.B(x, y); }, i, j);
    rhs_b += rhs_K2 / h;
  }
  if (p.K4 > 0 && h != 0) {
    const double rhs_K4 = -p.K4 * t.lap([&](int x, int y) { return t.BB4(x, y); }, i, j);
    rhs_b += rhs_K4 / h;
  }
  const double bt = p.bTime[lk + cell];
  if (bt > 0) {
    const double rhs_relax = -(bc - p.bRelax[lk + cell]) / bt;
    rhs_b += rhs_relax;
  }
  const size_t o = lk + cell;
  if (p.ab_mode == 0) {
    p.fb_out[o] = rhs_b;
    return;
  }
  double bn;
  if (p.ab_mode == 1) bn = bc + p.c0 * rhs_b;
  else if (p.ab_mode == 2) bn = bc + (p.c0 * rhs_b - p.c1 * p.f1b[o]);
  else bn = bc + (p.c0 * rhs_b - p.c1 * p.f1b[o] + p.c2 * p.f2b[o]);
  if (p.write_hist) p.fb_out[o] = rhs_b;
  p.b_out[o] = bn;
}

}  // namespace

void launch_tracer(const TracerParams& p, cudaStream_t s) {
  dim3 b(32, 8), g((p.Nx + 31) / 32, (p.Ny + 7) / 8, p.L);
  tracer_kernel<<<g, b, 0, s>>>(p);
}

}  // namespace pawsim
