// tracer.cu -- passive tracer tendency and Adams-Bashforth update (see tracer.cuh).
//
// The ghost semantics are those of the fused tendency kernel: b is a scalar mirrored at
// walls; the face thickness h_west / h_south, which the reference re-fills after computing
// it, is evaluated at the mirrored owned position; the fields the reference computes over
// its ghost ring and never re-fills (h u, h v, the tracer gradients and fluxes, BB4) are
// evaluated directly at the ghost position. Expression order follows work.c:1947-2144 so that the results are those
// of the reference bit for bit (this file is compiled with -fmad=false).
#include "common.cuh"
#include "tracer.cuh"

namespace pawsim {

namespace {

// minmod of three slopes (defs.c:1000-1014)
__device__ inline double mm3(double x, double y, double z) {
  if ((x > 0) && (y > 0) && (z > 0)) return fmin(x, fmin(y, z));
  if ((x < 0) && (y < 0) && (z < 0)) return fmax(x, fmax(y, z));
  return 0;
}

// ---------------------------------------------------------------- tile kernel
// One CTA owns a TTX x TTY tile and walks its layers. u, v, h, b are staged in shared memory over a
// TH-cell halo with the boundary maps; then, in stages separated by barriers, the face
// thickness (at the mirrored owned position), the mass fluxes, the scheme's
// gradients or second differences, the tracer fluxes and BB4 are formed over the part of
// the halo the owned cells read; finally each thread forms its cell's tendency and AB update.
constexpr int TTX = 32, TTY = 16, TNT = TTX * TTY, TH = 3;
constexpr int TRW = TTX + 2 * TH, TRH = TTY + 2 * TH, TRN = TRW * TRH;
enum { T_U, T_V, T_H, T_B, T_HW, T_HS, T_HUU, T_HVV, T_X1, T_X2, T_HUB, T_HVB, T_BB4, T_NUM };

__global__ void __launch_bounds__(TNT) tracer_tile_kernel(const TracerParams p) {
  extern __shared__ double tsm[];
  double (*S)[TRN] = reinterpret_cast<double (*)[TRN]>(tsm);
  const int tid = threadIdx.x;
  const int X0 = blockIdx.x * TTX, Y0 = blockIdx.y * TTY;
  // tiles whose halo lies inside the domain load without boundary maps
  const bool inner = X0 - TH >= 0 && X0 + TTX + TH <= p.Nx && Y0 - TH >= 0 && Y0 + TTY + TH <= p.Ny;
  const double dx = p.dx, dy = p.dy;
  auto at = [](int x, int y) { return y * TRW + x; };
  // local index of the owned cell a filled field copies at local x (y): the MAP_S mirror
  auto mlx = [&](int lx) {
    if (!p.wall_ew) return lx;
    int g = X0 - TH + lx;
    if (g < 0) g = -g - 1;
    else if (g >= p.Nx) g = 2 * p.Nx - g - 1;
    return g - X0 + TH;
  };
  auto mly = [&](int ly) {
    if (!p.wall_ns) return ly;
    int g = Y0 - TH + ly;
    if (g < 0) g = -g - 1;
    else if (g >= p.Ny) g = 2 * p.Ny - g - 1;
    return g - Y0 + TH;
  };
  for (int k = 0; k < p.L; ++k) {
  const size_t lk = (size_t)k * p.lstride;
  const double *uk = p.u + lk, *vk = p.v + lk, *hk = p.h + lk, *bk = p.b + lk;
  __syncthreads();   // the previous layer's stages are done with the tile
  // stage 0: the layer's u, v, h, b with the reference's ghost values
  if (inner) {
    for (int q = tid; q < TRN; q += TNT) {
      const int lx = q % TRW, ly = q / TRW;
      const size_t g = (size_t)(Y0 - TH + ly) * p.pitch + (X0 - TH + lx);
      S[T_U][q] = uk[g];
      S[T_V][q] = vk[g];
      S[T_H][q] = hk[g];
      S[T_B][q] = bk[g];
    }
  } else {
    for (int q = tid; q < TRN; q += TNT) {
      const int lx = q % TRW, ly = q / TRW;
      const int gx = X0 - TH + lx, gy = Y0 - TH + ly;
      const bool in = gx >= -TH && gx < p.Nx + TH && gy >= -TH && gy < p.Ny + TH;
      if (in && p.corners && is_corner(gx, gy, p.Nx, p.Ny)) {
        S[T_U][q] = corner_load(p.corners, CF_U, k, p.L, gx, gy, p.Nx, p.Ny, MAP_S);
        S[T_V][q] = corner_load(p.corners, CF_V, k, p.L, gx, gy, p.Nx, p.Ny, MAP_N);
        S[T_H][q] = corner_load(p.corners, CF_H, k, p.L, gx, gy, p.Nx, p.Ny, MAP_S);
        S[T_B][q] = corner_load(p.corners, CF_B, k, p.L, gx, gy, p.Nx, p.Ny, MAP_S);
        continue;
      }
      S[T_U][q] = in ? load_mapped(uk, p.pitch, gx, gy, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_N, MAP_S) : 0.0;
      S[T_V][q] = in ? load_mapped(vk, p.pitch, gx, gy, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_N) : 0.0;
      S[T_H][q] = in ? load_mapped(hk, p.pitch, gx, gy, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_S) : 0.0;
      S[T_B][q] = in ? load_mapped(bk, p.pitch, gx, gy, p.Nx, p.Ny, p.wall_ew, p.wall_ns, MAP_S, MAP_S) : 0.0;
    }
  }
  __syncthreads();
  const double* SU = S[T_U];
  const double* SV = S[T_V];
  const double* SH = S[T_H];
  const double* SB = S[T_B];
  // face thickness of work.c:566-684 at local (i, j) of an owned cell
  auto face_w = [&](int i, int j) {
    auto Hh = [&](int a, int c) { return SH[at(a, c)]; };
    const int TS = p.thick_scheme;
    if (TS == 1)
      return (1.0 / 3) * (Hh(i, j) + Hh(i - 1, j) + 0.25 * (Hh(i, j + 1) + Hh(i - 1, j + 1) + Hh(i, j - 1) + Hh(i - 1, j - 1)));
    if (TS == 2 || TS == 3) {
      const double uc = SU[at(i, j)];
      if (TS == 2) {
        const double d2m = Hh(i, j) - 2 * Hh(i - 1, j) + Hh(i - 2, j);
        const double d2c = Hh(i + 1, j) - 2 * Hh(i, j) + Hh(i - 1, j);
        return 0.5 * (Hh(i, j) + Hh(i - 1, j)) - (1 / 6.0) * ((uc > 0) ? d2m : d2c);
      }
      const double sg = p.kt00_sigma;
      const double dm = mm3(sg * (Hh(i, j) - Hh(i - 1, j)), 0.5 * (Hh(i, j) - Hh(i - 2, j)), sg * (Hh(i - 1, j) - Hh(i - 2, j)));
      const double dc = mm3(sg * (Hh(i + 1, j) - Hh(i, j)), 0.5 * (Hh(i + 1, j) - Hh(i - 1, j)), sg * (Hh(i, j) - Hh(i - 1, j)));
      return (uc > 0) ? Hh(i - 1, j) + 0.5 * dm : Hh(i, j) - 0.5 * dc;
    }
    return 0.5 * (Hh(i, j) + Hh(i - 1, j));
  };
  auto face_s = [&](int i, int j) {
    auto Hh = [&](int a, int c) { return SH[at(a, c)]; };
    const int TS = p.thick_scheme;
    if (TS == 1)
      return (1.0 / 3) * (Hh(i, j) + Hh(i, j - 1) + 0.25 * (Hh(i + 1, j) + Hh(i - 1, j) + Hh(i + 1, j - 1) + Hh(i - 1, j - 1)));
    if (TS == 2 || TS == 3) {
      const double vc = SV[at(i, j)];
      if (TS == 2) {
        const double d2m = Hh(i, j) - 2 * Hh(i, j - 1) + Hh(i, j - 2);
        const double d2c = Hh(i, j + 1) - 2 * Hh(i, j) + Hh(i, j - 1);
        return 0.5 * (Hh(i, j) + Hh(i, j - 1)) - (1 / 6.0) * ((vc > 0) ? d2m : d2c);
      }
      const double sg = p.kt00_sigma;
      const double dm = mm3(sg * (Hh(i, j) - Hh(i, j - 1)), 0.5 * (Hh(i, j) - Hh(i, j - 2)), sg * (Hh(i, j - 1) - Hh(i, j - 2)));
      const double dc = mm3(sg * (Hh(i, j + 1) - Hh(i, j)), 0.5 * (Hh(i, j + 1) - Hh(i, j - 1)), sg * (Hh(i, j) - Hh(i, j - 1)));
      return (vc > 0) ? Hh(i, j - 1) + 0.5 * dm : Hh(i, j) + 0.5 * dc;
    }
    return 0.5 * (Hh(i, j) + Hh(i, j - 1));
  };
  // stage 1: face thickness (local 2 .. RW-2 / RH-2) and the scheme's gradients
  for (int q = tid; q < TRN; q += TNT) {
    const int lx = q % TRW, ly = q / TRW;
    if (lx >= 2 && lx <= TRW - 2 && ly >= 2 && ly <= TRH - 2) {
      // owned cells read the face thickness at most two cells beyond the domain; there the
      // mirrored owned position's stencil is inside the tile
      const int gx = X0 - TH + lx, gy = Y0 - TH + ly;
      const bool nr = gx >= -2 && gx < p.Nx + 2 && gy >= -2 && gy < p.Ny + 2;
      const int mx = mlx(lx), my = mly(ly);
      if (nr && p.corners && !inner && (gx < 0 || gx >= p.Nx)) {
        S[T_HW][q] = corner_face<true>(hk, uk, p.pitch, p.Nx, p.Ny, p.thick_scheme, p.kt00_sigma, p.corners, k, p.L,
                                       gx, gy);
        S[T_HS][q] = corner_face<false>(hk, vk, p.pitch, p.Nx, p.Ny, p.thick_scheme, p.kt00_sigma, p.corners, k, p.L,
                                        gx, gy);
      } else {
        S[T_HW][q] = nr ? face_w(mx, my) : 0.0;
        S[T_HS][q] = nr ? face_s(mx, my) : 0.0;
      }
    }
    if (lx >= 1 && lx <= TRW - 2 && ly >= 1 && ly <= TRH - 2) {
      if (p.scheme == 0) {
        S[T_X1][q] = SU[q] * div_rn(SB[q] - SB[q - 1], dx, p.rdx);
        S[T_X2][q] = SV[q] * div_rn(SB[q] - SB[q - TRW], dy, p.rdy);
      } else if (p.scheme == 1) {
        S[T_X1][q] = SB[q + 1] - 2 * SB[q] + SB[q - 1];
        S[T_X2][q] = SB[q + TRW] - 2 * SB[q] + SB[q - TRW];
      } else {
        const double sg = p.kt00_sigma;
        S[T_X1][q] = div_rn(mm3(sg * (SB[q + 1] - SB[q]), 0.5 * (SB[q + 1] - SB[q - 1]), sg * (SB[q] - SB[q - 1])), dx,
                            p.rdx);
        S[T_X2][q] = div_rn(mm3(sg * (SB[q + TRW] - SB[q]), 0.5 * (SB[q + TRW] - SB[q - TRW]), sg * (SB[q] - SB[q - TRW])),
                            dy, p.rdy);
      }
    }
  }
  __syncthreads();
  const double* HW = S[T_HW];
  const double* HS = S[T_HS];
  const double* X1 = S[T_X1];
  const double* X2 = S[T_X2];
  const double dxsq = dx * dx, dysq = dy * dy;
  // thickness-weighted Laplacian over the face thickness (the K2 bracket and BB4's)
  auto lap = [&](const double* F, int q) {
    return div_rn(HW[q + 1] * (F[q + 1] - F[q]) - HW[q] * (F[q] - F[q - 1]), dxsq, p.rdxsq)
         + div_rn(HS[q + TRW] * (F[q + TRW] - F[q]) - HS[q] * (F[q] - F[q - TRW]), dysq, p.rdysq);
  };
  // stage 2: mass fluxes, tracer fluxes (local 2 .. RW-2) and BB4 (owned +- 1)
  for (int q = tid; q < TRN; q += TNT) {
    const int lx = q % TRW, ly = q / TRW;
    if (lx >= 2 && lx <= TRW - 2 && ly >= 2 && ly <= TRH - 2) {
      const double huu = SU[q] * HW[q], hvv = SV[q] * HS[q];
      S[T_HUU][q] = huu;
      S[T_HVV][q] = hvv;
      if (p.scheme == 1) {
        double r = 0.5 * (SB[q] + SB[q - 1]) - (1 / 6.0) * ((SU[q] > 0) ? X1[q - 1] : X1[q]);
        S[T_HUB][q] = r * huu;
        r = 0.5 * (SB[q] + SB[q - TRW]) - (1 / 6.0) * ((SV[q] > 0) ? X2[q - TRW] : X2[q]);
        S[T_HVB][q] = r * hvv;
      } else if (p.scheme == 2) {
        const double b_xm = SB[q - 1] + 0.5 * X1[q - 1] * dx;
        const double b_xp = SB[q] - 0.5 * X1[q] * dx;
        const double b_ym = SB[q - TRW] + 0.5 * X2[q - TRW] * dy;
        const double b_yp = SB[q] + 0.5 * X2[q] * dy;
        S[T_HUB][q] = ((SU[q] > 0) ? b_xm : b_xp) * huu;
        S[T_HVB][q] = ((SV[q] > 0) ? b_ym : b_yp) * hvv;
      }
    }
    if (p.K4 > 0 && lx >= TH - 1 && lx <= TH + TTX && ly >= TH - 1 && ly <= TH + TTY)
      S[T_BB4][q] = lap(SB, q) / SH[q];
  }
  __syncthreads();
  // stage 3: the owned cell's tendency (work.c:2055-2140) and AB update
  const int tx = tid % TTX, ty = tid / TTX;
  const int i = X0 + tx, j = Y0 + ty;
  if (i < p.Nx && j < p.Ny) {
  const int q = at(tx + TH, ty + TH);
  const double* HUU = S[T_HUU];
  const double* HVV = S[T_HVV];
  const double* HUB = S[T_HUB];
  const double* HVB = S[T_HVB];
  const size_t cell = (size_t)j * p.pitch + i;
  const double h = SH[q];
  const double bc = SB[q];
  const double rh = 1.0 / h;   // reciprocal for div_rn by h
  double rhs_b = 0;
  double rhs_adv = 0;
  if (p.scheme == 0) {
    rhs_adv = -0.5 * (X1[q + 1] + X1[q] + X2[q + TRW] + X2[q]);
  } else if (h != 0) {
    rhs_adv = div_rn(-(div_rn(HUB[q + 1] - HUB[q], dx, p.rdx) + div_rn(HVB[q + TRW] - HVB[q], dy, p.rdy)), h, rh)
            + div_rn(bc * (div_rn(HUU[q + 1] - HUU[q], dx, p.rdx) + div_rn(HVV[q + TRW] - HVV[q], dy, p.rdy)), h, rh);
  }
  rhs_b += rhs_adv;
  double rhs_wdia = 0, rhs_K2 = 0, rhs_K4 = 0, rhs_relax = 0;
  if (p.use_wdia && h != 0) {
    const double w0 = p.wdia[lk + cell], w1 = p.wdia[lk + p.lstride + cell];
    const double b_p = (k == 0) ? 0 : p.b[lk - p.lstride + cell];
    const double b_m = (k == p.L - 1) ? 0 : p.b[lk + p.lstride + cell];
    double db_p = (w0 > 0) ? 0 : b_p - bc;
    double db_m = (w1 > 0) ? bc - b_m : 0;
    if (p.use_buoy) {
      db_p += (w0 > 0) ? 0 : p.gg[k];
      db_m += ((k + 1 < p.L) && (w1 > 0)) ? p.gg[k + 1] : 0;
    }
    rhs_wdia = -(w0 * db_p + w1 * db_m);
    rhs_b += div_rn(rhs_wdia, h, rh);
  }
  double rhs_diadiff = 0;
  if (p.use_diadiff && h != 0) {
    // Fdia_b at interfaces k and k+1 of this column: the surface flux on top, zero at the
    // bottom, kappa (db + gg with buoyancy) / dz between layers, plus convDiff where the
    // local reduced gravity is negative (diapycnal.c:165-190)
    auto fdia = [&](int kk) -> double {
      if (kk == 0) return p.fsurf[cell];
      if (kk == p.L) return 0.0;
      const double ba = p.b[(kk - 1) * p.lstride + cell], bb = p.b[kk * p.lstride + cell];
      double db = ba - bb;
      const double dz = 0.5 * (p.h[kk * p.lstride + cell] + p.h[(kk - 1) * p.lstride + cell]);
      double kappa = p.kappa[kk * p.lstride + cell];
      if (p.use_buoy) db += p.gg[kk];
      double gprime = p.gg[kk];
      if (p.use_buoy) gprime += ba - bb;
      if (p.conv_diff != 0 && gprime < 0) kappa += p.conv_diff;
      return dz != 0 ? kappa * db / dz : 0.0;
    };
    rhs_diadiff = fdia(k) - fdia(k + 1);
    rhs_b += div_rn(rhs_diadiff, h, rh);
  }
  if (p.K2 > 0 && h != 0) {
    rhs_K2 = p.K2 * lap(SB, q);
    rhs_b += div_rn(rhs_K2, h, rh);
  }
  if (p.K4 > 0 && h != 0) {
    rhs_K4 = -p.K4 * lap(S[T_BB4], q);
    rhs_b += div_rn(rhs_K4, h, rh);
  }
  const double bt = p.bTime[lk + cell];
  if (bt > 0) {
    rhs_relax = -(bc - p.bRelax[lk + cell]) / bt;
    rhs_b += rhs_relax;
  }
  if (p.bud_b) {
    // work.c:2131-2136
    double* f = p.bud_b + lk + cell;
    const size_t P = (size_t)p.L * p.lstride;   // one term's planes
    f[0] = f[0] + h * rhs_adv * p.dt;
    f[P] = f[P] + rhs_wdia * p.dt;
    f[2 * P] = f[2 * P] + rhs_K2 * p.dt;
    f[3 * P] = f[3 * P] + rhs_K4 * p.dt;
    f[4 * P] = f[4 * P] + rhs_diadiff * p.dt;
    f[5 * P] = f[5 * P] + h * rhs_relax * p.dt;
  }
  const size_t o = lk + cell;
  if (p.ab_mode == 0) {
    p.fb_out[o] = rhs_b;
  } else {
    double bn;
    if (p.ab_mode == 1) bn = bc + p.c0 * rhs_b;
    else if (p.ab_mode == 2) bn = bc + (p.c0 * rhs_b - p.c1 * p.f1b[o]);
    else bn = bc + (p.c0 * rhs_b - p.c1 * p.f1b[o] + p.c2 * p.f2b[o]);
    if (p.write_hist) p.fb_out[o] = rhs_b;
    p.b_out[o] = bn;
  }
  }   // owned cell
  }   // layer
}

}  // namespace

void launch_tracer(const TracerParams& p, cudaStream_t s) {
  constexpr size_t shm = (size_t)T_NUM * TRN * sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tracer_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    attr = true;
  }
  dim3 g((p.Nx + TTX - 1) / TTX, (p.Ny + TTY - 1) / TTY);
  tracer_tile_kernel<<<g, TNT, shm, s>>>(p);
}

}  // namespace pawsim
