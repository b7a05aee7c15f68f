// mg.cu -- GPU multigrid for the rigid-lid pressure equation (see mg.cuh).
#include <math.h>
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
};

template <typename T>
LV<T> view(const Multigrid::Level& l);
template <>
LV<double> view<double>(const Multigrid::Level& l) {
  return LV<double>{l.Nx, l.Ny, l.pitch, l.Ow, l.Os, l.Osum, l.rOsum, l.e, l.rhs, l.res};
}
template <>
LV<float> view<float>(const Multigrid::Level& l) {
  return LV<float>{l.Nx, l.Ny, l.pitch, l.Ow32, l.Os32, l.Osum32, l.rOsum32, l.e32, l.rhs32, l.res32};
}

#define IX(l, i, j) ((size_t)(j) * (l).pitch + (i))

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

// first red sweep from a zero initial guess: neighbours are zero
template <typename T>
__global__ void smooth_zero_kernel(LV<T> l, T omega) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny) return;
  size_t c = IX(l, i, j);
  l.e[c] = (((i + j) & 1) == 0) ? omega * l.rOsum[c] * (-l.rhs[c]) : T(0);
}

template <typename T>
__global__ void residual_kernel(LV<T> l) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny) return;
  size_t c = IX(l, i, j);
  l.res[c] = neighbour_sum(l, l.e, i, j) - l.Osum[c] * l.e[c] - l.rhs[c];
}

// residual of the fine level restricted by 2x2 means straight into the coarse rhs
// (multigrid.c:599-668); the coarse correction starts from zero
template <typename T>
__global__ void residual_restrict_kernel(LV<T> f, LV<T> c) {
  int ic = blockIdx.x * blockDim.x + threadIdx.x;
  int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (ic >= c.Nx || jc >= c.Ny) return;
  T r[4];
  int q = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      int i = 2 * ic + di, j = 2 * jc + dj;
      size_t x = IX(f, i, j);
      r[q++] = neighbour_sum(f, f.e, i, j) - f.Osum[x] * f.e[x] - f.rhs[x];
    }
  // order of restrict_power2_MG: (2i,2j) + (2i+1,2j) + (2i,2j+1) + (2i+1,2j+1)
  c.rhs[IX(c, ic, jc)] = T(0.25) * (r[0] + r[1] + r[2] + r[3]);
  c.e[IX(c, ic, jc)] = T(0);
}

// area-weighted restriction for uneven pairs (multigrid.c:681-740)
template <typename T>
__global__ void restrict_general_kernel(LV<T> f, const T* src, LV<T> c, T* dst) {
  int ic = blockIdx.x * blockDim.x + threadIdx.x;
  int jc = blockIdx.y * blockDim.y + threadIdx.y;
  if (ic >= c.Nx || jc >= c.Ny) return;
  double x0 = (double)ic * f.Nx / c.Nx, x1 = (double)(ic + 1) * f.Nx / c.Nx;
  double y0 = (double)jc * f.Ny / c.Ny, y1 = (double)(jc + 1) * f.Ny / c.Ny;
  double acc = 0, wsum = 0;
  for (int fi = (int)floor(x0); fi < (int)ceil(x1); ++fi) {
    double wx = fmin(x1, (double)(fi + 1)) - fmax(x0, (double)fi);
    if (wx <= 0) continue;
    for (int fj = (int)floor(y0); fj < (int)ceil(y1); ++fj) {
      double wy = fmin(y1, (double)(fj + 1)) - fmax(y0, (double)fj);
      if (wy <= 0) continue;
      double w = wx * wy;
      acc += w * (double)src[IX(f, fi, fj)];
      wsum += w;
    }
  }
  dst[IX(c, ic, jc)] = (T)(wsum > 0 ? acc / wsum : acc);
  c.e[IX(c, ic, jc)] = T(0);
}

// bilinear prolongation of the coarse correction, subtracted from the fine level
// (multigrid.c:376-442, 827-932, 986-1004)
template <typename T>
__global__ void prolong_correct_kernel(LV<T> f, LV<T> c, int power2, int wew, int wns) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= f.Nx || j >= f.Ny) return;
  T val;
  if (power2) {
    int hx = f.Nx / 2, hy = f.Ny / 2;
    int ip = (((i + 1) - (i + 1) % 2) / 2 + hx) % hx, im = (ip - 1 + hx) % hx;
    int jp = (((j + 1) - (j + 1) % 2) / 2 + hy) % hy, jm = (jp - 1 + hy) % hy;
    T ai = (i % 2 == 1) ? T(0.75) : T(0.25), bi = (i % 2 == 1) ? T(0.25) : T(0.75);
    T aj = (j % 2 == 1) ? T(0.75) : T(0.25), bj = (j % 2 == 1) ? T(0.25) : T(0.75);
    T wmm = ai * aj, wmp = ai * bj, wpm = bi * aj, wpp = bi * bj;
    if (wns) {
      if (j == 0) { wmm = 0; wpm = 0; wmp = ai; wpp = bi; }
      if (j == f.Ny - 1) { wmp = 0; wpp = 0; wmm = ai; wpm = bi; }
    }
    if (wew) {
      if (i == 0) { wmm = 0; wmp = 0; wpm = aj; wpp = bj; }
      if (i == f.Nx - 1) { wpm = 0; wpp = 0; wmm = aj; wmp = bj; }
    }
    if (wns && wew) {
      if (i == 0 && j == 0) { wmm = 0; wmp = 0; wpm = 0; wpp = 1; }
      if (i == 0 && j == f.Ny - 1) { wmm = 0; wmp = 0; wpm = 1; wpp = 0; }
      if (i == f.Nx - 1 && j == 0) { wmm = 0; wmp = 1; wpm = 0; wpp = 0; }
      if (i == f.Nx - 1 && j == f.Ny - 1) { wmm = 1; wmp = 0; wpm = 0; wpp = 0; }
    }
    val = wmm * c.e[IX(c, im, jm)] + wpm * c.e[IX(c, ip, jm)] + wmp * c.e[IX(c, im, jp)] + wpp * c.e[IX(c, ip, jp)];
  } else {
    double x = ((double)i + 0.5) * c.Nx / f.Nx - 0.5, y = ((double)j + 0.5) * c.Ny / f.Ny - 0.5, tx, ty;
    int imr, jmr;
    if (wew && x <= 0) { imr = 0; tx = 0; }
    else if (wew && x >= c.Nx - 1) { imr = c.Nx - 1; tx = 0; }
    else { imr = (int)floor(x); tx = x - imr; }
    if (wns && y <= 0) { jmr = 0; ty = 0; }
    else if (wns && y >= c.Ny - 1) { jmr = c.Ny - 1; ty = 0; }
    else { jmr = (int)floor(y); ty = y - jmr; }
    auto idx = [](int v, int n, int wall) {
      if (n <= 1) return 0;
      if (wall) return v < 0 ? 0 : (v >= n ? n - 1 : v);
      return ((v % n) + n) % n;
    };
    int im = idx(imr, c.Nx, wew), ip = idx(imr + 1, c.Nx, wew);
    int jm = idx(jmr, c.Ny, wns), jp = idx(jmr + 1, c.Ny, wns);
    val = (T)((1 - tx) * (1 - ty) * (double)c.e[IX(c, im, jm)] + tx * (1 - ty) * (double)c.e[IX(c, ip, jm)]
              + (1 - tx) * ty * (double)c.e[IX(c, im, jp)] + tx * ty * (double)c.e[IX(c, ip, jp)]);
  }
  f.e[IX(f, i, j)] -= val;
}

// max |pi - Jacobi(pi)| on the fine level (multigrid.c:1123-1156); NaNs are ignored like fmax
__global__ void max_residual_kernel(LV<double> l, unsigned long long* bits) {
  double m = 0;
  int n = l.Nx * l.Ny;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    int i = q % l.Nx, j = q / l.Nx;
    size_t c = IX(l, i, j);
    double r = l.e[c] - l.rOsum[c] * (neighbour_sum(l, l.e, i, j) - l.rhs[c]);
    m = fmax(m, fabs(r));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

// FP64 defect step: pi -= e32 (when `correct`), then r = L(pi) - rhs stored as FP32 on the
// fine FP32 level, plus the stopping measure of the updated pi
__global__ void defect_kernel(LV<double> l, const float* __restrict__ e32, int p32, float* r32, float* ez32,
                              int correct, unsigned long long* bits) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  double m = 0;
  if (i < l.Nx && j < l.Ny) {
    int ip1 = i + 1 == l.Nx ? 0 : i + 1, im1 = i == 0 ? l.Nx - 1 : i - 1;
    int jp1 = j + 1 == l.Ny ? 0 : j + 1, jm1 = j == 0 ? l.Ny - 1 : j - 1;
    auto P = [&](int a, int b) {
      double v = l.e[IX(l, a, b)];
      if (correct) v -= (double)e32[(size_t)b * p32 + a];
      return v;
    };
    double pc = P(i, j);
    double s = l.Os[IX(l, i, jp1)] * P(i, jp1) + l.Os[IX(l, i, j)] * P(i, jm1)
             + l.Ow[IX(l, ip1, j)] * P(ip1, j) + l.Ow[IX(l, i, j)] * P(im1, j);
    size_t c = IX(l, i, j);
    double crit = pc - l.rOsum[c] * (s - l.rhs[c]);
    m = fabs(crit);
    if (m != m) m = 0;
    r32[(size_t)j * p32 + i] = (float)(s - l.Osum[c] * pc - l.rhs[c]);
    ez32[(size_t)j * p32 + i] = 0.f;
    l.res[c] = pc;   // updated pi, copied back by commit_kernel
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

__global__ void commit_kernel(LV<double> l) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny) return;
  l.e[IX(l, i, j)] = l.res[IX(l, i, j)];
}

__global__ void zero_kernel_d(double* a, int Nx, int Ny, int pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < Nx && j < Ny) a[(size_t)j * pitch + i] = 0;
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
  // Hc on every level, reference arithmetic; host arrays are i-major like the reference
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
    L.e32 = dalloc<float>(np); L.rhs32 = dalloc<float>(np); L.res32 = dalloc<float>(np);
    good = good && L.e && L.rhs && L.res && L.e32 && L.rhs32 && L.res32;
  }
  dmax_ = dalloc<double>(2);
  dbits_ = dalloc<unsigned long long>(2);
  ok_ = good && dmax_ && dbits_;
}

Multigrid::~Multigrid() {
  for (auto& L : lv_) {
    cudaFree(L.Ow); cudaFree(L.Os); cudaFree(L.Osum); cudaFree(L.rOsum);
    cudaFree(L.Ow32); cudaFree(L.Os32); cudaFree(L.Osum32); cudaFree(L.rOsum32);
    cudaFree(L.e); cudaFree(L.rhs); cudaFree(L.res);
    cudaFree(L.e32); cudaFree(L.rhs32); cudaFree(L.res32);
  }
  cudaFree(dmax_);
  cudaFree(dbits_);
}

template <typename T>
void Multigrid::smooth(int n, int sweeps) {
  LV<T> l = view<T>(lv_[n]);
  if (n == (int)lv_.size() - 1 && sizeof(T) == 8) {
    l.e = reinterpret_cast<T*>(fine_pi_);
    l.rhs = const_cast<T*>(reinterpret_cast<const T*>(fine_rhs_));
  }
  for (int s = 0; s < sweeps; ++s) {
    smooth_kernel<T><<<g2(l.Nx, l.Ny), B2, 0, s_>>>(l, 0, (T)opt_.omega_rb);
    smooth_kernel<T><<<g2(l.Nx, l.Ny), B2, 0, s_>>>(l, 1, (T)opt_.omega_rb);
    g_launches += 2;
  }
}

template <typename T>
void Multigrid::vcycle(int n) {
  Level& F = lv_[n];
  LV<T> f = view<T>(F);
  if (n == 0) {
    // coarsest level (multigrid.c:461-511): a single cell carries no information
    if (F.Nx == 1 && F.Ny == 1) {
      cudaMemsetAsync(f.e, 0, sizeof(T), s_);
      return;
    }
  }
  smooth<T>(n, opt_.pre);
  if (n == 0) {
    smooth<T>(n, opt_.post);
    return;
  }
  LV<T> c = view<T>(lv_[n - 1]);
  if (F.power2) {
    residual_restrict_kernel<T><<<g2(c.Nx, c.Ny), B2, 0, s_>>>(f, c);
    ++g_launches;
  } else {
    g_launches += 2;
    residual_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f);
    restrict_general_kernel<T><<<g2(c.Nx, c.Ny), B2, 0, s_>>>(f, f.res, c, c.rhs);
  }
  vcycle<T>(n - 1);
  prolong_correct_kernel<T><<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, c, F.power2 ? 1 : 0, wew_, wns_);
  ++g_launches;
  smooth<T>(n, opt_.post);
}

double Multigrid::max_residual(const double* pi, int pitch, const double* rhs, int rhs_pitch) {
  Level& F = lv_.back();
  LV<double> f = view<double>(F);
  f.e = const_cast<double*>(pi);
  f.rhs = const_cast<double*>(rhs);
  (void)pitch; (void)rhs_pitch;
  cudaMemsetAsync(dbits_, 0, sizeof(unsigned long long), s_);
  max_residual_kernel<<<148, 256, 0, s_>>>(f, dbits_);
  ++g_launches;
  unsigned long long b = 0;
  cudaMemcpyAsync(&b, dbits_, sizeof(b), cudaMemcpyDeviceToHost, s_);
  cudaStreamSynchronize(s_);
  double m;
  memcpy(&m, &b, sizeof(m));
  return m;
}

int Multigrid::solve(double* pi, int pitch, const double* rhs, int rhs_pitch, double tol, int maxiters,
                     double* maxres_out) {
  const int top = (int)lv_.size() - 1;
  fine_pi_ = pi;
  fine_rhs_ = rhs;
  Level& F = lv_[top];
  int iters = 0;
  double maxres = tol + 1;
  if (!opt_.fp32_cycles) {
    // the fine level of the FP64 hierarchy works on the caller's pi and rhs
    double *se = F.e, *sr = F.rhs;
    F.e = pi;
    F.rhs = const_cast<double*>(rhs);
    while (maxres > tol && iters < maxiters) {
      vcycle<double>(top);
      maxres = max_residual(pi, pitch, rhs, rhs_pitch);
      ++iters;
    }
    F.e = se;
    F.rhs = sr;
  } else {
    LV<double> f = view<double>(F);
    f.e = pi;
    f.rhs = const_cast<double*>(rhs);
    int correct = 0;
    // the first defect step only forms the residual of the initial pi
    cudaMemsetAsync(dbits_, 0, sizeof(unsigned long long), s_);
    defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e32, F.pitch, F.rhs32, F.e32, correct, dbits_);
    ++g_launches;
    while (maxres > tol && iters < maxiters) {
      vcycle<float>(top);
      cudaMemsetAsync(dbits_, 0, sizeof(unsigned long long), s_);
      defect_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f, F.e32, F.pitch, F.rhs32, F.res32, 1, dbits_);
      commit_kernel<<<g2(f.Nx, f.Ny), B2, 0, s_>>>(f);
      g_launches += 2;
      // the zeroed correction for the next cycle was written to res32; swap the buffers
      float* t = F.e32; F.e32 = F.res32; F.res32 = t;
      unsigned long long b = 0;
      cudaMemcpyAsync(&b, dbits_, sizeof(b), cudaMemcpyDeviceToHost, s_);
      cudaStreamSynchronize(s_);
      memcpy(&maxres, &b, sizeof(maxres));
      ++iters;
    }
  }
  if (maxres_out) *maxres_out = maxres;
  return iters;
}

template void Multigrid::vcycle<double>(int);
template void Multigrid::vcycle<float>(int);

}  // namespace pawsim
