// dmg.cu -- the reference's distributed multigrid (pressureSolver 2) on the GPU (dmg.cuh).
#include <math.h>
#include <string.h>

#include <vector>

#include "common.cuh"
#include "dmg.cuh"
#include "pressure.cuh"

namespace pawsim {

namespace {

constexpr int DMG_PRE = 3, DMG_POST = 3, DMG_MIN = 8;

inline dim3 grid_of(int Nx, int Ny) { return dim3((Nx + 31) / 32, (Ny + 7) / 8); }
const dim3 BLK(32, 8);

// largest |v| of the block into *acc (bit pattern of a non-negative double)
__device__ inline void block_max(double v, unsigned long long* acc) {
  __shared__ double wm[8];
  const int t = threadIdx.x + threadIdx.y * blockDim.x;
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((t & 31) == 0) wm[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    double b = 0;
    for (int w = 0; w < 8; ++w) b = fmax(b, wm[w]);
    if (b > 0) atomicMax(acc, (unsigned long long)__double_as_longlong(b));
  }
}

struct LD {   // device view of a level
  int Nx, Ny;
  double *x, *rhs, *res;
  const double *Ow, *Os;
};

// operator coefficients around cell (i, j): west = Ow[i], east = Ow[i+1 mod Nx] (zero on a
// wall: the west face of cell 0 is stored as zero), likewise south/north
struct Nb {
  int ip, im, jp, jm;
  double Ow, Oe, Os, On;
};
__device__ inline Nb nbrs(const LD& l, int i, int j) {
  Nb n;
  n.ip = i + 1 == l.Nx ? 0 : i + 1;
  n.im = i == 0 ? l.Nx - 1 : i - 1;
  n.jp = j + 1 == l.Ny ? 0 : j + 1;
  n.jm = j == 0 ? l.Ny - 1 : j - 1;
  const size_t c = (size_t)j * l.Nx + i;
  n.Ow = l.Ow[c];
  n.Oe = l.Ow[(size_t)j * l.Nx + n.ip];
  n.Os = l.Os[c];
  n.On = l.Os[(size_t)n.jp * l.Nx + i];
  return n;
}

// one colour of a weighted sweep (pressure.c:1387-1438); with `track` the largest update
__global__ void dmg_smooth_kernel(LD l, int color, double omega, int track, unsigned long long* acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  double d = 0;
  if (i < l.Nx && j < l.Ny && ((i + j) & 1) == color) {
    const Nb n = nbrs(l, i, j);
    const double Osum = n.Ow + n.Oe + n.Os + n.On;
    if (Osum != 0) {
      const size_t c = (size_t)j * l.Nx + i;
      const double xo = l.x[c];
      const double xj = (n.Oe * l.x[(size_t)j * l.Nx + n.ip] + n.Ow * l.x[(size_t)j * l.Nx + n.im]
                         + n.On * l.x[(size_t)n.jp * l.Nx + i] + n.Os * l.x[(size_t)n.jm * l.Nx + i] - l.rhs[c])
                      / Osum;
      const double xn = xo + omega * (xj - xo);
      l.x[c] = xn;
      d = fabs(xn - xo);
    }
  }
  if (track) block_max(d, acc);
}

// res = rhs - L(x) (pressure.c:1441-1466)
__global__ void dmg_residual_kernel(LD l) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= l.Nx || j >= l.Ny) return;
  const Nb n = nbrs(l, i, j);
  const size_t c = (size_t)j * l.Nx + i;
  const double xc = l.x[c];
  l.res[c] = l.rhs[c] - (n.Oe * (l.x[(size_t)j * l.Nx + n.ip] - xc) + n.Ow * (l.x[(size_t)j * l.Nx + n.im] - xc)
                         + n.On * (l.x[(size_t)n.jp * l.Nx + i] - xc) + n.Os * (l.x[(size_t)n.jm * l.Nx + i] - xc));
}

// coarse rhs = 2x2 mean of the fine residual, coarse x = 0 (pressure.c:1469-1494)
__global__ void dmg_restrict_kernel(LD f, LD c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.Nx || j >= c.Ny) return;
  const double* r = f.res + (size_t)(2 * j) * f.Nx + 2 * i;
  c.rhs[(size_t)j * c.Nx + i] = 0.25 * (r[0] + r[1] + r[f.Nx] + r[f.Nx + 1]);
  c.x[(size_t)j * c.Nx + i] = 0;
}

// coarse index with the scalar ghost fill: periodic wrap, or the wall's mirror
__device__ inline int cidx(int a, int n, bool wall) {
  if (a < 0) return wall ? 0 : n - 1;
  if (a >= n) return wall ? n - 1 : 0;
  return a;
}

// fine x += bilinear coarse correction with 9/16, 3/16, 3/16, 1/16 (pressure.c:1547-1600)
__global__ void dmg_prolong_kernel(LD f, LD c, int wew, int wns, unsigned long long* acc) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y * blockDim.y + threadIdx.y;
  double d = 0;
  if (a < f.Nx && b < f.Ny) {
    const int ic = a >> 1, jc = b >> 1;
    const int di = (a & 1) ? 1 : -1, dj = (b & 1) ? 1 : -1;   // sw, se, nw, ne quadrants
    const int i2 = cidx(ic + di, c.Nx, wew), j2 = cidx(jc + dj, c.Ny, wns);
    auto X = [&](int i, int j) { return c.x[(size_t)j * c.Nx + i]; };
    const double e = 0.5625 * X(ic, jc) + 0.1875 * X(i2, jc) + 0.1875 * X(ic, j2) + 0.0625 * X(i2, j2);
    f.x[(size_t)b * f.Nx + a] += e;
    d = fabs(e);
  }
  block_max(d, acc);
}

// last level: red-black SOR from faces averaged out of Hc with modular indices, walls
// zeroed, until the largest update is at most tol (pressure.c:360-437), then the mean
// (summed x outer, y inner) removed. One CTA; the level has at most a few hundred cells.
__global__ void __launch_bounds__(1024) dmg_tail_kernel(int Nx, int Ny, double dx, double dy, double* x,
                                                        const double* rhs, const double* Hc, int wew, int wns,
                                                        double omega, double tol, int maxiters) {
  __shared__ double red[32];
  __shared__ double mu_s;
  const int n = Nx * Ny, t = threadIdx.x;
  auto Hw = [&](int i, int j) {
    if (wew && i == 0) return 0.0;
    const int im1 = (i + Nx - 1) % Nx;
    return 0.5 * (Hc[(size_t)j * Nx + i] + Hc[(size_t)j * Nx + im1]);
  };
  auto Hs = [&](int i, int j) {
    if (wns && j == 0) return 0.0;
    const int jm1 = (j + Ny - 1) % Ny;
    return 0.5 * (Hc[(size_t)j * Nx + i] + Hc[(size_t)jm1 * Nx + i]);
  };
  double mu = tol + 1;
  int iters = 0;
  while (mu > tol && iters < maxiters) {
    double m = 0;
    for (int color = 0; color < 2; ++color) {
      for (int q = t; q < n; q += blockDim.x) {
        const int i = q % Nx, j = q / Nx;
        if (((i + j) & 1) != color) continue;
        const int ip1 = (i + 1) % Nx, im1 = (i + Nx - 1) % Nx, jp1 = (j + 1) % Ny, jm1 = (j + Ny - 1) % Ny;
        const double Ow = Hw(i, j) / (dx * dx);
        const double Oe = (wew && i + 1 == Nx) ? 0.0 : Hw(ip1, j) / (dx * dx);
        const double Os = Hs(i, j) / (dy * dy);
        const double On = (wns && j + 1 == Ny) ? 0.0 : Hs(i, jp1) / (dy * dy);
        const double Osum = Ow + Oe + Os + On;
        if (Osum == 0) continue;
        const double old = x[(size_t)j * Nx + i];
        const double nv = (1 - omega) * old
                        + omega * (Oe * x[(size_t)j * Nx + ip1] + Ow * x[(size_t)j * Nx + im1]
                                   + On * x[(size_t)jp1 * Nx + i] + Os * x[(size_t)jm1 * Nx + i] - rhs[(size_t)j * Nx + i])
                              / Osum;
        x[(size_t)j * Nx + i] = nv;
        m = fmax(m, fabs(nv - old));
      }
      __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((t & 31) == 0) red[t >> 5] = m;
    __syncthreads();
    if (t == 0) {
      double b = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, red[w]);
      mu_s = b;
    }
    __syncthreads();
    mu = mu_s;
    ++iters;
    __syncthreads();
  }
  if (t == 0) {
    double mean = 0;
    for (int i = 0; i < Nx; ++i)
      for (int j = 0; j < Ny; ++j) mean += x[(size_t)j * Nx + i];
    mu_s = mean / ((double)Nx * (double)Ny);
  }
  __syncthreads();
  for (int q = t; q < n; q += blockDim.x) x[q] -= mu_s;
}

// level-0 copies between the model's pitched arrays and the dense level
__global__ void dmg_copy_kernel(double* dst, int dpitch, const double* src, int spitch, int Nx, int Ny) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < Nx && j < Ny) dst[(size_t)j * dpitch + i] = src[(size_t)j * spitch + i];
}

template <typename T> T* dalloc(size_t n, std::vector<void*>* own = nullptr) {
  T* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, n * sizeof(T));
  (void)own;
  return p;
}

LD view(const DMG::Level& L) { return LD{L.Nx, L.Ny, L.x, L.rhs, L.res, L.Ow, L.Os}; }

}  // namespace

bool DMG::can_start(int Nx, int Ny) { return Nx > DMG_MIN && Ny > DMG_MIN && Nx % 2 == 0 && Ny % 2 == 0; }

DMG::DMG(int Nx, int Ny, double Lx, double Ly, bool wall_ew, bool wall_ns, const double* Hc_host, double omega,
         double sor_rp, cudaStream_t s)
    : Nx_(Nx), Ny_(Ny), wew_(wall_ew), wns_(wall_ns), omega_(omega), sor_rp_(sor_rp), Lx_(Lx), Ly_(Ly), s_(s) {
  if (!can_start(Nx, Ny)) return;
  // host hierarchy of Hc, Hw, Hs (owned values; the level-0 faces are centred means of the
  // scalar-filled Hc, as the static geometry builds them)
  std::vector<std::vector<double>> Hc, Hw, Hs;
  std::vector<int> nx, ny;
  int lx = Nx, ly = Ny;
  while (true) {
    nx.push_back(lx);
    ny.push_back(ly);
    if (lx <= DMG_MIN || ly <= DMG_MIN || lx % 2 || ly % 2) break;
    lx = (lx + 1) / 2;
    ly = (ly + 1) / 2;
  }
  const int n = (int)nx.size();
  Hc.resize(n);
  Hw.resize(n);
  Hs.resize(n);
  Hc[0].assign(Hc_host, Hc_host + (size_t)Nx * Ny);
  Hw[0].resize((size_t)Nx * Ny);
  Hs[0].resize((size_t)Nx * Ny);
  auto fill = [](int a, int N, bool wall) { return a < 0 ? (wall ? 0 : N - 1) : a; };
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const int im = fill(i - 1, Nx, wall_ew), jm = fill(j - 1, Ny, wall_ns);
      Hw[0][(size_t)j * Nx + i] = 0.5 * (Hc[0][(size_t)j * Nx + i] + Hc[0][(size_t)j * Nx + im]);
      Hs[0][(size_t)j * Nx + i] = 0.5 * (Hc[0][(size_t)j * Nx + i] + Hc[0][(size_t)jm * Nx + i]);
    }
  for (int l = 1; l < n; ++l) {
    const int fx = nx[l - 1], cx = nx[l], cy = ny[l];
    Hc[l].resize((size_t)cx * cy);
    Hw[l].resize((size_t)cx * cy);
    Hs[l].resize((size_t)cx * cy);
    for (int j = 0; j < cy; ++j)
      for (int i = 0; i < cx; ++i) {
        auto F = [&](const std::vector<double>& v, int a, int b) { return v[(size_t)b * fx + a]; };
        const int a = 2 * i, b = 2 * j;
        Hc[l][(size_t)j * cx + i] = 0.25 * (F(Hc[l - 1], a, b) + F(Hc[l - 1], a + 1, b) + F(Hc[l - 1], a, b + 1)
                                            + F(Hc[l - 1], a + 1, b + 1));
        Hw[l][(size_t)j * cx + i] = 0.5 * (F(Hw[l - 1], a, b) + F(Hw[l - 1], a, b + 1));
        Hs[l][(size_t)j * cx + i] = 0.5 * (F(Hs[l - 1], a, b) + F(Hs[l - 1], a + 1, b));
      }
  }
  bool good = true;
  lv_.resize(n);
  for (int l = 0; l < n; ++l) {
    Level& L = lv_[l];
    L.Nx = nx[l];
    L.Ny = ny[l];
    const size_t N = (size_t)L.Nx * L.Ny;
    const double dx = Lx / L.Nx, dy = Ly / L.Ny;
    std::vector<double> Ow(N), Os(N);
    for (int j = 0; j < L.Ny; ++j)
      for (int i = 0; i < L.Nx; ++i) {
        Ow[(size_t)j * L.Nx + i] = (wall_ew && i == 0) ? 0.0 : Hw[l][(size_t)j * L.Nx + i] / (dx * dx);
        Os[(size_t)j * L.Nx + i] = (wall_ns && j == 0) ? 0.0 : Hs[l][(size_t)j * L.Nx + i] / (dy * dy);
      }
    L.x = dalloc<double>(N);
    L.rhs = dalloc<double>(N);
    L.res = dalloc<double>(N);
    L.Ow = dalloc<double>(N);
    L.Os = dalloc<double>(N);
    L.Hc = dalloc<double>(N);
    good = good && L.x && L.rhs && L.res && L.Ow && L.Os && L.Hc;
    if (!good) break;
    cudaMemcpy(L.Ow, Ow.data(), N * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(L.Os, Os.data(), N * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(L.Hc, Hc[l].data(), N * sizeof(double), cudaMemcpyHostToDevice);
  }
  acc_ = dalloc<unsigned long long>(1);
  scratch_ = dalloc<double>(reduce_scratch_elems(Nx, Ny) + 1);
  sum_ = dalloc<double>(1);
  ok_ = good && acc_ && scratch_ && sum_;
}

DMG::~DMG() {
  for (Level& L : lv_) {
    cudaFree(L.x); cudaFree(L.rhs); cudaFree(L.res); cudaFree(L.Ow); cudaFree(L.Os); cudaFree(L.Hc);
  }
  cudaFree(acc_);
  cudaFree(scratch_);
  cudaFree(sum_);
}

// pressure.c:2063-2123 (serial build: every transfer is local, the last level is the tail)
void DMG::vcycle(int l, unsigned long long* acc) {
  Level& L = lv_[l];
  LD d = view(L);
  const dim3 g = grid_of(L.Nx, L.Ny);
  if (l == (int)lv_.size() - 1) {
    const double dx = Lx_ / L.Nx, dy = Ly_ / L.Ny;
    dmg_tail_kernel<<<1, 1024, 0, s_>>>(L.Nx, L.Ny, dx, dy, L.x, L.rhs, L.Hc, wew_, wns_, sor_rp_, tol_, maxiters_);
    ++g_launches;
    return;
  }
  auto smooth = [&](int sweeps) {
    for (int q = 0; q < sweeps; ++q) {
      const int track = q == sweeps - 1;   // the measure takes the last sweep's updates
      dmg_smooth_kernel<<<g, BLK, 0, s_>>>(d, 0, omega_, track, acc);
      dmg_smooth_kernel<<<g, BLK, 0, s_>>>(d, 1, omega_, track, acc);
      g_launches += 2;
    }
  };
  smooth(DMG_PRE);
  dmg_residual_kernel<<<g, BLK, 0, s_>>>(d);
  Level& C = lv_[l + 1];
  LD c = view(C);
  dmg_restrict_kernel<<<grid_of(C.Nx, C.Ny), BLK, 0, s_>>>(d, c);
  g_launches += 2;
  vcycle(l + 1, acc);
  dmg_prolong_kernel<<<g, BLK, 0, s_>>>(d, c, wew_, wns_, acc);
  ++g_launches;
  smooth(DMG_POST);
}

int DMG::solve(double* pi, int pitch, const double* rhs, int rhs_pitch, double tol, int maxiters,
               double* last_update) {
  if (!ok_) return -1;
  tol_ = tol;
  maxiters_ = maxiters;
  Level& L0 = lv_[0];
  const dim3 g = grid_of(Nx_, Ny_);
  dmg_copy_kernel<<<g, BLK, 0, s_>>>(L0.x, Nx_, pi, pitch, Nx_, Ny_);
  dmg_copy_kernel<<<g, BLK, 0, s_>>>(L0.rhs, Nx_, rhs, rhs_pitch, Nx_, Ny_);
  g_launches += 2;
  const bool serial = (long long)Nx_ * Ny_ <= 65536;
  double mu = tol + 1;
  int cycles = 0;
  while (mu > tol && cycles < maxiters) {
    cudaMemsetAsync(acc_, 0, sizeof(unsigned long long), s_);
    vcycle(0, acc_);
    launch_sum(L0.x, Nx_, Ny_, Nx_, serial, scratch_, sum_, s_);
    launch_subtract_mean(L0.x, Nx_, Ny_, Nx_, sum_, s_);
    g_launches += serial ? 2 : 3;
    unsigned long long b = 0;
    if (cudaMemcpyAsync(&b, acc_, sizeof(b), cudaMemcpyDeviceToHost, s_) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s_) != cudaSuccess) return -1;
    memcpy(&mu, &b, sizeof(mu));
    ++cycles;
  }
  dmg_copy_kernel<<<g, BLK, 0, s_>>>(pi, pitch, L0.x, Nx_, Nx_, Ny_);
  ++g_launches;
  if (last_update) *last_update = mu;
  return cudaGetLastError() == cudaSuccess ? cycles : -1;
}

}  // namespace pawsim
