// warmstart.cu -- the learned pressure warm start (see warmstart.cuh).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "mg.cuh"
#include "nn.cuh"
#include "warmstart.cuh"

namespace pawsim {

using nn::bf16;

const WarmNet::LayerDef WarmNet::kLayers[WarmNet::NL] = {
    {16, 32, 0, 1}, {32, 32, 0, 1}, {32, 64, 1, 1}, {64, 64, 1, 1}, {64, 64, 2, 1},
    {64, 64, 3, 1}, {64, 64, 2, 1}, {64, 32, 1, 1}, {32, 32, 0, 1}, {32, 16, 0, 0}};

namespace {

constexpr int RED = 256;   // threads of the reduction kernels

// deterministic block sum of NV values per thread into part[block * NV + v]
template <int NV>
__device__ void block_sums(double (&v)[NV], double* part) {
  __shared__ double sh[NV][RED];
  const int t = threadIdx.x + threadIdx.y * blockDim.x;
  for (int k = 0; k < NV; ++k) sh[k][t] = v[k];
  __syncthreads();
  for (int s = RED / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int k = 0; k < NV; ++k) sh[k][t] += sh[k][t + s];
    __syncthreads();
  }
  if (t == 0) {
    const int b = blockIdx.x + blockIdx.y * gridDim.x;
    for (int k = 0; k < NV; ++k) part[(size_t)b * NV + k] = sh[k][0];
  }
}

// ---- network elementwise kernels (NHWC, C a multiple of 8) ----

__global__ void pool_bf16_kernel(const bf16* __restrict__ in, int B, int H, int W, int C, bf16* __restrict__ out) {
  const long long n = (long long)B * (H / 2) * (W / 2) * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    long long r = q / C;
    const int x = (int)(r % (W / 2));
    r /= (W / 2);
    const int y = (int)(r % (H / 2));
    const int b = (int)(r / (H / 2));
    const bf16* p = in + (((size_t)b * H + 2 * y) * W + 2 * x) * C + c;
    const float s = ((__bfloat162float(p[0]) + __bfloat162float(p[C])) + __bfloat162float(p[(size_t)W * C]))
                  + __bfloat162float(p[(size_t)W * C + C]);
    out[q] = __float2bfloat16_rn(0.25f * s);
  }
}

// out = up2(low) + skip
__global__ void up_add_bf16_kernel(const bf16* __restrict__ low, const bf16* __restrict__ skip, int B, int H, int W,
                                   int C, bf16* __restrict__ out) {
  const long long n = (long long)B * H * W * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    long long r = q / C;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    const float lo = __bfloat162float(low[(((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]);
    out[q] = __float2bfloat16_rn(lo + __bfloat162float(skip[q]));
  }
}

// g = bf16(act > 0 ? d : 0)
__global__ void relu_mask_kernel(const float* __restrict__ d, const bf16* __restrict__ act, long long n,
                                 bf16* __restrict__ g) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    g[q] = __float2bfloat16_rn(__bfloat162float(act[q]) > 0.f ? d[q] : 0.f);
}

// out (B, H/2, W/2, C) = sum of the 2x2 block of in (the gradient of nearest upsampling)
__global__ void pool_sum_kernel(const float* __restrict__ in, int B, int H, int W, int C, float* __restrict__ out) {
  const long long n = (long long)B * (H / 2) * (W / 2) * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    long long r = q / C;
    const int x = (int)(r % (W / 2));
    r /= (W / 2);
    const int y = (int)(r % (H / 2));
    const int b = (int)(r / (H / 2));
    const float* p = in + (((size_t)b * H + 2 * y) * W + 2 * x) * C + c;
    out[q] = ((p[0] + p[C]) + p[(size_t)W * C]) + p[(size_t)W * C + C];
  }
}

// dst (B, H, W, C) += 0.25 up2(src) (the gradient of 2x2 mean pooling)
__global__ void up_quarter_add_kernel(const float* __restrict__ src, int B, int H, int W, int C, float* __restrict__ dst) {
  const long long n = (long long)B * H * W * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    long long r = q / C;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    dst[q] += 0.25f * src[(((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
  }
}

// loss partial sums and the output gradient: dout ch0 = 2 (o - t) / n, other channels 0
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ tgt, long long n,
                            bf16* __restrict__ dout, double* part) {
  double v[1] = {0};
  const long long q = blockIdx.x * (long long)RED + threadIdx.x;
  if (q < n) {
    const float d = out[q * 16] - tgt[q];
    v[0] = (double)d * d;
    const float gv = 2.f * d / (float)n;
    dout[q * 16] = __float2bfloat16_rn(gv);
    for (int c = 1; c < 16; ++c) dout[q * 16 + c] = __float2bfloat16_rn(0.f);
  }
  block_sums<1>(v, part);
}

__global__ void finish_sum_kernel(const double* part, int nb, double scale, double* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int b = 0; b < nb; ++b) s += part[b];
    *dst = s * scale;
  }
}

__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, long long n, float lr_t, float b1, float b2, float eps) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    w[q] -= lr_t * mq / (sqrtf(vq) + eps);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ a, long long n, bf16* __restrict__ b) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = __float2bfloat16_rn(a[q]);
}

inline int grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (int)std::min<long long>(std::max<long long>(g, 1), 148 * 16);
}

// ---- warm-start kernels on the fine grid ----

// coarse F x F means of rhs, pi1 - pi2, pi1 and (optionally) pnew - 2 pi1 + pi2, with
// partial sums of cr^2, cd^2, cp, cp^2
__global__ void coarse_kernel(int F, const double* __restrict__ rhs, const double* __restrict__ pi1,
                              const double* __restrict__ pi2, const double* __restrict__ pnew, int pitch, int Hc,
                              int Wc, double* cr, double* cd, double* cp, double* ct, double* part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  double v[4] = {0, 0, 0, 0};
  if (i < Wc && j < Hc) {
    double sr = 0, sd = 0, sp = 0, st = 0;
    for (int b = 0; b < F; ++b)
      for (int a = 0; a < F; ++a) {
        const size_t g = (size_t)(j * F + b) * pitch + (i * F + a);
        const double p1 = pi1[g], p2 = pi2[g];
        sr += rhs[g];
        sd += p1 - p2;
        sp += p1;
        if (pnew) st += pnew[g] - (2 * p1 - p2);
      }
    const double inv = 1.0 / ((double)F * F);
    const size_t c = (size_t)j * Wc + i;
    cr[c] = sr * inv;
    cd[c] = sd * inv;
    cp[c] = sp * inv;
    if (pnew) ct[c] = st * inv;
    v[0] = cr[c] * cr[c];
    v[1] = cd[c] * cd[c];
    v[2] = cp[c];
    v[3] = cp[c] * cp[c];
  }
  block_sums<4>(v, part);
}

// scal = {s_d, s_p, mean_p, s_pp}
__global__ void scales_kernel(const double* part, int nb, double n, double* scal) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[4] = {0, 0, 0, 0};
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < 4; ++k) s[k] += part[(size_t)b * 4 + k];
  const double tiny = 1e-30;
  const double mean = s[2] / n;
  scal[0] = sqrt(s[0] / n) + tiny;
  scal[1] = sqrt(s[1] / n) + tiny;
  scal[2] = mean;
  scal[3] = sqrt(fmax(s[3] / n - mean * mean, 0.0)) + tiny;
}

// normalised inputs into (Hc, Wc, cstride) bf16 (channels 3.. zero)
__global__ void feat_kernel(const double* cr, const double* cd, const double* cp, const double* scal, int n,
                            int cstride, bf16* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  bf16* o = out + (size_t)q * cstride;
  o[0] = __float2bfloat16_rn((float)(cr[q] / scal[0]));
  o[1] = __float2bfloat16_rn((float)(cd[q] / scal[1]));
  o[2] = __float2bfloat16_rn((float)((cp[q] - scal[2]) / scal[3]));
  for (int c = 3; c < cstride; ++c) o[c] = __float2bfloat16_rn(0.f);
}

__global__ void target_kernel(const double* ct, const double* scal, int n, float* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) out[q] = (float)(ct[q] / scal[1]);
}

// batch b <- replay pair idx[b] (4 stored channels widened to 16)
__global__ void gather_kernel(const bf16* __restrict__ rx, const float* __restrict__ rt, const int* idx, int B,
                              int n, bf16* __restrict__ x, float* __restrict__ t) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= (long long)B * n) return;
  const int b = (int)(q / n), p = (int)(q % n);
  const size_t src = (size_t)idx[b] * n + p;
  bf16* o = x + q * 16;
  for (int c = 0; c < 4; ++c) o[c] = rx[src * 4 + c];
  for (int c = 4; c < 16; ++c) o[c] = __float2bfloat16_rn(0.f);
  t[q] = rt[src];
}

// pi = 2 pi1 - pi2 + s_p * P(d), P the cell-centred bilinear prolongation by F (clamped)
__global__ void guess_kernel(const float* __restrict__ out, int F, int Hc, int Wc, const double* __restrict__ pi1,
                             const double* __restrict__ pi2, const double* scal, int Nx, int Ny, int pitch,
                             double* __restrict__ pi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  double d;
  if (F == 1) {
    d = out[((size_t)j * Wc + i) * 16];
  } else {
    const double xc = (i + 0.5) / F - 0.5, yc = (j + 0.5) / F - 0.5;
    int i0 = (int)floor(xc), j0 = (int)floor(yc);
    const double tx = xc - i0, ty = yc - j0;
    const int i1 = min(i0 + 1, Wc - 1), j1 = min(j0 + 1, Hc - 1);
    i0 = max(i0, 0);
    j0 = max(j0, 0);
    auto o = [&](int a, int b) { return (double)out[((size_t)b * Wc + a) * 16]; };
    d = (1 - ty) * ((1 - tx) * o(i0, j0) + tx * o(i1, j0)) + ty * ((1 - tx) * o(i0, j1) + tx * o(i1, j1));
  }
  const size_t g = (size_t)j * pitch + i;
  pi[g] = 2 * pi1[g] - pi2[g] + scal[1] * d;
}

// keep pi(t-1) when the guess's measure (bits[0]) is not below that of pi(t-1) (bits[1])
__global__ void select_kernel(const unsigned long long* bits, const double* __restrict__ pi1, int Nx, int Ny,
                              int pitch, double* __restrict__ pi, int* decision) {
  const bool reject = !(__longlong_as_double((long long)bits[0]) < __longlong_as_double((long long)bits[1]));
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i == 0 && j == 0) *decision = reject ? 2 : 1;
  if (!reject || i >= Nx || j >= Ny) return;
  pi[(size_t)j * pitch + i] = pi1[(size_t)j * pitch + i];
}

// splitmix64 stream with Box-Muller normals, for a platform-independent initialisation
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double normal() { return sqrt(-2.0 * log(uniform())) * cos(6.283185307179586 * uniform()); }
};

}  // namespace

// ------------------------------------------------------------------ WarmNet

template <typename T>
T* WarmNet::alloc(size_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
  allocs_.push_back(p);
  return static_cast<T*>(p);
}

WarmNet::WarmNet(int H, int W, int Bmax, unsigned long long seed) : H_(H), W_(W), Bmax_(Bmax) {
  if (H % 8 || W % 8 || H < 8 || W < 8 || Bmax < 1) return;
  size_t off = 0;
  for (int l = 0; l < NL; ++l) {
    woff_[l] = off;
    off += (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
    boff_[l] = off;
    off += kLayers[l].cout;
  }
  nparam_ = off;
  w32_ = alloc<float>(nparam_);
  m_ = alloc<float>(nparam_);
  v_ = alloc<float>(nparam_);
  g_ = alloc<float>(nparam_);
  bool good = w32_ && m_ && v_ && g_;
  const size_t px0 = (size_t)Bmax * H * W;
  auto px = [&](int level) { return px0 >> (2 * level); };
  for (int l = 0; l < NL && good; ++l) {
    const size_t nw = (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
    wbf_[l] = alloc<bf16>(nw);
    wt_[l] = alloc<bf16>(nw);
    A_[l] = l < NL - 1 ? alloc<bf16>(px(kLayers[l].level) * kLayers[l].cout) : nullptr;
    G_[l] = l < NL - 1 ? alloc<float>(px(kLayers[l].level) * kLayers[l].cout) : nullptr;
    good = wbf_[l] && wt_[l] && (l == NL - 1 || (A_[l] && G_[l]));
  }
  P1_ = alloc<bf16>(px(1) * 32);
  P2_ = alloc<bf16>(px(2) * 64);
  P3_ = alloc<bf16>(px(3) * 64);
  U3_ = alloc<bf16>(px(2) * 64);
  U2_ = alloc<bf16>(px(1) * 64);
  U1_ = alloc<bf16>(px(0) * 32);
  dout_ = alloc<bf16>(px(0) * 16);
  gs_ = alloc<bf16>(px(0) * 32);
  out_ = alloc<float>(px(0) * 16);
  tmp_ = alloc<float>(std::max(px(1) * 32, px(2) * 64));
  part_ = alloc<double>((px(0) + RED - 1) / RED + 1);
  err_ = alloc<int>(1);
  good = good && P1_ && P2_ && P3_ && U3_ && U2_ && U1_ && dout_ && gs_ && out_ && tmp_ && part_ && err_;
  if (!good) return;
  // He-normal weights (the output layer scaled by 0.1 so the first guesses stay close to
  // the extrapolation), zero biases
  Rng rng{seed};
  std::vector<float> p(nparam_, 0.f);
  for (int l = 0; l < NL; ++l) {
    const double sd = sqrt(2.0 / (9.0 * kLayers[l].cin)) * (l == NL - 1 ? 0.1 : 1.0);
    for (size_t q = woff_[l]; q < boff_[l]; ++q) p[q] = (float)(sd * rng.normal());
  }
  ok_ = set_params(p.data()) == 0;
}

WarmNet::~WarmNet() {
  for (void* p : allocs_) cudaFree(p);
}

int WarmNet::refresh_bf16(cudaStream_t s) {
  for (int l = 0; l < NL; ++l) {
    const long long nw = (long long)kLayers[l].cout * 9 * kLayers[l].cin;
    to_bf16_kernel<<<grid_for(nw), 256, 0, s>>>(w32_ + woff_[l], nw, wbf_[l]);
    nn::flip_weights(wbf_[l], kLayers[l].cout, kLayers[l].cin, wt_[l], s);
    ++g_launches;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int WarmNet::set_params(const float* host) {
  if (cudaMemcpy(w32_, host, nparam_ * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  cudaMemset(m_, 0, nparam_ * sizeof(float));
  cudaMemset(v_, 0, nparam_ * sizeof(float));
  step_ = 0;
  int r = refresh_bf16(0);
  return r ? r : (cudaDeviceSynchronize() == cudaSuccess ? 0 : -1);
}

int WarmNet::get_params(float* host) const {
  return cudaMemcpy(host, w32_, nparam_ * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

int WarmNet::get_grads(float* host) const {
  return cudaMemcpy(host, g_, nparam_ * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

int WarmNet::forward(const bf16* in, int B, cudaStream_t s) {
  if (B < 1 || B > Bmax_) return -2;
  const int H = H_, W = W_;
  auto conv = [&](int l, const bf16* x, bf16* yb, float* yf) {
    const LayerDef& d = kLayers[l];
    return nn::conv3x3(x, B, H >> d.level, W >> d.level, d.cin, wbf_[l], w32_ + boff_[l], d.cout, d.relu != 0, yb,
                       yf, err_, s);
  };
  auto pool = [&](const bf16* x, int level, int C, bf16* y) {
    const long long n = (long long)B * (H >> (level + 1)) * (W >> (level + 1)) * C;
    pool_bf16_kernel<<<grid_for(n), 256, 0, s>>>(x, B, H >> level, W >> level, C, y);
    ++g_launches;
  };
  auto up_add = [&](const bf16* low, const bf16* skip, int level, int C, bf16* y) {
    const long long n = (long long)B * (H >> level) * (W >> level) * C;
    up_add_bf16_kernel<<<grid_for(n), 256, 0, s>>>(low, skip, B, H >> level, W >> level, C, y);
    ++g_launches;
  };
  int r = 0;
  r |= conv(0, in, A_[0], nullptr);
  r |= conv(1, A_[0], A_[1], nullptr);
  pool(A_[1], 0, 32, P1_);
  r |= conv(2, P1_, A_[2], nullptr);
  r |= conv(3, A_[2], A_[3], nullptr);
  pool(A_[3], 1, 64, P2_);
  r |= conv(4, P2_, A_[4], nullptr);
  pool(A_[4], 2, 64, P3_);
  r |= conv(5, P3_, A_[5], nullptr);
  up_add(A_[5], A_[4], 2, 64, U3_);
  r |= conv(6, U3_, A_[6], nullptr);
  up_add(A_[6], A_[3], 1, 64, U2_);
  r |= conv(7, U2_, A_[7], nullptr);
  up_add(A_[7], A_[1], 0, 32, U1_);
  r |= conv(8, U1_, A_[8], nullptr);
  r |= conv(9, A_[8], nullptr, out_);
  return r ? -1 : (cudaGetLastError() == cudaSuccess ? 0 : -1);
}

int WarmNet::backward(const bf16* in, const float* target, int B, double* loss_dev, cudaStream_t s) {
  if (B < 1 || B > Bmax_) return -2;
  const int H = H_, W = W_;
  int r = forward(in, B, s);
  if (r) return r;
  const long long n0 = (long long)B * H * W;
  const int nb = (int)((n0 + RED - 1) / RED);
  loss_kernel<<<nb, RED, 0, s>>>(out_, target, n0, dout_, part_);
  finish_sum_kernel<<<1, 1, 0, s>>>(part_, nb, 1.0 / (double)n0, loss_dev);
  g_launches += 2;
  cudaMemsetAsync(g_, 0, nparam_ * sizeof(float), s);
  const bf16* layer_in[NL] = {in, A_[0], P1_, A_[2], P2_, P3_, U3_, U2_, U1_, A_[8]};
  auto lvl = [&](int l) { return kLayers[l].level; };
  // gradient of layer l's output (FP32 G[l], or dout for the last layer) -> weight and bias
  // gradients, and the input gradient into `gin` (nullable)
  auto layer_back = [&](int l, float* gin) {
    const LayerDef& d = kLayers[l];
    const int h = H >> d.level, w = W >> d.level;
    const long long n = (long long)B * h * w * d.cout;
    const bf16* g = dout_;
    if (l != NL - 1) {
      relu_mask_kernel<<<grid_for(n), 256, 0, s>>>(G_[l], A_[l], n, gs_);
      ++g_launches;
      g = gs_;
    }
    int e = nn::conv3x3_wgrad(layer_in[l], g, B, h, w, d.cin, d.cout, g_ + woff_[l], g_ + boff_[l], err_, s);
    if (gin) e |= nn::conv3x3(g, B, h, w, d.cout, wt_[l], nullptr, d.cin, false, nullptr, gin, err_, s);
    return e;
  };
  auto pool_sum = [&](const float* x, int level, int C, float* y) {
    const long long n = (long long)B * (H >> (level + 1)) * (W >> (level + 1)) * C;
    pool_sum_kernel<<<grid_for(n), 256, 0, s>>>(x, B, H >> level, W >> level, C, y);
    ++g_launches;
  };
  auto up_q_add = [&](const float* x, int level, int C, float* y) {
    const long long n = (long long)B * (H >> level) * (W >> level) * C;
    up_quarter_add_kernel<<<grid_for(n), 256, 0, s>>>(x, B, H >> level, W >> level, C, y);
    ++g_launches;
  };
  r |= layer_back(9, G_[8]);
  r |= layer_back(8, G_[1]);            // U1 = up(A7) + A1
  pool_sum(G_[1], lvl(8), 32, G_[7]);
  r |= layer_back(7, G_[3]);            // U2 = up(A6) + A3
  pool_sum(G_[3], lvl(7), 64, G_[6]);
  r |= layer_back(6, G_[4]);            // U3 = up(A5) + A4
  pool_sum(G_[4], lvl(6), 64, G_[5]);
  r |= layer_back(5, tmp_);             // P3 = pool(A4)
  up_q_add(tmp_, lvl(4), 64, G_[4]);
  r |= layer_back(4, tmp_);             // P2 = pool(A3)
  up_q_add(tmp_, lvl(3), 64, G_[3]);
  r |= layer_back(3, G_[2]);
  r |= layer_back(2, tmp_);             // P1 = pool(A1)
  up_q_add(tmp_, lvl(1), 32, G_[1]);
  r |= layer_back(1, G_[0]);
  r |= layer_back(0, nullptr);
  return r ? -1 : (cudaGetLastError() == cudaSuccess ? 0 : -1);
}

int WarmNet::adam_step(float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  ++step_;
  const double c1 = 1 - pow((double)b1, step_), c2 = 1 - pow((double)b2, step_);
  const float lr_t = (float)(lr * sqrt(c2) / c1);
  adam_kernel<<<grid_for((long long)nparam_), 256, 0, s>>>(w32_, m_, v_, g_, (long long)nparam_, lr_t, b1, b2, eps);
  ++g_launches;
  return refresh_bf16(s);
}

// ------------------------------------------------------------------ WarmStart

int WarmStart::factor(int Nx, int Ny) {
  int F = 1;
  while (Nx / F > 256 || Ny / F > 256) F *= 2;
  if (Nx % (8 * F) || Ny % (8 * F) || Nx / F < 8 || Ny / F < 8) return 0;
  return F;
}

template <typename T>
T* WarmStart::alloc(size_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
  allocs_.push_back(p);
  return static_cast<T*>(p);
}

WarmStart::WarmStart(int Nx, int Ny, int pitch, int max_pairs, int batch, unsigned long long seed, cudaStream_t s)
    : Nx_(Nx), Ny_(Ny), pitch_(pitch), max_pairs_(max_pairs), batch_(batch) {
  (void)s;
  F_ = factor(Nx, Ny);
  if (!F_ || max_pairs < 1 || batch < 1) return;
  Hc_ = Ny / F_;
  Wc_ = Nx / F_;
  const size_t nf = (size_t)pitch * Ny, nc = (size_t)Hc_ * Wc_;
  const int nb = ((Wc_ + 31) / 32) * ((Hc_ + 7) / 8);
  pi1_ = alloc<double>(nf);
  pi2_ = alloc<double>(nf);
  cr_ = alloc<double>(nc);
  cd_ = alloc<double>(nc);
  cp_ = alloc<double>(nc);
  ct_ = alloc<double>(nc);
  part_ = alloc<double>((size_t)nb * 4);
  scal_ = alloc<double>(8);
  xin_ = alloc<bf16>((size_t)batch * nc * 16);
  rx_ = alloc<bf16>((size_t)max_pairs * nc * 4);
  rt_ = alloc<float>((size_t)max_pairs * nc);
  tgt_ = alloc<float>((size_t)batch * nc);
  idx_ = alloc<int>(batch);
  bits_ = alloc<unsigned long long>(2);
  decision_ = alloc<int>(1);
  loss_ = alloc<double>(1);
  if (!(pi1_ && pi2_ && cr_ && cd_ && cp_ && ct_ && part_ && scal_ && xin_ && rx_ && rt_ && tgt_ && idx_ && bits_ &&
        decision_ && loss_))
    return;
  net_ = new WarmNet(Hc_, Wc_, batch, seed);
  ok_ = net_->ok();
}

WarmStart::~WarmStart() {
  delete net_;
  for (void* p : allocs_) cudaFree(p);
}

void WarmStart::coarse(const double* rhs, const double* pnew, cudaStream_t s) {
  dim3 b(32, 8), g((Wc_ + 31) / 32, (Hc_ + 7) / 8);
  coarse_kernel<<<g, b, 0, s>>>(F_, rhs, pi1_, pi2_, pnew, pitch_, Hc_, Wc_, cr_, cd_, cp_, ct_, part_);
  scales_kernel<<<1, 1, 0, s>>>(part_, (int)(g.x * g.y), (double)Hc_ * Wc_, scal_);
  g_launches += 2;
}

int WarmStart::before_solve(double* pi, const double* rhs, Multigrid* mg, bool use, cudaStream_t s) {
  guessed_ = false;
  if (!ok_) return -1;
  cudaMemcpyAsync(pi1_, pi, (size_t)pitch_ * Ny_ * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (!use || !trained_ || hist_ < 2 || !mg) return 0;
  const int nc = Hc_ * Wc_;
  coarse(rhs, nullptr, s);
  feat_kernel<<<(nc + 255) / 256, 256, 0, s>>>(cr_, cd_, cp_, scal_, nc, 16, xin_);
  ++g_launches;
  if (net_->forward(xin_, 1, s)) return -1;
  dim3 b(32, 8), g((Nx_ + 31) / 32, (Ny_ + 7) / 8);
  guess_kernel<<<g, b, 0, s>>>(net_->out(), F_, Hc_, Wc_, pi1_, pi2_, scal_, Nx_, Ny_, pitch_, pi);
  ++g_launches;
  mg->measure2_async(pi, pi1_, rhs, bits_, s);
  select_kernel<<<g, b, 0, s>>>(bits_, pi1_, Nx_, Ny_, pitch_, pi, decision_);
  ++g_launches;
  guessed_ = true;
  return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

int WarmStart::after_solve(const double* pi, const double* rhs, bool collect, cudaStream_t s) {
  if (!ok_) return -1;
  // a pair needs pi(t-1) and pi(t-2) from earlier solves of this run
  if (collect && hist_ >= 2 && max_pairs_ > 0) {
    const int nc = Hc_ * Wc_;
    coarse(rhs, pi, s);
    feat_kernel<<<(nc + 255) / 256, 256, 0, s>>>(cr_, cd_, cp_, scal_, nc, 4, rx_ + (size_t)next_ * nc * 4);
    target_kernel<<<(nc + 255) / 256, 256, 0, s>>>(ct_, scal_, nc, rt_ + (size_t)next_ * nc);
    g_launches += 2;
    next_ = (next_ + 1) % max_pairs_;
    npairs_ = std::min(npairs_ + 1, max_pairs_);
  }
  std::swap(pi1_, pi2_);   // pi(t-1) of this step is pi(t-2) of the next
  ++hist_;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int WarmStart::last_decision(cudaStream_t s) {
  if (!guessed_) return 0;
  int d = 0;
  cudaMemcpyAsync(&d, decision_, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return d;
}

int WarmStart::train(int epochs, float lr, unsigned long long seed, double* loss, cudaStream_t s) {
  if (!ok_ || npairs_ < 1 || epochs < 1) return -1;
  const int nc = Hc_ * Wc_;
  std::vector<int> order(npairs_);
  for (int q = 0; q < npairs_; ++q) order[q] = q;
  Rng rng{seed};
  double last = 0;
  for (int e = 0; e < epochs; ++e) {
    for (int q = npairs_ - 1; q > 0; --q) std::swap(order[q], order[(size_t)(rng.next() % (uint64_t)(q + 1))]);
    double sum = 0;
    int nbat = 0;
    for (int k = 0; k < npairs_; k += batch_) {
      const int B = std::min(batch_, npairs_ - k);
      if (cudaMemcpyAsync(idx_, order.data() + k, B * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess) return -1;
      const long long n = (long long)B * nc;
      gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rx_, rt_, idx_, B, nc, xin_, tgt_);
      ++g_launches;
      if (net_->backward(xin_, tgt_, B, loss_, s)) return -1;
      if (net_->adam_step(lr, s)) return -1;
      double l = 0;
      if (cudaMemcpyAsync(&l, loss_, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
      if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
      sum += l;
      ++nbat;
    }
    last = sum / nbat;
  }
  int herr = 0;
  cudaMemcpy(&herr, net_->err(), sizeof(int), cudaMemcpyDeviceToHost);
  if (herr) return -3;
  if (loss) *loss = last;
  trained_ = true;
  return 0;
}

}  // namespace pawsim
