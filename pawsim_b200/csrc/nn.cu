// nn.cu -- 3x3 convolutions of the warm-start network on the tcgen05 tensor cores.
//
// Forward (and, with flipped weights, the input gradient) is an implicit GEMM with
// M = 128 output pixels per CTA, N = Cout, K = 9 * Cin in steps of 16 (one 3x3 tap and 16
// channels). The CTA keeps all of B (the weights, K-major) resident in shared memory and
// stages A (the shifted input pixels) in two buffers of four K steps; one thread issues
// tcgen05.mma into an FP32 accumulator in tensor memory and tcgen05.commit signals an
// mbarrier when a buffer may be refilled. The epilogue reads the accumulator with
// tcgen05.ld, adds the bias, applies ReLU and stores bf16 and/or FP32.
// The weight gradient is the GEMM D[(tap,ci)][co] = sum_p in[p+tap][ci] * dout[p][co] with
// K = pixels, on the same machinery; each CTA reduces a range of pixels and adds its FP32
// partial sums into the gradient with atomics.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout: core matrices of
// 8 rows x 16 bytes (8 bf16 along K) stored as 128 contiguous bytes; "SBO" is the byte
// distance between 8-row groups and "LBO" between the two 8-element halves of a K step.
// Every wait on an mbarrier is bounded: on time-out the kernel records an error in *err,
// waits once more (bounded) for its own tensor-core work, frees its tensor memory and
// returns.
#include <stdint.h>

#include <algorithm>

#include "../../include/pawsim_b200.h"
#include "common.cuh"
#include "nn.cuh"

namespace pawsim {
namespace nn {

namespace {

constexpr int MT = 128;                       // UMMA M: rows per CTA tile
constexpr int KS = 16;                        // K of one tcgen05.mma (bf16)
constexpr int RSTEPS = 4;                     // K steps staged per round
constexpr int NTH = 128;                      // one warpgroup
constexpr int A_STAGE = RSTEPS * 2 * (MT / 8) * 128;   // bytes of one A buffer (16 KB)
constexpr uint32_t LBO_A = (MT / 8) * 128;    // 2048 bytes between K halves of A
constexpr long long WAIT_LIMIT = 1LL << 22;   // polls of an mbarrier (with back-off)

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (bit layout of cute::UMMA::SmemDescriptor): start address,
// leading and stride byte offsets (all >> 4), version 1, no swizzle
__device__ inline uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16 (cute::UMMA::InstrDescriptor): FP32 D, BF16 A and B,
// both K-major, M = 128, N
__host__ __device__ constexpr uint32_t make_idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(MT >> 4) << 24);
}

__device__ inline void mbar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(b)) : "memory");
}

// bounded wait for the phase with the given parity; false when the limit ran out
__device__ inline bool mbar_wait(uint64_t* b, uint32_t parity) {
  const uint32_t a = smem_u32(b);
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (i > 64) __nanosleep(128);
  }
  return false;
}

__device__ inline void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(mask0), "r"(mask1), "r"(mask2),
        "r"(mask3)
      : "memory");
}

__device__ inline void umma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b))
               : "memory");
}

template <int NCOLS>
__device__ inline void tmem_alloc(uint32_t* dst) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "n"(NCOLS)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

template <int NCOLS>
__device__ inline void tmem_free(uint32_t base) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "n"(NCOLS) : "memory");
}

__device__ inline void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

template <int N>
__host__ __device__ constexpr int tmem_cols() {
  return N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
}

// Common prologue: barriers and tensor memory. Returns the accumulator's TMEM address.
template <int NCOLS>
__device__ inline uint32_t umma_setup(uint64_t* mbar, uint32_t* tmem_sh) {
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0]);
    mbar_init(&mbar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) tmem_alloc<NCOLS>(tmem_sh);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return *tmem_sh;
}

// Wait for the commit of the last issued round (it covers every earlier MMA of the CTA).
// True, for the whole CTA, when all `expected` rounds were issued and completed in time;
// otherwise the error is recorded and the CTA still waits (bounded) for what it issued.
__device__ inline bool umma_drain(uint64_t* mbar, int issued, int expected, int* err) {
  bool ok = issued == expected;
  if (issued > 0) {
    const int last = issued - 1;
    const uint32_t par = (uint32_t)((last >> 1) & 1);
    if (!mbar_wait(&mbar[last & 1], par)) {
      ok = false;
      mbar_wait(&mbar[last & 1], par);
    }
  }
  ok = !__syncthreads_or(!ok);
  if (!ok && threadIdx.x == 0 && err) atomicExch(err, 1);
  tc_fence_after();
  return ok;
}

// ------------------------------------------------------------------ forward convolution

template <int CIN, int COUT>
__global__ void __launch_bounds__(NTH) conv_fwd_kernel(const bf16* __restrict__ in, int B, int H, int W,
                                                       const bf16* __restrict__ w, const float* __restrict__ bias,
                                                       int relu, bf16* __restrict__ out_bf,
                                                       float* __restrict__ out_f32, int* err) {
  constexpr int K = 9 * CIN, S = K / KS, ROUNDS = (S + RSTEPS - 1) / RSTEPS;
  constexpr int NCOLS = tmem_cols<COUT>();
  constexpr int B_BYTES = COUT * K * 2;
  constexpr uint32_t LBO_B = (COUT / 8) * 128;
  constexpr uint32_t IDESC = make_idesc(COUT);
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sB = smem;
  unsigned char* sA = smem + B_BYTES;   // B_BYTES is a multiple of 128
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_sh;

  const int tid = threadIdx.x;
  const long long npix = (long long)B * H * W;
  const long long ntiles = (npix + MT - 1) / MT;
  // weights, K-major: 16-byte chunk (n, k8) at ((k8 * COUT/8) + n/8) * 128 + (n%8) * 16;
  // loaded once and kept for every tile this (persistent) CTA computes
  for (int q = tid; q < COUT * (K / 8); q += NTH) {
    const int n = q / (K / 8), k8 = q - n * (K / 8);
    const uint4 v = *reinterpret_cast<const uint4*>(w + (size_t)n * K + k8 * 8);
    *reinterpret_cast<uint4*>(sB + (k8 * (COUT / 8) + n / 8) * 128 + (n % 8) * 16) = v;
  }
  const uint32_t tmem = umma_setup<NCOLS>(mbar, &tmem_sh);
  int rg = 0;   // rounds issued by this CTA over all its tiles (mbarrier phases)
  bool ok = true;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long p = tile * MT + tid;   // this thread's output pixel (A row)
    int pb = 0, py = 0, px = 0;
    const bool pvalid = p < npix;
    if (pvalid) {
      px = (int)(p % W);
      const long long t = p / W;
      py = (int)(t % H);
      pb = (int)(t / H);
    }
    int issued = 0;
    for (int r = 0; r < ROUNDS; ++r) {
      const int buf = rg & 1;
      unsigned char* a = sA + buf * A_STAGE;
      const bool fail = rg >= 2 && !mbar_wait(&mbar[buf], (uint32_t)(((rg - 2) >> 1) & 1));
      if (__syncthreads_or(fail)) break;
      // stage this thread's row of A for the round's K steps
#pragma unroll
      for (int sl = 0; sl < RSTEPS; ++sl) {
        const int s = r * RSTEPS + sl;
        if (s >= S) break;
        const int tap = (s * KS) / CIN, ci0 = (s * KS) % CIN;
        const int yy = py + tap / 3 - 1, xx = px + tap % 3 - 1;
        uint4 v0 = make_uint4(0, 0, 0, 0), v1 = v0;
        if (pvalid && yy >= 0 && yy < H && xx >= 0 && xx < W) {
          const bf16* src = in + (((size_t)pb * H + yy) * W + xx) * CIN + ci0;
          v0 = *reinterpret_cast<const uint4*>(src);
          v1 = *reinterpret_cast<const uint4*>(src + 8);
        }
        unsigned char* dst = a + (2 * sl * (MT / 8) + tid / 8) * 128 + (tid % 8) * 16;
        *reinterpret_cast<uint4*>(dst) = v0;
        *reinterpret_cast<uint4*>(dst + LBO_A) = v1;
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t abase = smem_u32(a), bbase = smem_u32(sB);
        for (int sl = 0; sl < RSTEPS; ++sl) {
          const int s = r * RSTEPS + sl;
          if (s >= S) break;
          umma_bf16(tmem, make_desc(abase + 2 * sl * LBO_A, LBO_A, 128),
                    make_desc(bbase + 2 * s * LBO_B, LBO_B, 128), IDESC, s > 0 ? 1u : 0u);
        }
        umma_commit(&mbar[buf]);
      }
      ++issued;
      ++rg;
    }
    // wait for this tile's last commit (it covers every earlier MMA of the CTA)
    bool done = issued == ROUNDS;
    if (issued > 0) {
      const uint32_t par = (uint32_t)(((rg - 1) >> 1) & 1);
      if (!mbar_wait(&mbar[(rg - 1) & 1], par)) {
        done = false;
        mbar_wait(&mbar[(rg - 1) & 1], par);
      }
    }
    ok = !__syncthreads_or(!done);
    tc_fence_after();
    if (!ok) {
      if (tid == 0 && err) atomicExch(err, 1);
      break;
    }
    // row `tid` of the accumulator sits in TMEM lane tid (warp w reads lanes 32w..32w+31);
    // every lane takes part in the warp-wide loads, lanes without a pixel store nothing
    const uint32_t trow = tmem + ((uint32_t)((tid / 32) * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
      float v[8];
      tmem_ld8(trow + c0, v);
      if (!pvalid) continue;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (bias) v[i] += bias[c0 + i];
        if (relu) v[i] = fmaxf(v[i], 0.f);
      }
      if (out_f32) {
        float4* o = reinterpret_cast<float4*>(out_f32 + p * COUT + c0);
        o[0] = make_float4(v[0], v[1], v[2], v[3]);
        o[1] = make_float4(v[4], v[5], v[6], v[7]);
      }
      if (out_bf) {
        __align__(16) bf16 hv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) hv[i] = __float2bfloat16_rn(v[i]);
        *reinterpret_cast<uint4*>(out_bf + p * COUT + c0) = *reinterpret_cast<const uint4*>(hv);
      }
    }
    // the next tile's MMAs overwrite the accumulator only after every lane has read it
    tc_fence_before();
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) tmem_free<NCOLS>(tmem);
}

// ------------------------------------------------------------------ weight gradient

constexpr int WG_PIX_MAX = 2048;   // most pixels reduced by one CTA

template <int CIN, int COUT>
__global__ void __launch_bounds__(NTH) conv_wgrad_kernel(const bf16* __restrict__ in, const bf16* __restrict__ dout,
                                                         int B, int H, int W, int pix_per_cta, float* __restrict__ dw,
                                                         int* err) {
  constexpr int MROWS = 9 * CIN;          // rows (tap, ci) of the gradient
  constexpr int NCOLS = tmem_cols<COUT>();
  constexpr uint32_t LBO_B = (COUT / 8) * 128;
  constexpr int B_STAGE = RSTEPS * 2 * (COUT / 8) * 128;
  constexpr uint32_t IDESC = make_idesc(COUT);
  const int ROUNDS = pix_per_cta / (RSTEPS * KS);   // 64 pixels per round
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;                         // 2 x A_STAGE
  unsigned char* sB = smem + 2 * A_STAGE;           // 2 x B_STAGE
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_sh;

  const int tid = threadIdx.x;
  const int row0 = blockIdx.x * MT;                 // first (tap, ci) row of this tile
  const long long npix = (long long)B * H * W;
  const long long pix0 = (long long)blockIdx.y * pix_per_cta;
  const uint32_t tmem = umma_setup<NCOLS>(mbar, &tmem_sh);
  int issued = 0;
  for (int r = 0; r < ROUNDS; ++r) {
    const int buf = r & 1;
    unsigned char* a = sA + buf * A_STAGE;
    unsigned char* bm = sB + buf * B_STAGE;
    const bool fail = r >= 2 && !mbar_wait(&mbar[buf], (uint32_t)(((r - 2) >> 1) & 1));
    if (__syncthreads_or(fail)) break;
    // A: rows (tap, ci) x 64 pixels; one uint4 = 8 channels of one shifted pixel, scattered
    // into 8 rows at that pixel's K position
    for (int q = tid; q < 64 * (MT / 8); q += NTH) {
      const int kk = q % 64, g = q / 64;        // pixel within the round, 8-row group
      const int row = row0 + g * 8;
      __align__(16) bf16 v[8];
      *reinterpret_cast<uint4*>(v) = make_uint4(0, 0, 0, 0);
      const long long pp = pix0 + r * 64 + kk;
      if (row < MROWS && pp < npix) {
        const int tap = row / CIN, ci0 = row % CIN;
        const int x = (int)(pp % W);
        const long long t = pp / W;
        const int y = (int)(t % H), b = (int)(t / H);
        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
        if (yy >= 0 && yy < H && xx >= 0 && xx < W)
          *reinterpret_cast<uint4*>(v) =
              *reinterpret_cast<const uint4*>(in + (((size_t)b * H + yy) * W + xx) * CIN + ci0);
      }
      const int sl = kk / KS, kin = kk % KS;
      unsigned char* dst = a + ((2 * sl + kin / 8) * (MT / 8) + g) * 128 + (kin % 8) * 2;
#pragma unroll
      for (int j = 0; j < 8; ++j) *reinterpret_cast<bf16*>(dst + j * 16) = v[j];
    }
    // B: rows co x 64 pixels, from dout[p][co0..co0+7]
    for (int q = tid; q < 64 * (COUT / 8); q += NTH) {
      const int kk = q % 64, g = q / 64;
      __align__(16) bf16 v[8];
      *reinterpret_cast<uint4*>(v) = make_uint4(0, 0, 0, 0);
      const long long pp = pix0 + r * 64 + kk;
      if (pp < npix) *reinterpret_cast<uint4*>(v) = *reinterpret_cast<const uint4*>(dout + pp * COUT + g * 8);
      const int sl = kk / KS, kin = kk % KS;
      unsigned char* dst = bm + ((2 * sl + kin / 8) * (COUT / 8) + g) * 128 + (kin % 8) * 2;
#pragma unroll
      for (int j = 0; j < 8; ++j) *reinterpret_cast<bf16*>(dst + j * 16) = v[j];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t abase = smem_u32(a), bbase = smem_u32(bm);
      for (int sl = 0; sl < RSTEPS; ++sl)
        umma_bf16(tmem, make_desc(abase + 2 * sl * LBO_A, LBO_A, 128), make_desc(bbase + 2 * sl * LBO_B, LBO_B, 128),
                  IDESC, (r > 0 || sl > 0) ? 1u : 0u);
      umma_commit(&mbar[buf]);
    }
    ++issued;
  }
  const bool ok = umma_drain(mbar, issued, ROUNDS, err);
  if (ok) {
    const uint32_t trow = tmem + ((uint32_t)((tid / 32) * 32) << 16);
    const int row = row0 + tid;
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
      float v[8];
      tmem_ld8(trow + c0, v);
      if (row < MROWS)
#pragma unroll
        for (int i = 0; i < 8; ++i) atomicAdd(dw + (size_t)(c0 + i) * MROWS + row, v[i]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) tmem_free<NCOLS>(tmem);
}

// db[co] += sum_p dout[p][co]
__global__ void bias_grad_kernel(const bf16* __restrict__ dout, long long npix, int C, float* __restrict__ db) {
  __shared__ float acc[64];
  if (threadIdx.x < 64) acc[threadIdx.x] = 0;
  __syncthreads();
  const int c = threadIdx.x % C;
  float s = 0;
  for (long long p = (long long)blockIdx.x * (blockDim.x / C) + threadIdx.x / C; p < npix;
       p += (long long)gridDim.x * (blockDim.x / C))
    if (threadIdx.x < (blockDim.x / C) * C) s += __bfloat162float(dout[p * C + c]);
  if (threadIdx.x < (blockDim.x / C) * C) atomicAdd(&acc[c], s);
  __syncthreads();
  if (threadIdx.x < C) atomicAdd(db + threadIdx.x, acc[threadIdx.x]);
}

__global__ void flip_kernel(const bf16* __restrict__ w, int Cout, int Cin, bf16* __restrict__ wt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Cout * 9 * Cin) return;
  const int ci = q % Cin, tap = (q / Cin) % 9, co = q / (9 * Cin);
  wt[((size_t)ci * 9 + (8 - tap)) * Cout + co] = w[q];
}

template <int CIN, int COUT>
int launch_fwd(const bf16* in, int B, int H, int W, const bf16* w, const float* bias, bool relu, bf16* ob,
               float* of, int* err, cudaStream_t s) {
  constexpr int K = 9 * CIN;
  const size_t smem = (size_t)COUT * K * 2 + 2 * A_STAGE;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(conv_fwd_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return -1;
    attr = true;
  }
  static int per_sm = 0, nsm = 0;
  if (!per_sm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv_fwd_kernel<CIN, COUT>, NTH, smem) != cudaSuccess)
      per_sm = 0;
    // shared memory is the binding limit (each CTA holds the weights and two A stages; the
    // tensor memory of 4 CTAs x 64 columns fits the SM's 512)
    const int by_smem = (int)((227u * 1024u) / (smem + 1024));
    per_sm = std::max(per_sm, std::min(4, std::max(1, by_smem)));
  }
  const long long ntiles = ((long long)B * H * W + MT - 1) / MT;
  const unsigned grid = (unsigned)std::min<long long>(ntiles, (long long)nsm * per_sm);
  conv_fwd_kernel<CIN, COUT><<<grid, NTH, smem, s>>>(in, B, H, W, w, bias, relu ? 1 : 0, ob, of, err);
  ++g_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <int CIN, int COUT>
int launch_wgrad(const bf16* in, const bf16* dout, int B, int H, int W, float* dw, int* err, cudaStream_t s) {
  const size_t smem = 2 * (size_t)A_STAGE + 2 * (size_t)(RSTEPS * 2 * (COUT / 8) * 128);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(conv_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return -1;
    attr = true;
  }
  const long long npix = (long long)B * H * W;
  // pixels per CTA: a multiple of 64, small enough that the grid covers about 4 CTAs per SM
  const int mtiles = (9 * CIN + MT - 1) / MT;
  long long per = (npix * mtiles + 4 * 148 - 1) / (4 * 148);
  per = std::min<long long>(WG_PIX_MAX, std::max<long long>(64, (per + 63) / 64 * 64));
  dim3 grid(mtiles, (unsigned)((npix + per - 1) / per));
  conv_wgrad_kernel<CIN, COUT><<<grid, NTH, smem, s>>>(in, dout, B, H, W, (int)per, dw, err);
  ++g_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

#define PAWSIM_NN_DISPATCH(FN, CIN, COUT, ...)                                   \
  switch (CIN * 1000 + COUT) {                                                     \
    case 16016: return FN<16, 16>(__VA_ARGS__);                                    \
    case 16032: return FN<16, 32>(__VA_ARGS__);                                    \
    case 16048: return FN<16, 48>(__VA_ARGS__);                                    \
    case 16064: return FN<16, 64>(__VA_ARGS__);                                    \
    case 32016: return FN<32, 16>(__VA_ARGS__);                                    \
    case 32032: return FN<32, 32>(__VA_ARGS__);                                    \
    case 32048: return FN<32, 48>(__VA_ARGS__);                                    \
    case 32064: return FN<32, 64>(__VA_ARGS__);                                    \
    case 48016: return FN<48, 16>(__VA_ARGS__);                                    \
    case 48032: return FN<48, 32>(__VA_ARGS__);                                    \
    case 48048: return FN<48, 48>(__VA_ARGS__);                                    \
    case 48064: return FN<48, 64>(__VA_ARGS__);                                    \
    case 64016: return FN<64, 16>(__VA_ARGS__);                                    \
    case 64032: return FN<64, 32>(__VA_ARGS__);                                    \
    case 64048: return FN<64, 48>(__VA_ARGS__);                                    \
    case 64064: return FN<64, 64>(__VA_ARGS__);                                    \
    default: return -2;                                                            \
  }

}  // namespace

int conv3x3(const bf16* in, int B, int H, int W, int Cin, const bf16* w, const float* bias, int Cout, bool relu,
            bf16* out_bf, float* out_f32, int* err, cudaStream_t s) {
  if (B < 1 || H < 1 || W < 1) return -2;
  PAWSIM_NN_DISPATCH(launch_fwd, Cin, Cout, in, B, H, W, w, bias, relu, out_bf, out_f32, err, s)
}

int conv3x3_wgrad(const bf16* in, const bf16* dout, int B, int H, int W, int Cin, int Cout, float* dw, float* db,
                  int* err, cudaStream_t s) {
  if (B < 1 || H < 1 || W < 1) return -2;
  if (db) {
    const long long npix = (long long)B * H * W;
    int blocks = (int)((npix + 255) / 256);
    if (blocks > 1184) blocks = 1184;
    bias_grad_kernel<<<blocks, 256, 0, s>>>(dout, npix, Cout, db);
    ++g_launches;
  }
  PAWSIM_NN_DISPATCH(launch_wgrad, Cin, Cout, in, dout, B, H, W, dw, err, s)
}

int flip_weights(const bf16* w, int Cout, int Cin, bf16* w_t, cudaStream_t s) {
  const int n = Cout * 9 * Cin;
  flip_kernel<<<(n + 255) / 256, 256, 0, s>>>(w, Cout, Cin, w_t);
  ++g_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace nn
}  // namespace pawsim

extern "C" {

PAWSIM_API int pawsim_nn_conv3x3(const void* in, int B, int H, int W, int Cin, const void* w, const float* bias,
                                 int Cout, int relu, void* out_bf16, float* out_f32, int* dev_err, void* stream) {
  using namespace pawsim;
  if (!in || !w || (!out_bf16 && !out_f32)) return PAWSIM_GPU_EBADCONFIG;
  int r = nn::conv3x3(static_cast<const nn::bf16*>(in), B, H, W, Cin, static_cast<const nn::bf16*>(w), bias, Cout,
                      relu != 0, static_cast<nn::bf16*>(out_bf16), out_f32, dev_err,
                      static_cast<cudaStream_t>(stream));
  if (r == -2) return PAWSIM_GPU_EUNSUPPORTED;
  return r ? set_cuda_error(cudaGetLastError(), "pawsim_nn_conv3x3", __FILE__, __LINE__) : 0;
}

PAWSIM_API int pawsim_nn_conv3x3_wgrad(const void* in, const void* dout, int B, int H, int W, int Cin, int Cout,
                                       float* dw, float* db, int* dev_err, void* stream) {
  using namespace pawsim;
  if (!in || !dout || !dw) return PAWSIM_GPU_EBADCONFIG;
  int r = nn::conv3x3_wgrad(static_cast<const nn::bf16*>(in), static_cast<const nn::bf16*>(dout), B, H, W, Cin,
                            Cout, dw, db, dev_err, static_cast<cudaStream_t>(stream));
  if (r == -2) return PAWSIM_GPU_EUNSUPPORTED;
  return r ? set_cuda_error(cudaGetLastError(), "pawsim_nn_conv3x3_wgrad", __FILE__, __LINE__) : 0;
}

PAWSIM_API int pawsim_nn_flip_weights(const void* w, int Cout, int Cin, void* w_t, void* stream) {
  using namespace pawsim;
  if (!w || !w_t) return PAWSIM_GPU_EBADCONFIG;
  int r = nn::flip_weights(static_cast<const nn::bf16*>(w), Cout, Cin, static_cast<nn::bf16*>(w_t),
                           static_cast<cudaStream_t>(stream));
  return r ? set_cuda_error(cudaGetLastError(), "pawsim_nn_flip_weights", __FILE__, __LINE__) : 0;
}

}  // extern "C"
