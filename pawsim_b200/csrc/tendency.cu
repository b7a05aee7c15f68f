// tendency.cu -- chooses the tile height of the fused tendency kernel (tendency_tile.cu).
//
// Every height computes the same values. Tiles are 32 cells wide; 32 x 12 tiles (384 threads)
// run three CTAs per SM when three fit in its shared memory, 32 x 16 tiles (512 threads) two,
// then 32 x 12 tiles two, and 32 x 8 tiles (256 threads) take what is left.
// Taller tiles spend fewer halo evaluations per owned cell; more resident warps hide more
// latency. Measured on the lean 2048 x 2048 x 2 gyre step: 32 x 12 at three CTAs 0.672 ms,
// 32 x 16 at two 0.690 ms.
#include <cuda_runtime.h>

#include "tendency.cuh"

namespace pawsim {

size_t tendency_smem_ty8(const TendParams& p, int ts);
size_t tendency_smem_ty12(const TendParams& p, int ts);
size_t tendency_smem_ty16(const TendParams& p, int ts);
// one translation unit per tile height and momentum scheme (compiled in parallel)
#define PAWSIM_DECL_TEND(TY)                                                   \
  int launch_tendency_ty##TY##_m0(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m1(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m2(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m3(const TendParams& p, int ms, int ts, cudaStream_t s);
PAWSIM_DECL_TEND(8)
PAWSIM_DECL_TEND(12)
PAWSIM_DECL_TEND(16)
#undef PAWSIM_DECL_TEND
#define PAWSIM_DECL_BATCH(TY, M)                                                                         \
  int batch_launch_tendency_ty##TY##_m##M(const TendParams& p0, const TendParams* ps, const int* work, \
                                           int nwork, int members, int* done, int ms, int ts, cudaStream_t s);
PAWSIM_DECL_BATCH(8, 0) PAWSIM_DECL_BATCH(8, 1) PAWSIM_DECL_BATCH(8, 2) PAWSIM_DECL_BATCH(8, 3)
PAWSIM_DECL_BATCH(12, 0) PAWSIM_DECL_BATCH(12, 1) PAWSIM_DECL_BATCH(12, 2) PAWSIM_DECL_BATCH(12, 3)
PAWSIM_DECL_BATCH(16, 0) PAWSIM_DECL_BATCH(16, 1) PAWSIM_DECL_BATCH(16, 2) PAWSIM_DECL_BATCH(16, 3)
#undef PAWSIM_DECL_BATCH
int launch_tendency_budget_tile(const TendParams& p, int ms, int ts, cudaStream_t s);

int tendency_tile_height(const TendParams& p, int ts) {
  // 228 KB of shared memory per SM, 1 KB reserved per CTA
  constexpr size_t kThreePerSM = 74 * 1024, kTwoPerSM = 113 * 1024;
  if (tendency_smem_ty12(p, ts) <= kThreePerSM) return 12;
  if (tendency_smem_ty16(p, ts) <= kTwoPerSM) return 16;
  // 32 x 12 at two CTAs (24 warps) beats 32 x 8 at two (16 warps): 0.82 against 1.07 ms on
  // the 1024 x 1024 x 4 full-physics set-up (A4, w_dia, restoring)
  if (tendency_smem_ty12(p, ts) <= kTwoPerSM) return 12;
  return 8;
}

int launch_tendency(const TendParams& p, int ms, int ts, cudaStream_t s) {
#define PAWSIM_TEND_CASE(M)                                           \
  case M:                                                             \
    switch (ty) {                                                     \
      case 12: return launch_tendency_ty12_m##M(p, ms, ts, s);        \
      case 16: return launch_tendency_ty16_m##M(p, ms, ts, s);        \
      default: return launch_tendency_ty8_m##M(p, ms, ts, s);         \
    }
  const int ty = tendency_tile_height(p, ts);
  switch (ms) {
    PAWSIM_TEND_CASE(0)
    PAWSIM_TEND_CASE(1)
    PAWSIM_TEND_CASE(2)
    PAWSIM_TEND_CASE(3)
  }
#undef PAWSIM_TEND_CASE
  return -1;
}

int launch_tendency_budget(const TendParams& p, int ms, int ts, cudaStream_t s) {
  return launch_tendency_budget_tile(p, ms, ts, s);
}

int launch_tendency_batch(const TendParams& p0, const TendParams* ps, const int* work, int nwork, int members,
                          int* done, int ms, int ts, cudaStream_t s) {
  const int ty = tendency_tile_height(p0, ts);
#define PAWSIM_BATCH_CASE(M)                                                                               \
  case M:                                                                                                  \
    switch (ty) {                                                                                          \
      case 12: return batch_launch_tendency_ty12_m##M(p0, ps, work, nwork, members, done, ms, ts, s);      \
      case 16: return batch_launch_tendency_ty16_m##M(p0, ps, work, nwork, members, done, ms, ts, s);      \
      default: return batch_launch_tendency_ty8_m##M(p0, ps, work, nwork, members, done, ms, ts, s);       \
    }
  switch (ms) {
    PAWSIM_BATCH_CASE(0)
    PAWSIM_BATCH_CASE(1)
    PAWSIM_BATCH_CASE(2)
    PAWSIM_BATCH_CASE(3)
  }
#undef PAWSIM_BATCH_CASE
  return -1;
}

}  // namespace pawsim
