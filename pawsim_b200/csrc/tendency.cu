// tendency.cu -- chooses the tile height of the fused tendency kernel (tendency_tile.cu).
//
// Both heights compute the same values; 32 x 16 tiles (512 threads) spend fewer halo
// evaluations per owned cell than 32 x 8 tiles (256 threads) but hold twice the shared
// memory. The taller tile is used while two of its CTAs still fit in one SM's shared memory.
#include <cuda_runtime.h>

#include "tendency.cuh"

namespace pawsim {

size_t tendency_smem_ty8(const TendParams& p, int ts);
size_t tendency_smem_ty16(const TendParams& p, int ts);
// one translation unit per tile height and momentum scheme (compiled in parallel)
#define PAWSIM_DECL_TEND(TY)                                                   \
  int launch_tendency_ty##TY##_m0(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m1(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m2(const TendParams& p, int ms, int ts, cudaStream_t s); \
  int launch_tendency_ty##TY##_m3(const TendParams& p, int ms, int ts, cudaStream_t s);
PAWSIM_DECL_TEND(8)
PAWSIM_DECL_TEND(16)
#undef PAWSIM_DECL_TEND
#define PAWSIM_DECL_BATCH(TY, M)                                                                         \
  int batch_launch_tendency_ty##TY##_m##M(const TendParams& p0, const TendParams* ps, const int* work, \
                                           int nwork, int members, int* done, int ms, int ts, cudaStream_t s);
PAWSIM_DECL_BATCH(8, 0) PAWSIM_DECL_BATCH(8, 1) PAWSIM_DECL_BATCH(8, 2) PAWSIM_DECL_BATCH(8, 3)
PAWSIM_DECL_BATCH(16, 0) PAWSIM_DECL_BATCH(16, 1) PAWSIM_DECL_BATCH(16, 2) PAWSIM_DECL_BATCH(16, 3)
#undef PAWSIM_DECL_BATCH
int launch_tendency_budget_tile(const TendParams& p, int ms, int ts, cudaStream_t s);

static int launch_tendency_ty8(const TendParams& p, int ms, int ts, cudaStream_t s) {
  switch (ms) {
    case 0: return launch_tendency_ty8_m0(p, ms, ts, s);
    case 1: return launch_tendency_ty8_m1(p, ms, ts, s);
    case 2: return launch_tendency_ty8_m2(p, ms, ts, s);
    case 3: return launch_tendency_ty8_m3(p, ms, ts, s);
  }
  return -1;
}

static int launch_tendency_ty16(const TendParams& p, int ms, int ts, cudaStream_t s) {
  switch (ms) {
    case 0: return launch_tendency_ty16_m0(p, ms, ts, s);
    case 1: return launch_tendency_ty16_m1(p, ms, ts, s);
    case 2: return launch_tendency_ty16_m2(p, ms, ts, s);
    case 3: return launch_tendency_ty16_m3(p, ms, ts, s);
  }
  return -1;
}

int launch_tendency(const TendParams& p, int ms, int ts, cudaStream_t s) {
  // two CTAs per SM: 228 KB of shared memory, 1 KB reserved per CTA
  constexpr size_t kTwoPerSM = 113 * 1024;
  if (tendency_smem_ty16(p, ts) <= kTwoPerSM) return launch_tendency_ty16(p, ms, ts, s);
  return launch_tendency_ty8(p, ms, ts, s);
}

int launch_tendency_budget(const TendParams& p, int ms, int ts, cudaStream_t s) {
  return launch_tendency_budget_tile(p, ms, ts, s);
}

int tendency_tile_height(const TendParams& p, int ts) {
  constexpr size_t kTwoPerSM = 113 * 1024;
  return tendency_smem_ty16(p, ts) <= kTwoPerSM ? 16 : 8;
}

int launch_tendency_batch(const TendParams& p0, const TendParams* ps, const int* work, int nwork, int members,
                          int* done, int ms, int ts, cudaStream_t s) {
  const bool tall = tendency_tile_height(p0, ts) == 16;
#define PAWSIM_BATCH_CASE(M)                                                                         \
  case M:                                                                                            \
    return tall ? batch_launch_tendency_ty16_m##M(p0, ps, work, nwork, members, done, ms, ts, s)   \
                : batch_launch_tendency_ty8_m##M(p0, ps, work, nwork, members, done, ms, ts, s);
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
