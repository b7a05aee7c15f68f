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

}  // namespace pawsim
