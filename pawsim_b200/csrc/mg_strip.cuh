// mg_strip.cuh -- streaming variants of the fused multigrid level kernels (included by
// mg.cu after the tile kernels; same arithmetic in the same order, so the results are bit
// for bit those of the tile kernels).
//
// One warp owns a strip of SP_OWN columns and a segment of S rows. Its 32 lanes hold the
// strip's 64 columns (SP_HALO halo columns on each side) as pairs of adjacent cells
// (c0 at an even column, c1 = c0 + 1), so each row of each array arrives with one aligned
// vector load per lane. Rows stream through a ring of six register slots: at step t the
// warp loads row t+1 (prefetch), the red half sweep runs on row t-1, the black half sweep
// on row t-2, and the residual with the 2x2 restriction (down) or the stopping measure (up)
// on row t-3. West and east neighbours come from the adjacent lanes by shuffles. There is
// no shared memory and no barrier: a warp's traffic is its rows, read once from HBM; the
// halo rows and columns it shares with neighbouring warps come from L2.
//
// Colours: a cell (i, j) is red when i + j is even. Strips start at even columns and
// segments at even rows (S is a multiple of 6), so the colour of c0 and c1 and the parity
// of every ring slot are known at compile time inside the six-step unrolled body.
#pragma once

constexpr int SP_OWN = 56;     // owned columns of a strip
constexpr int SP_HALO = 4;     // halo columns on each side (even: strips start on even columns)
constexpr int SP_WARPS = 2;    // warps (strips) per CTA
constexpr int SP_CTAS_DOWN = 7;   // resident CTAs per SM (shared memory: 30 KB each in FP64)
constexpr int SP_CTAS_UP = 6;     // (36 KB each in FP64)
constexpr int SP_RING = 6;     // row slots, in registers and in each warp's staging area
constexpr int SP_AHEAD = 3;    // rows in flight per warp (cp.async into the staging area)

// staging slot of one row: e, rhs, 1/Osum, Ow, Os (64 cells each), and in the up kernel
// the coarse correction on the coarse rows south and north of the row (32 coarse cells each)
constexpr int SL_E = 0, SL_RHS = 64, SL_RO = 128, SL_OW = 192, SL_OS = 256, SL_CM = 320, SL_CP = 352;
constexpr int SL_DOWN = 320, SL_UP = 384;   // slot sizes in elements
constexpr int SL_SCRATCH = 32;               // one word per lane after a warp's slots

template <typename T>
constexpr size_t strip_smem_bytes(bool up) {
  return (size_t)SP_WARPS * (SP_RING * (up ? SL_UP : SL_DOWN) + SL_SCRATCH) * sizeof(T);
}

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <typename T>
__device__ __forceinline__ void lds_pair(const T* p, T& a, T& b) {
  const typename Vec2<T>::type v = *reinterpret_cast<const typename Vec2<T>::type*>(p);
  a = v.x;
  b = v.y;
}
template <typename T>
__device__ __forceinline__ void st_pair(T* p, T a, T b) {
  typename Vec2<T>::type v;
  v.x = a;
  v.y = b;
  *reinterpret_cast<typename Vec2<T>::type*>(p) = v;
}
// asynchronous copy of a lane's cell pair (16 bytes FP64, 8 bytes FP32) or of one value
template <typename T>
__device__ __forceinline__ void cp_async_pair(T* dst, const T* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
template <typename T>
__device__ __forceinline__ T from_west(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T from_east(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// The FP64 down kernel forms 1/Osum from the face coefficients it already holds instead of
// reading it (8 bytes less per cell): Osum summed in the order of the operator set-up and the
// IEEE division give the stored value bit for bit (0 where Osum is 0, as stored). The up
// kernel, which issues more instructions per cell, and FP32 (whose stored value is the FP64
// reciprocal rounded to FP32) read the stored value. RCP selects the first way.
template <typename T, bool UP>
constexpr bool kStripRcp = sizeof(T) == 8 && !UP;
template <typename T>
__device__ __forceinline__ T strip_rcp(T osum) {
  const T q = T(1) / osum;
  return isfinite(q) ? q : T(0);
}

// one row of a lane in registers: e, rhs, 1/Osum (FP32 only), Ow, Os at c0 and c1
template <typename T>
struct SRow {
  T e0, e1, r0, r1, q0, q1, w0, w1, s0, s1;
};

// store one register written by each shared-memory load of a row to the lane's scratch
// word: the stores cannot issue before those loads have returned, so the row's staging slot
// may be refilled after them
template <typename T, bool RCP>
__device__ __forceinline__ void strip_consume(const SRow<T>& R, T* scratch) {
  volatile T* v = scratch;
  *v = R.e0;
  *v = R.r0;
  if (!RCP) *v = R.q0;
  *v = R.w0;
  *v = R.s0;
}

// start the copies of row y (wrapped) into a staging slot; with `coarse` also the coarse
// correction at the lane's coarse column ic on the rows south and north of y
template <typename T, bool RCP>
__device__ __forceinline__ void strip_issue(const LV<T>& f, const T* e, int gx, int y, bool zero_e, T* slot,
                                            int lane, const LV<T>* c, int ic) {
  const size_t o = (size_t)wrapi(y, f.Ny) * f.pitch + gx;
  T* d = slot + 2 * lane;
  if (!zero_e) cp_async_pair(d + SL_E, e + o);
  cp_async_pair(d + SL_RHS, f.rhs + o);
  if (!RCP) cp_async_pair(d + SL_RO, f.rOsum + o);
  cp_async_pair(d + SL_OW, f.Ow + o);
  cp_async_pair(d + SL_OS, f.Os + o);
  if (c) {
    // coarse rows south and north of the (wrapped) fine row, as prolong_at indexes them
    const int hy = f.Ny / 2;
    int jp = (wrapi(y, f.Ny) + 1) >> 1;
    if (jp >= hy) jp -= hy;
    const int jm = jp == 0 ? hy - 1 : jp - 1;
    cp_async(slot + SL_CM + lane, c->e + (size_t)jm * c->pitch + ic);
    cp_async(slot + SL_CP + lane, c->e + (size_t)jp * c->pitch + ic);
  }
}

template <typename T, bool RCP>
__device__ __forceinline__ void strip_read(const T* slot, int lane, bool zero_e, SRow<T>& R) {
  const T* d = slot + 2 * lane;
  if (zero_e) {
    R.e0 = T(0);
    R.e1 = T(0);
  } else {
    lds_pair(d + SL_E, R.e0, R.e1);
  }
  lds_pair(d + SL_RHS, R.r0, R.r1);
  if (!RCP) lds_pair(d + SL_RO, R.q0, R.q1);
  lds_pair(d + SL_OW, R.w0, R.w1);
  lds_pair(d + SL_OS, R.s0, R.s1);
}

// weighted Gauss-Seidel update of c0 (west neighbour from lane-1) and of c1 (east
// neighbour and east face from lane+1) on row R between rows Sr (south) and Nr (north);
// the order of half_sweep in the tile kernels
template <typename T, bool RCP>
__device__ __forceinline__ T strip_q0(const SRow<T>& R, const SRow<T>& Nr) {
  if constexpr (RCP) return strip_rcp(R.w0 + R.w1 + R.s0 + Nr.s0);
  else return R.q0;
}
template <typename T, bool RCP>
__device__ __forceinline__ T strip_q1(const SRow<T>& R, const SRow<T>& Nr, T w2) {
  if constexpr (RCP) return strip_rcp(R.w1 + w2 + R.s1 + Nr.s1);
  else return R.q1;
}
// (with RCP the reciprocal formed here is left in R.q0 / R.q1)
template <typename T, bool RCP>
__device__ __forceinline__ T strip_upd_c0(SRow<T>& R, const SRow<T>& Sr, const SRow<T>& Nr, T omega) {
  const T wn = from_west(R.e1);
  const T s = Nr.s0 * Nr.e0 + R.s0 * Sr.e0 + R.w1 * R.e1 + R.w0 * wn;
  R.q0 = strip_q0<T, RCP>(R, Nr);
  return omega * R.q0 * (s - R.r0) + (T(1) - omega) * R.e0;
}
template <typename T, bool RCP>
__device__ __forceinline__ T strip_upd_c1(SRow<T>& R, const SRow<T>& Sr, const SRow<T>& Nr, T omega) {
  const T en = from_east(R.e0);
  const T w2 = from_east(R.w0);
  const T s = Nr.s1 * Nr.e1 + R.s1 * Sr.e1 + w2 * en + R.w1 * R.e0;
  R.q1 = strip_q1<T, RCP>(R, Nr, w2);
  return omega * R.q1 * (s - R.r1) + (T(1) - omega) * R.e1;
}

// neighbour sums of both cells (for the residual and the stopping measure)
template <typename T>
__device__ __forceinline__ void strip_nsum(const SRow<T>& R, const SRow<T>& Sr, const SRow<T>& Nr, T& s0, T& s1,
                                           T& w2) {
  const T wn = from_west(R.e1), en = from_east(R.e0);
  w2 = from_east(R.w0);
  s0 = Nr.s0 * Nr.e0 + R.s0 * Sr.e0 + R.w1 * R.e1 + R.w0 * wn;
  s1 = Nr.s1 * Nr.e1 + R.s1 * Sr.e1 + w2 * en + R.w1 * R.e0;
}

// rows per segment: the smallest multiple of 6 (at least 24) that keeps every strip's
// segments within one wave of resident warps
inline int strip_rows(int Nx, int Ny, int sms) {
  const int nstrips = (Nx + SP_OWN - 1) / SP_OWN;
  const int slots = sms * SP_CTAS_UP * SP_WARPS;
  int segs = slots / nstrips;
  if (segs < 1) segs = 1;
  int S = (Ny + segs - 1) / segs;
  S = (S + 5) / 6 * 6;
  return S < 24 ? 24 : S;
}

// The row loop of both kernels. Step t (rows Y0-3 .. Y0+S+2) reads row t from its staging
// slot into register slot t mod 6, then starts the copy of row t+3 into the staging slot
// of row t-3, whose registers the red half sweep of step t-2 has read. The first row is
// never swept: stores of its registers to a scratch word precede the reuse of its slot.
// cp.async groups are committed once per step, so waiting until at most SP_AHEAD-1 groups
// are pending means row t has arrived; each lane reads back only what it copied itself.

// pre-smoothing (one red-black sweep) of f.e (or of zero) into `out`, residual and 2x2
// restriction into the coarse rhs: down_tile with NU = 1, streamed
template <typename T>
__device__ __forceinline__ void down_strip_body(const LV<T>& f, const LV<T>& c, T omega, int zero_e,
                                                T* __restrict__ out, int S, int nstrips, int nsegs, int bx) {
  extern __shared__ __align__(16) unsigned char sp_raw[];
  const int lane = threadIdx.x & 31;
  const int w = bx * SP_WARPS + (threadIdx.x >> 5);
  if (w >= nstrips * nsegs) return;   // whole warps only: the kernel has no barrier
  T* stage = reinterpret_cast<T*>(sp_raw) + (threadIdx.x >> 5) * (SP_RING * SL_DOWN + SL_SCRATCH);
  T* scratch = stage + SP_RING * SL_DOWN + lane;
  const int X0 = (w % nstrips) * SP_OWN - SP_HALO, Y0 = (w / nstrips) * S;
  const int cx = X0 + 2 * lane;
  const int gx = wrapi(cx, f.Nx);
  const bool ownx = lane >= SP_HALO / 2 && lane < 32 - SP_HALO / 2 && cx < f.Nx;
  constexpr bool RCP = kStripRcp<T, false>;
  const bool ze = zero_e != 0;
  const int first = Y0 - 3, last = Y0 + S + 2;
  for (int k = 0; k < SP_AHEAD; ++k) {
    strip_issue<T, RCP>(f, f.e, gx, first + k, ze, stage + k * SL_DOWN, lane, nullptr, 0);
    cp_async_commit();
  }
  SRow<T> R[SP_RING];
  T p0 = T(0), p1 = T(0);   // residuals of the even row of a restriction pair
  const int nb = (S + 6) / 6;
  for (int b = 0; b < nb; ++b) {
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      const int t = first + 6 * b + u;   // parity of t is that of u + 1
      cp_async_wait<SP_AHEAD - 1>();
      strip_read<T, RCP>(stage + u * SL_DOWN, lane, ze, R[u]);
      if (b == 0 && u == SP_AHEAD) strip_consume<T, RCP>(R[0], scratch);
      if (t + SP_AHEAD <= last)
        strip_issue<T, RCP>(f, f.e, gx, t + SP_AHEAD, ze, stage + ((u + SP_AHEAD) % 6) * SL_DOWN, lane, nullptr, 0);
      cp_async_commit();
      // red half sweep on row t-1 (from Y0-2): c0 is red on even rows
      if (b > 0 || u >= 2) {
        SRow<T>& Rr = R[(u + 5) % 6];
        if ((u & 1) == 0) Rr.e0 = strip_upd_c0<T, RCP>(Rr, R[(u + 4) % 6], R[u], omega);
        else Rr.e1 = strip_upd_c1<T, RCP>(Rr, R[(u + 4) % 6], R[u], omega);
      }
      // black half sweep on row t-2 (from Y0-1): c0 is black on odd rows
      if (b > 0 || u >= 4) {
        SRow<T>& Rb = R[(u + 4) % 6];
        if ((u & 1) == 0) Rb.e0 = strip_upd_c0<T, RCP>(Rb, R[(u + 3) % 6], R[(u + 5) % 6], omega);
        else Rb.e1 = strip_upd_c1<T, RCP>(Rb, R[(u + 3) % 6], R[(u + 5) % 6], omega);
      }
      // residual and restriction on row t-3 (from Y0), as down_tile
      if (b > 0) {
        const SRow<T>& Rq = R[(u + 3) % 6];
        const SRow<T>& Nq = R[(u + 4) % 6];
        T s0, s1, w2;
        strip_nsum(Rq, R[(u + 2) % 6], Nq, s0, s1, w2);
        const T o0 = Rq.w0 + Rq.w1 + Rq.s0 + Nq.s0;
        const T o1 = Rq.w1 + w2 + Rq.s1 + Nq.s1;
        const T x0 = s0 - o0 * Rq.e0 - Rq.r0;
        const T x1 = s1 - o1 * Rq.e1 - Rq.r1;
        const int r = t - 3;
        const bool own = ownx && r < f.Ny;
        if (own) st_pair(out + (size_t)r * f.pitch + gx, Rq.e0, Rq.e1);
        if (u & 1) {
          // odd row: restriction, order (2i,2j) + (2i+1,2j) + (2i,2j+1) + (2i+1,2j+1)
          if (own) c.rhs[(size_t)(r >> 1) * c.pitch + (gx >> 1)] = T(0.25) * (p0 + p1 + x0 + x1);
        } else {
          p0 = x0;
          p1 = x1;
        }
      }
    }
  }
  cp_async_wait<0>();
}

// prolongation of the coarse correction c.e, correction of f.e (the pre-smoothed field),
// post-smoothing into `out` and, with MEASURE, the stopping measure max |e - Jacobi(e)|
// over the owned cells into *bits: up_tile with NU = 1, streamed
template <typename T, bool MEASURE>
__device__ __forceinline__ void up_strip_body(const LV<T>& f, const LV<T>& c, T omega, int wew, int wns,
                                              unsigned long long* bits, T* __restrict__ out, int S, int nstrips,
                                              int nsegs, int bx) {
  extern __shared__ __align__(16) unsigned char sp_raw[];
  const int lane = threadIdx.x & 31;
  const int w = bx * SP_WARPS + (threadIdx.x >> 5);
  const bool active = w < nstrips * nsegs;   // inactive warps still reach the block reduction
  constexpr bool RCP = kStripRcp<T, true>;
  double m = 0;
  if (active) {
    T* stage = reinterpret_cast<T*>(sp_raw) + (threadIdx.x >> 5) * (SP_RING * SL_UP + SL_SCRATCH);
    T* scratch = stage + SP_RING * SL_UP + lane;
    const int X0 = (w % nstrips) * SP_OWN - SP_HALO, Y0 = (w / nstrips) * S;
    const int cx = X0 + 2 * lane;
    const int gx = wrapi(cx, f.Nx);
    const bool ownx = lane >= SP_HALO / 2 && lane < 32 - SP_HALO / 2 && cx < f.Nx;
    // the coarse column of the lane's pair (c0 = 2 ic); its west and east neighbours are the
    // adjacent lanes' (wrapped like the fine columns), and the coarse values of the rows
    // south and north of each fine row arrive with that row
    const int ic = gx >> 1;
    const int first = Y0 - 3, last = Y0 + S + 2;
    for (int k = 0; k < SP_AHEAD; ++k) {
      strip_issue<T, RCP>(f, f.e, gx, first + k, false, stage + k * SL_UP, lane, &c, ic);
      cp_async_commit();
    }
    // warps whose cells (columns X0 .. X0+63, rows Y0-3 .. Y0+S+2) touch no wall cell take
    // the plain bilinear weights (compile-time constants per row parity); the others
    // evaluate the wall and corner overrides
    const bool plain_x = !wew || (X0 >= 1 && X0 + 64 <= f.Nx - 1);
    const bool plain_y = !wns || (Y0 - 3 >= 1 && Y0 + S + 3 <= f.Ny - 1);
    const bool plain = plain_x && plain_y;
    // e -= bilinear coarse correction (the weights and the order of prolong_at)
    auto correct = [&](int t, const T* slot, SRow<T>& R, bool odd_row) {
      const T cm = slot[SL_CM + lane], cp = slot[SL_CP + lane];
      const T wcm = from_west(cm), ecm = from_east(cm), wcp = from_west(cp), ecp = from_east(cp);
      if (plain) {
        const T aj = odd_row ? T(0.75) : T(0.25), bj = odd_row ? T(0.25) : T(0.75);
        // c0: even column (ai = 1/4), coarse west = ic - 1, east = ic
        R.e0 -= (T(0.25) * aj) * wcm + (T(0.75) * aj) * cm + (T(0.25) * bj) * wcp + (T(0.75) * bj) * cp;
        // c1: odd column (ai = 3/4), coarse west = ic, east = ic + 1
        R.e1 -= (T(0.75) * aj) * cm + (T(0.25) * aj) * ecm + (T(0.75) * bj) * cp + (T(0.25) * bj) * ecp;
      } else {
        const int gy = wrapi(t, f.Ny);
        T wmm, wpm, wmp, wpp;
        prolong_weights<T>(gx, gy, f.Nx, f.Ny, wew, wns, wmm, wpm, wmp, wpp);
        R.e0 -= wmm * wcm + wpm * cm + wmp * wcp + wpp * cp;
        prolong_weights<T>(gx + 1, gy, f.Nx, f.Ny, wew, wns, wmm, wpm, wmp, wpp);
        R.e1 -= wmm * cm + wpm * ecm + wmp * cp + wpp * ecp;
      }
    };
    SRow<T> R[SP_RING];
    const int nb = (S + 6) / 6;
    for (int b = 0; b < nb; ++b) {
#pragma unroll
      for (int u = 0; u < 6; ++u) {
        const int t = first + 6 * b + u;   // parity of t is that of u + 1
        cp_async_wait<SP_AHEAD - 1>();
        strip_read<T, RCP>(stage + u * SL_UP, lane, false, R[u]);
        correct(t, stage + u * SL_UP, R[u], (u & 1) == 0);
        if (b == 0 && u == SP_AHEAD) strip_consume<T, RCP>(R[0], scratch);
        if (t + SP_AHEAD <= last)
          strip_issue<T, RCP>(f, f.e, gx, t + SP_AHEAD, false, stage + ((u + SP_AHEAD) % 6) * SL_UP, lane, &c, ic);
        cp_async_commit();
        if (b > 0 || u >= 2) {
          SRow<T>& Rr = R[(u + 5) % 6];
          if ((u & 1) == 0) Rr.e0 = strip_upd_c0<T, RCP>(Rr, R[(u + 4) % 6], R[u], omega);
          else Rr.e1 = strip_upd_c1<T, RCP>(Rr, R[(u + 4) % 6], R[u], omega);
        }
        if (b > 0 || u >= 4) {
          SRow<T>& Rb = R[(u + 4) % 6];
          if ((u & 1) == 0) Rb.e0 = strip_upd_c0<T, RCP>(Rb, R[(u + 3) % 6], R[(u + 5) % 6], omega);
          else Rb.e1 = strip_upd_c1<T, RCP>(Rb, R[(u + 3) % 6], R[(u + 5) % 6], omega);
          const int r = t - 2;
          if (ownx && r >= Y0 && r < Y0 + S && r < f.Ny) st_pair(out + (size_t)r * f.pitch + gx, Rb.e0, Rb.e1);
        }
        if constexpr (MEASURE) {
          if (b > 0) {
            const SRow<T>& Rq = R[(u + 3) % 6];
            T s0, s1, w2;
            strip_nsum(Rq, R[(u + 2) % 6], R[(u + 4) % 6], s0, s1, w2);
            const int r = t - 3;
            if (ownx && r < f.Ny) {
              // both cells of the row were swept (red two steps ago, black one step ago),
              // which left 1/Osum in q0 and q1
              const T x0 = Rq.e0 - Rq.q0 * (s0 - Rq.r0);
              const T x1 = Rq.e1 - Rq.q1 * (s1 - Rq.r1);
              m = fmax(m, fabs((double)x0));
              m = fmax(m, fabs((double)x1));
            }
          }
        }
      }
    }
    cp_async_wait<0>();
  }
  if constexpr (MEASURE) block_max_to(m, bits);
}

template <typename T>
__global__ void __launch_bounds__(SP_WARPS * 32, SP_CTAS_DOWN)
down_strip(LV<T> f, LV<T> c, T omega, int zero_e, T* __restrict__ out, int S, int nstrips, int nsegs) {
  down_strip_body<T>(f, c, omega, zero_e, out, S, nstrips, nsegs, blockIdx.x);
}

template <typename T, bool MEASURE>
__global__ void __launch_bounds__(SP_WARPS * 32, SP_CTAS_UP)
up_strip(LV<T> f, LV<T> c, T omega, int wew, int wns, unsigned long long* bits, T* __restrict__ out, int S,
         int nstrips, int nsegs) {
  up_strip_body<T, MEASURE>(f, c, omega, wew, wns, bits, out, S, nstrips, nsegs, blockIdx.x);
}
