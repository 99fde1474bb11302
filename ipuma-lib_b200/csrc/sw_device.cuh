// sw_device.cuh -- device-side building blocks of the affine-gap
// Smith-Waterman (Gotoh) kernels for sm_100a.
//
// The recurrence is the one of the ipuma codelet SWAffine::compute
// (src/codelets/codelet_batch_affine.cpp:65-85):
//
//   E      = max(Hleft + gI + gE, E + gE)         E starts at gI on every row
//   F[j]   = max(Hup[j] + gI + gE, F[j] + gE)     F starts at 0
//   H      = max(Hdiag + sim[a[j]][b[i]], E, F[j], 0)
//   best   : first strict maximum in (i over B, j over A) row-major order
//
// Kernels keep H in the reference's frame and E, F shifted by -(gI + gE)
// (Ê = E - gI - gE, F̂ = F - gI - gE).  Writing Y = max(Hdiag + sim,
// F, 0), the left neighbour's H + gI + gE = max(Y, E) + gI + gE, and
// E + gI + gE <= E + gE whenever gI <= 0, so the E recurrence needs Y only:
//   F̂  = max(F̂ + gE, Hup)                      F̂ = -gI - gE at the start
//   Y  = max(Hdiag + sim, F̂ + gI + gE, 0)
//   Ê  = max(Ê + gE', Yleft)                    gE' = max(gE, gI + gE)
//   H  = max(Y, Ê + gI + gE)                     Ê = -gE at a row start
// (with gE' the E chain is exact for gI > 0 too).  Every line is one fused
// DPX add-max (__viaddmax / __viaddmax_relu) except the add F̂ + gI + gE,
// and only Ê depends on the previous column of the same row, so the
// row-serial chain is one instruction per cell.
//
// Layout of the work: one warp aligns one pair (s32 lanes) or two pairs
// (s16x2 lanes, pair P in the low and pair Q in the high halfword).  Lane l
// owns K consecutive A columns of a 32*K wide strip; B rows stream through
// the warp as an anti-diagonal wavefront (lane l works on row t - l at step
// t) and the left neighbour's last-column (HG, E) arrives through
// __shfl_up_sync.  A longer than one strip is processed strip by strip; the
// last column of a strip is handed to the next one through per-warp global
// scratch (a strip team, StripTeam, spreads one couple's strips over the
// warps of a block instead).  Substitution scores come from a per-strip
// query profile in shared memory (int8, one row per B letter plus a
// padding row).
//
// Invalid cells (columns past |A|, rows past |B| of the shorter pair of an
// s16x2 couple) get the profile value SUB_PAD.  With gI + gE < 0 and
// gE <= 0 every such cell stays strictly below the best valid cell seen so
// far, so it can never win or tie the maximum; configurations outside that
// range run on the exact per-thread kernel instead.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <type_traits>

// Steps per unrolled check-free block (0: by K, as measured; >= LANES:
// the whole block).
#ifndef IPUMA_STEP_UNROLL
#define IPUMA_STEP_UNROLL 0
#endif

namespace ipuma_dev {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SUB_PAD = -64;  // profile value of padding columns and rows

// Scoring constants shared by all kernels of one launch.
struct SwConst {
  int gI;       // gap init (ipu::SWConfig::gapInit)
  int gE;       // gap extend (ipu::SWConfig::gapExtend)
  int gIgE;     // gI + gE
  int M;        // alphabet size (rows/cols of the substitution matrix)
  int forwardOnly;
  int s16Limit; // a pair whose score exceeds this is rerun in s32 (signed halves)
  int u16Limit; // the same for the biased halves of the wavefront classes (LaneB16x2)
  int maxSub;   // largest substitution score (strip bound of the hybrid pass)
  int bits;     // bits per residue of the code array (8, or packed 2/4/5: code_at)
  int P;        // letters of the query profile (M, or 4 for 2-bit A/C/G/T codes)
  int pshift;   // profile row of a code: code - pshift (1 for 2-bit codes, else 0)
};

// Control of a hybrid pass (sw_pass with HYB): an s16x2 pass that stops
// before the first strip whose values could pass the 16-bit lanes' limit, and the s32
// pass that continues one of its pairs from there.  A strip's H values are
// at most max(0, H of the boundary column entering it) + maxSub * strip
// width: a path enters from that column or starts inside the strip, and
// gains at most maxSub per diagonal step, of which a strip holds at most
// its width.
struct PassCtl {
  int strip0 = 0;          // first strip of this pass
  int bndHalf = -1;        // strip0 > 0: half (0/1) of the packed s16x2 boundary to read
  int scrBase = 0;         // scratch buffer (0..2) holding that boundary
  int stoppedAt = -1;      // out (s16x2 pass): strip it stopped before, -1: none
};

// Early stop of a reverse pass (sw_pass with EARLY): the reverse maximum of
// a pair equals its forward score, so a strip may end once every pair's
// group has reached its target and all lanes have passed that row, and a
// later strip (larger columns) can only win with a smaller row, so it runs
// only the rows above the best row found so far.  Exact under the
// first-strict-maximum tie-break.
struct PassStop {
  bool on = false;
  int target[2] = {0, 0};  // per pair; 0 for a pair without a reverse pass
};

// Strip team: the `warps` warps of a block run one pass together, warp w
// taking strips w, w + warps, w + 2 * warps, ...  Strip s writes its
// boundary column to scratch buffer s % warps and, after every block of
// steps, publishes (s << 16) | rows-written in prog[warp]; strip s + 1
// waits for the rows it is about to read.  The values only grow within a
// pass (a warp moves to higher strips), so a consumer never mistakes the
// producer's next strip for the one it reads.  Strip s + warps overwrites
// buffer s % warps only after strip s + 1 has read those rows: it depends,
// through strips s + warps - 1, ..., s + 2, on rows that strip s + 1
// produced after reading them.  Every wait is bounded: past kTeamWaitNs
// the warp sets `*err` (if 0) to errCode and `*abort`, and every warp of
// the team leaves the pass at its next wait or block.
constexpr unsigned long long kTeamWaitNs = 2000000000ull;
struct StripTeam {
  int* prog = nullptr;   // shared memory, one word per warp
  int* abort = nullptr;  // shared memory: nonzero once any warp gave up
  int* err = nullptr;    // status word of the launch
  int errCode = 0;
  int warp = 0;
  int warps = 1;
};

// Device clock in nanoseconds (bounded waits; the trace of class launches).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// -------------------------------------------------------------------------
// Lane types
// -------------------------------------------------------------------------

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// One pair per warp, exact int32 arithmetic.
struct LaneS32 {
  using V = int;
  static constexpr int NP = 1;
  __device__ __forceinline__ static V splat(int x) { return x; }
  __device__ __forceinline__ static V add(V a, V b) { return a + b; }
  // max(a + b, c)
  __device__ __forceinline__ static V addmax(V a, V b, V c) { return __viaddmax_s32(a, b, c); }
  // max(a, b, c, 0)
  __device__ __forceinline__ static V max3relu(V a, V b, V c) { return __vimax3_s32_relu(a, b, c); }
  // max(a + b, c, 0)
  __device__ __forceinline__ static V addmax_relu(V a, V b, V c) { return __viaddmax_s32_relu(a, b, c); }
  __device__ __forceinline__ static V max2(V a, V b) { return max(a, b); }
  __device__ __forceinline__ static V max3(V a, V b, V c) { return __vimax3_s32(a, b, c); }
  // Substitution value of byte `c` (0..3) of the profile word, sign-extended.
  template <int C>
  __device__ __forceinline__ static V sub(uint32_t wp, uint32_t /*wq*/) {
    return (int)prmt(wp, 0u, (uint32_t)(C | ((C | 8) << 4) | ((C | 8) << 8) | ((C | 8) << 12)));
  }
  __device__ __forceinline__ static int half(V v, int /*h*/) { return v; }
  __device__ __forceinline__ static V pack2(int lo, int /*hi*/) { return lo; }
  __device__ __forceinline__ static V shfl_up(V v) { return __shfl_up_sync(FULL, v, 1); }
};

// Two pairs per warp in s16x2 halves (pair P low, pair Q high).
struct LaneS16x2 {
  using V = uint32_t;
  static constexpr int NP = 2;
  __device__ __forceinline__ static V splat(int x) {
    return (uint32_t)(x & 0xffff) | ((uint32_t)(x & 0xffff) << 16);
  }
  __device__ __forceinline__ static V add(V a, V b) {
    V d;
    asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
  }
  __device__ __forceinline__ static V addmax(V a, V b, V c) { return __viaddmax_s16x2(a, b, c); }
  __device__ __forceinline__ static V max3relu(V a, V b, V c) { return __vimax3_s16x2_relu(a, b, c); }
  __device__ __forceinline__ static V addmax_relu(V a, V b, V c) { return __viaddmax_s16x2_relu(a, b, c); }
  __device__ __forceinline__ static V max2(V a, V b) {
    V d;
    asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
  }
  __device__ __forceinline__ static V max3(V a, V b, V c) { return __vimax3_s16x2(a, b, c); }
  template <int C>
  __device__ __forceinline__ static V sub(uint32_t wp, uint32_t wq) {
    return prmt(wp, wq, (uint32_t)(C | ((C | 8) << 4) | ((4 + C) << 8) | (((4 + C) | 8) << 12)));
  }
  __device__ __forceinline__ static int half(V v, int h) {
    return h == 0 ? (int)(int16_t)(v & 0xffff) : (int)(int16_t)(v >> 16);
  }
  __device__ __forceinline__ static V pack2(int lo, int hi) {
    return (uint32_t)(lo & 0xffff) | ((uint32_t)(hi & 0xffff) << 16);
  }
  __device__ __forceinline__ static V shfl_up(V v) { return __shfl_up_sync(FULL, v, 1); }
};

// Two pairs per warp in biased 16-bit halves (pair P low, pair Q high): a
// score v is held as the signed halfword v + BIAS - 32768, so the signed
// range [-32768, 32767] covers scores [-BIAS, 65535 - BIAS] -- twice the
// plain signed halfword's range -- with the same instructions per cell:
// signed max orders the shifted values like the scores, and the sums are
// the same modular adds.  Every stored value (H, Y, and E, F shifted by
// -(gI + gE)) is >= 0, so it sits at least BIAS above the bottom of the
// range; a sum with a profile byte (>= -128), gI + gE or gE (> -1000 on
// this path) stays in range and no halfword wraps.  The floor 0 of the
// recurrence is folded into the F term of Y (Cell::fterm), so Y needs no
// relu.  The running best compares halves as signed integers
// (update_best), since two halves may differ by more than 32767.
struct LaneB16x2 {
  using V = uint32_t;
  static constexpr int NP = 2;
  static constexpr int BIAS = 1024;
  static constexpr int OFFSET = BIAS - 32768;  // score -> stored halfword
  __device__ __forceinline__ static V splat(int x) {  // a score
    const uint32_t v = (uint32_t)(x + OFFSET) & 0xffffu;
    return v | (v << 16);
  }
  __device__ __forceinline__ static V delta(int x) {  // an addend
    const uint32_t v = (uint32_t)x & 0xffffu;
    return v | (v << 16);
  }
  __device__ __forceinline__ static V add(V a, V b) {
    V d;
    asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
  }
  __device__ __forceinline__ static V addmax(V a, V b, V c) { return __viaddmax_s16x2(a, b, c); }
  __device__ __forceinline__ static V max2(V a, V b) {
    V d;
    asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
  }
  template <int C>
  __device__ __forceinline__ static V sub(uint32_t wp, uint32_t wq) {
    return prmt(wp, wq, (uint32_t)(C | ((C | 8) << 4) | ((4 + C) << 8) | (((4 + C) | 8) << 12)));
  }
  __device__ __forceinline__ static int half(V v, int h) {
    return (h == 0 ? (int)(int16_t)(v & 0xffffu) : (int)(int16_t)(v >> 16)) - OFFSET;
  }
  __device__ __forceinline__ static V pack2(int lo, int hi) {  // two scores
    return ((uint32_t)(lo + OFFSET) & 0xffffu) | (((uint32_t)(hi + OFFSET) & 0xffffu) << 16);
  }
  __device__ __forceinline__ static V shfl_up(V v) { return __shfl_up_sync(FULL, v, 1); }
};

// The 16-bit lanes of the engine's wavefront classes, and those of the
// hybrid class, which takes the pairs whose score can pass the signed
// halfword's range (its strips run in biased halves while their values
// provably fit, then in s32).  The biased form costs one more add-max per
// cell (the recurrence's floor), so the ordinary classes keep signed halves.
using Lane16 = LaneS16x2;
using LaneHi = LaneB16x2;

// The pieces of one cell that differ between lane types.
//   fterm(F̂, gI+gE)    the F term of Y: F̂ + gI + gE (with the floor 0 of
//                      the recurrence for biased lanes)
//   ymax(Hdiag, s, f)  Y = max(Hdiag + s, f, 0)
//   delta(x)           an addend (gap penalties) in the lane's format
//   limit(sc)          largest score a lane may hold before the next cells
//                      could leave its range (checked every 32 steps)
template <class T>
struct Cell {
  __device__ __forceinline__ static typename T::V fterm(typename T::V f, typename T::V gIgE) {
    return T::add(f, gIgE);
  }
  __device__ __forceinline__ static typename T::V ymax(typename T::V d, typename T::V s, typename T::V f) {
    return T::addmax_relu(d, s, f);
  }
  __device__ __forceinline__ static typename T::V delta(int x) { return T::splat(x); }
  __device__ __forceinline__ static int limit(const SwConst& sc) { return sc.s16Limit; }
};
template <>
struct Cell<LaneB16x2> {
  using V = LaneB16x2::V;
  __device__ __forceinline__ static V fterm(V f, V gIgE) {
    return LaneB16x2::addmax(f, gIgE, LaneB16x2::splat(0));
  }
  __device__ __forceinline__ static V ymax(V d, V s, V f) { return LaneB16x2::addmax(d, s, f); }
  __device__ __forceinline__ static V delta(int x) { return LaneB16x2::delta(x); }
  __device__ __forceinline__ static int limit(const SwConst& sc) { return sc.u16Limit; }
};

// -------------------------------------------------------------------------
// Pair views
// -------------------------------------------------------------------------

// Residue codes in device memory.  bits = 8: one byte per residue.  bits =
// 2, 4 or 5: a little-endian bit stream of fields, residue r in bits
// [bits * r, bits * r + bits), read through the two 32-bit words around it
// (one funnel shift); 2-bit fields hold code - 1 (A, T, C, G = codes 1..4),
// wider ones the code itself.  A packed array starts 4-byte aligned and is
// readable one word past the word of its last field.
__device__ __forceinline__ int code_at(const uint8_t* base, long long idx, int bits) {
  if (bits == 8) return base[idx];
  const long long bit = idx * bits;
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base) + (bit >> 5);
  const uint32_t v = __funnelshift_r(__ldg(w), __ldg(w + 1), (uint32_t)bit & 31u);
  const int x = (int)(v & ((1u << bits) - 1u));
  return bits == 2 ? x + 1 : x;
}

// Sequential reader of residues idx, idx + 1, ... of a packed code array
// (bits = 2, 4 or 5, layout as in code_at): one 32-bit load per word of the
// stream, each word loaded only once the next residue reaches into it.
struct PackedStream {
  const uint32_t* w;  // next word to load
  uint64_t buf;       // bits not yet consumed, lowest first
  int nbuf;           // valid bits in buf
  int bits;
  __device__ __forceinline__ PackedStream(const uint8_t* base, long long idx, int bits_) : bits(bits_) {
    const long long bit = idx * bits;
    w = reinterpret_cast<const uint32_t*>(base) + (bit >> 5);
    const int skip = (int)(bit & 31);
    buf = (uint64_t)__ldg(w++) >> skip;
    nbuf = 32 - skip;
  }
  __device__ __forceinline__ int next() {
    if (nbuf < bits) {
      buf |= (uint64_t)__ldg(w++) << nbuf;
      nbuf += 32;
    }
    const int x = (int)(buf & ((1u << bits) - 1u));
    buf >>= bits;
    nbuf -= bits;
    return bits == 2 ? x + 1 : x;
  }
};

// One sequence pair as seen by a pass: A[j] = residue a + j * da and
// B[i] = residue b + i * db of the code array at `base` (bits per residue
// in SwConst).  The reverse pass reads A[Aend..0] and B[Bend..0] with
// da = db = -1.
struct PassSeq {
  const uint8_t* base;
  long long a;
  long long b;
  int alen;
  int blen;
  int da;
  int db;
};

// Best cell of a pass: score, row (B index), column (A index).
struct Best {
  int s, i, j;
};

// The reference keeps the first strict maximum in (i, j) row-major order.
__device__ __forceinline__ bool better(int s1, int i1, int j1, int s2, int i2, int j2) {
  return s1 > s2 || (s1 == s2 && (i1 < i2 || (i1 == i2 && j1 < j2)));
}

// -------------------------------------------------------------------------
// Query profile of one group's strip: lane l's K columns of letter x at
// prof[x * LANES * KP + l * KP + c] = sim[A[col0 + l * K + c]][x] as int8,
// KP = K rounded up to whole 32-bit words (bytes c >= K are unused).  The
// profile has P + 1 rows: row x < P is letter x + pshift (2-bit A/C/G/T
// codes need only the rows of codes 1..4), row P (the padding letter) and
// columns past |A| hold SUB_PAD.
// -------------------------------------------------------------------------
template <int K>
struct ProfileWords {
  static constexpr int KP = ((K + 3) / 4) * 4;  // profile bytes per lane
  static constexpr int W = KP / 4;              // 32-bit words per lane
};

template <int K, int LANES>
__device__ __forceinline__ void build_profile(uint8_t* prof, const int8_t* s_simp, const SwConst& sc,
                                              const PassSeq& ps, int col0, int lane) {
  // s_simp[a * (M + 1) + x] = sim[a][x] and SUB_PAD for x == M.
  const int M = sc.M, P = sc.P, bits = sc.bits;
  constexpr int KP = ProfileWords<K>::KP;
  constexpr int SWP = LANES * KP;
  int acode[KP];
#pragma unroll
  for (int c = 0; c < KP; ++c) {
    const int col = col0 + lane * K + c;
    acode[c] = (c < K && col < ps.alen) ? code_at(ps.base, ps.a + (long long)col * ps.da, bits) : -1;
  }
  for (int x = 0; x <= P; ++x) {
    const int xs = x < P ? x + sc.pshift : M;  // column of s_simp
#pragma unroll
    for (int w = 0; w < KP / 4; ++w) {
      uint32_t word = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int a = acode[4 * w + q];
        const int v = (a >= 0) ? (int)s_simp[a * (M + 1) + xs] : SUB_PAD;
        word |= ((uint32_t)(uint8_t)(int8_t)v) << (8 * q);
      }
      *reinterpret_cast<uint32_t*>(prof + x * SWP + lane * KP + 4 * w) = word;
    }
  }
}

// Loads KB bytes (a multiple of 4) of a profile row into words.
template <int K>
__device__ __forceinline__ void load_profile_row(uint32_t (&w)[K / 4], const uint8_t* p) {
  if constexpr (K % 16 == 0) {
#pragma unroll
    for (int q = 0; q < K / 16; ++q) {
      uint4 v = reinterpret_cast<const uint4*>(p)[q];
      w[4 * q + 0] = v.x;
      w[4 * q + 1] = v.y;
      w[4 * q + 2] = v.z;
      w[4 * q + 3] = v.w;
    }
  } else if constexpr (K % 8 == 0) {
#pragma unroll
    for (int q = 0; q < K / 8; ++q) {
      uint2 v = reinterpret_cast<const uint2*>(p)[q];
      w[2 * q + 0] = v.x;
      w[2 * q + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < K / 4; ++q) w[q] = reinterpret_cast<const uint32_t*>(p)[q];
  }
}

template <int LANES>
__device__ __forceinline__ void group_best_reduce(int& s, int& i, int& j) {
#pragma unroll
  for (int off = LANES / 2; off > 0; off >>= 1) {
    int s2 = __shfl_xor_sync(FULL, s, off, LANES);
    int i2 = __shfl_xor_sync(FULL, i, off, LANES);
    int j2 = __shfl_xor_sync(FULL, j, off, LANES);
    if (better(s2, i2, j2, s, i, j)) {
      s = s2;
      i = i2;
      j = j2;
    }
  }
}

// Keep-mask of the running best: all-ones in the halfwords (or the word)
// where the row maximum `rm` does NOT exceed the best `b`.  For s16x2,
// rm + ~b = rm - b - 1 is negative exactly there; the halfword signs are
// replicated with prmt.  (The difference only leaves int16 for cells above
// the s16 limit, whose pair is then rerun in s32 lanes.)
__device__ __forceinline__ uint32_t keep_mask(LaneS16x2, uint32_t rm, uint32_t b) {
  return prmt(LaneS16x2::add(rm, ~b), 0u, 0xBB99u);
}
__device__ __forceinline__ uint32_t keep_mask(LaneS32, int rm, int b) {
  return (uint32_t)((rm + ~b) >> 31);
}

// Raises the running best `b` to the row maximum `rm` and returns the keep
// mask of the halves (or word) that did not improve.
template <class T>
__device__ __forceinline__ uint32_t update_best(T, typename T::V& b, typename T::V rm) {
  const uint32_t keep = keep_mask(T{}, rm, b);
  b = T::max2(b, rm);
  return keep;
}
// Biased halves of two scores may differ by more than 32767, so the
// signed-difference trick does not apply: each half is compared as a
// signed integer (a half keeps its best and its snapshot while rm <= b).
__device__ __forceinline__ uint32_t update_best(LaneB16x2, uint32_t& b, uint32_t rm) {
  const uint32_t keep_lo = ((int16_t)(rm & 0xffffu) <= (int16_t)(b & 0xffffu)) ? 0x0000ffffu : 0u;
  const uint32_t keep_hi = ((int16_t)(rm >> 16) <= (int16_t)(b >> 16)) ? 0xffff0000u : 0u;
  b = LaneB16x2::max2(b, rm);
  return keep_lo | keep_hi;
}

// Raises each lane's running best to the best of its group (per pair)
// minus one.  A row maximum strictly below a score that some cell of the
// pair already holds can never be the pair's answer, so after the raise
// only rows that can still win (ties included: the row order decides
// those) pass update_best and take the snapshot blend.  A lane left at the
// raised value holds no cell of that score, and its best stays below the
// group's, so it never wins the group reduction at the end of the strip.
template <class T, int LANES>
__device__ __forceinline__ typename T::V raise_to_group(typename T::V best) {
  typename T::V g = best;
#pragma unroll
  for (int off = LANES / 2; off > 0; off >>= 1)
    g = T::max2(g, (typename T::V)__shfl_xor_sync(FULL, g, off, LANES));
  return T::max2(best, T::add(g, Cell<T>::delta(-1)));
}

// -------------------------------------------------------------------------
// One full pass (forward or reverse) of one warp.
//
// The warp is split into 32 / LANES groups of LANES lanes; each group aligns
// its own NP pairs (`ps`, the lane's group) with a wavefront of LANES lanes,
// K columns per lane.  All groups step in lockstep (the shuffles span the
// warp) for the warp-wide maximum of rows and strips.  Steps run in blocks
// of LANES; blocks in which every lane of every group has a row to work on
// take an unrolled path without per-step activity checks.
//
// Returns false when s16x2 lanes gave up because a running best passed
// the lane's limit (Cell::limit, checked every 32 steps, warp-uniformly); the caller reruns
// the warp's pairs in s32 lanes.
//
//   s_prof   : this group's profile area, NP * (P + 1) * LANES * KP bytes
//   s_simp   : substitution table with the padding column (build_profile)
//   s_bring  : this group's rings of B letters, 64 entries per pair stored
//              twice (pair h at s_bring + 128 h, entry e also at e + 64, so
//              a block of steps reads base + k without wrapping), each the
//              byte offset of the letter's profile row (letter * LANES * KP)
//   scr      : this group's scratch, 2 * rowsCap int2 (only used when the
//              pass needs more than one strip)
//   out      : best cell per pair, in pass coordinates
// -------------------------------------------------------------------------
// HYB: three scratch buffers of rowsCap per group, and `ctl` in use -- an
// s16x2 pass (ctl->strip0 == 0) stops before an unsafe strip and reports
// it; an s32 pass with ctl->strip0 > 0 starts there from the packed
// boundary half ctl->bndHalf in buffer ctl->scrBase, keeping `out` (the
// best of the strips before) and using the two other buffers.
template <class T, int K, int LANES, bool HYB = false, bool EARLY = false, bool TEAM = false>
__device__ __forceinline__ bool sw_pass(const SwConst& sc, uint8_t* s_prof, const int8_t* s_simp,
                                        uint16_t* s_bring, const PassSeq (&ps)[T::NP], int2* scr,
                                        long rowsCap, Best (&out)[T::NP], PassCtl* ctl = nullptr,
                                        PassStop stop = PassStop{}, StripTeam team = StripTeam{}) {
  static_assert(!TEAM || (LANES == 32 && !HYB && !EARLY), "strip teams run whole-warp passes without an early stop");
  using V = typename T::V;
  constexpr int SW = LANES * K;          // columns per strip
  constexpr int KP = ProfileWords<K>::KP;
  constexpr int SWP = LANES * KP;        // profile bytes per letter
  constexpr int NP = T::NP;
  const int lane = threadIdx.x & (LANES - 1);
  const int P = sc.P;
  const int profStride = (P + 1) * SWP;
  const uint8_t* profP = s_prof + lane * KP;  // this lane's columns of pair P's profile
  const uint8_t* profQ = profP + profStride;  // ... and of pair Q's

  const int strip0 = HYB ? ctl->strip0 : 0;
  int rowsG = 0, amax = 0;
#pragma unroll
  for (int h = 0; h < NP; ++h) {
    rowsG = max(rowsG, ps[h].blen);
    amax = max(amax, ps[h].alen);
    if (strip0 == 0) {
      out[h].s = 0;
      out[h].i = 0;
      out[h].j = 0;
    }
  }
  int rowsW = __reduce_max_sync(FULL, rowsG);
  int rowsMin = __reduce_min_sync(FULL, rowsG);
  const int nstrips = (__reduce_max_sync(FULL, amax) + SW - 1) / SW;
  // EARLY: rows each pair still needs (its best row once it reached its
  // target), and this lane's group in the warp.
  int capRows[NP];
#pragma unroll
  for (int h = 0; h < NP; ++h) capRows[h] = ps[h].blen;
  const unsigned gmask = (LANES == 32) ? FULL : (((1u << LANES) - 1u) << (threadIdx.x & (32 - LANES)));
  using C = Cell<T>;
  const V vgE = C::delta(sc.gE);
  const V vgEp = C::delta(max(sc.gE, sc.gIgE));
  const V vgIgE = C::delta(sc.gIgE);
  // Ê handed to column 0 (and the initial hand-over value): -gE' makes the
  // first column's Ê come out as the reference's E = max(gI, H - gI) + gE.
  const V vE0 = T::splat(-max(sc.gE, sc.gIgE));
  const V vF0 = T::splat(-sc.gIgE);   // F̂ where F = 0 (pass start)
  const V vZero = T::splat(0);
  const int lim = C::limit(sc);
  // Steps unrolled in a check-free block: the block's code has to stay in
  // the instruction cache next to the checked path.
  // (Measured on B200: 8 steps for K <= 12, 4 for K = 16; the full LANES
  // steps stalled on instruction fetch.)
  constexpr int kStepUnroll = IPUMA_STEP_UNROLL > 0 ? (IPUMA_STEP_UNROLL < LANES ? IPUMA_STEP_UNROLL : LANES)
                                                   : (K > 12 ? 4 : 8);

  // Scratch buffer written by strip s: 0/1 alternating, or for an s32
  // continuation the two buffers other than the one holding its input.
  auto wbuf = [&](int sidx) -> int {
    if constexpr (TEAM) return sidx % team.warps;
    if (!HYB || strip0 == 0) return sidx & 1;
    return (ctl->scrBase + 1 + ((sidx - strip0) & 1)) % 3;
  };
  // H of the last column, maximum over rows, per half (HYB s16x2 pass):
  // the bound of the next strip.
  V bmax = vZero;

  // TEAM: marks the team as given up (overflow, or a wait that ran out).
  auto team_fail = [&]() {
    if constexpr (TEAM) {
      if (lane == 0) *(volatile int*)team.abort = 1;
    }
  };
  // TEAM: waits until the previous warp published `need` rows of strip
  // s's boundary.  Warp-uniform result; false once the team gave up.
  auto team_wait = [&](int s, int need) -> bool {
    bool ok = true;
    if constexpr (TEAM) {
      const int target = (s << 16) | need;
      const volatile int* pr = team.prog + (team.warp + team.warps - 1) % team.warps;
      const volatile int* ab = team.abort;
      unsigned long long t_start = 0;
      for (int it = 0; *pr < target; ++it) {
        if (*ab != 0) {
          ok = false;
          break;
        }
        if ((it & 255) == 0) {
          const unsigned long long now = global_ns();
          if (it == 0) t_start = now;
          if (now - t_start > kTeamWaitNs || it >= (1 << 26)) {
            atomicCAS(team.err, 0, team.errCode);
            *(volatile int*)team.abort = 1;
            ok = false;
            break;
          }
        }
        __nanosleep(64);
      }
      __threadfence_block();  // the boundary rows are read after the flag
      ok = __all_sync(FULL, ok);
    }
    return ok;
  };
  bool teamGaveUp = false;

  const int stripFirst = strip0 + (TEAM ? team.warp : 0);
  const int stripStep = TEAM ? team.warps : 1;
  for (int strip = stripFirst; strip < nstrips; strip += stripStep) {
    if constexpr (EARLY) {
      if (stop.on && strip > strip0) {
        rowsG = 0;
#pragma unroll
        for (int h = 0; h < NP; ++h) rowsG = max(rowsG, min(ps[h].blen, capRows[h]));
        rowsW = __reduce_max_sync(FULL, rowsG);
        rowsMin = __reduce_min_sync(FULL, rowsG);
        if (rowsW == 0) break;  // caps only shrink: no later strip can win
      }
    }
    const int col0 = strip * SW;
    const bool hasIn = strip > 0;
    const bool hasOut = strip + 1 < nstrips;
    const bool packedIn = HYB && strip == strip0 && strip0 > 0;  // unpack a half of the s16x2 boundary
    const int2* scrIn = scr + (packedIn ? ctl->scrBase : hasIn ? wbuf(strip - 1) : 0) * rowsCap;
    int2* scrOut = scr + wbuf(strip) * rowsCap;
    if constexpr (HYB && NP == 2) {
      if (strip > 0) {
        // Stop before a strip that could leave int16: the caller continues
        // each pair in s32 from the boundary this pass left behind.
        const V bm = __shfl_sync(FULL, bmax, LANES - 1, LANES);
        const int lim2 = lim - sc.maxSub * SW;
        if (__any_sync(FULL, T::half(bm, 0) > lim2 || T::half(bm, 1) > lim2)) {
          ctl->stoppedAt = strip;
          ctl->scrBase = wbuf(strip - 1);
          return true;
        }
        bmax = vZero;
      }
    }
    auto bnd = [&](int r) -> int2 {
      const int2 v = scrIn[r];
      if (HYB && NP == 1 && packedIn) {
        return make_int2(LaneHi::half((uint32_t)v.x, ctl->bndHalf), LaneHi::half((uint32_t)v.y, ctl->bndHalf));
      }
      return v;
    };

    __syncwarp();
#pragma unroll
    for (int h = 0; h < NP; ++h)
      build_profile<K, LANES>(s_prof + h * profStride, s_simp, sc, ps[h], col0, lane);
    __threadfence_block();
    __syncwarp();

    V H[K], Fh[K], snap[K];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      H[c] = vZero;
      Fh[c] = vF0;
      snap[c] = vZero;
    }
    V outY = vZero, outE = vE0, diagIn = vZero;
    // Running best of the lane, started one below the pair's best of the
    // strips before (a cell that ties it can still win on its row).
    V best = T::pack2(max(out[0].s - 1, 0), max(out[NP - 1].s - 1, 0));
    // Row of each lane's best, one halfword per pair (rows < 65536).
    uint32_t brow = 0;

    // Boundary (Y, Ê) of the previous strip's last column: lane k of the
    // group's chunk registers holds row (chunkBase + k).
    int2 chunk = make_int2(0, 0), chunkNext = make_int2(0, 0);
    if constexpr (TEAM) {
      if (hasIn && !team_wait(strip - 1, min(2 * LANES, rowsG))) {
        teamGaveUp = true;
        break;
      }
    }
    if (hasIn) {
      if (lane < rowsG) chunk = bnd(lane);
      if (LANES + lane < rowsG) chunkNext = bnd(LANES + lane);
    }

    // B letters, LANES rows at a time: lane k of `bnext` holds the profile
    // row offsets of row (t0 + LANES + k) (pair h in halfword h) and is
    // parked in the group's rings every LANES steps.
    auto fetch_letters = [&](int r) -> uint32_t {
      uint32_t v = 0;
#pragma unroll
      for (int h = 0; h < NP; ++h) {
        const int x = (r < ps[h].blen) ? code_at(ps[h].base, ps[h].b + (long long)r * ps[h].db, sc.bits) - sc.pshift : P;
        v |= (uint32_t)(x * SWP) << (16 * h);
      }
      return v;
    };
    uint32_t bnext = fetch_letters(lane);

    // Ring slot of this lane's row at the first step of the current block.
    int ringBase = 0;

    // One wavefront step, step k of the block starting at t0 = t - k: lane
    // works on row t - lane (when CHECK, only if that row exists for its
    // group).
    auto step = [&](int t, int k, auto check) {
      V recvY = __shfl_up_sync(FULL, outY, 1, LANES);
      V recvE = __shfl_up_sync(FULL, outE, 1, LANES);
      if (hasIn) {
        const int bx = __shfl_sync(FULL, chunk.x, k, LANES);
        const int by = __shfl_sync(FULL, chunk.y, k, LANES);
        if (lane == 0) {
          recvY = (V)bx;
          recvE = (V)by;
        }
      } else if (lane == 0) {
        recvY = vZero;
        recvE = vE0;
      }
      // H of the left neighbour's last column, the next row's diagonal.
      const V diag0 = diagIn;
      diagIn = T::addmax(recvE, vgIgE, recvY);
      const int i = t - lane;
      if (!decltype(check)::value || (i >= 0 && i < rowsG)) {
        uint32_t wp[KP / 4], wq[KP / 4];
        const int slot = ringBase + k;  // (i mod 64), < 64 + LANES
        load_profile_row<KP>(wp, profP + s_bring[slot]);
        if constexpr (NP == 2) {
          load_profile_row<KP>(wq, profQ + s_bring[128 + slot]);
        } else {
#pragma unroll
          for (int q = 0; q < KP / 4; ++q) wq[q] = 0;
        }
        // The left neighbour hands over (Y, Ê) of its last column; lane 0
        // of the first strip starts the row with Y = 0, Ê = -gE.
        V yl = recvY;
        V e = recvE;
        V diag = diag0;
#pragma unroll
        for (int c = 0; c < K; ++c) {
          V sb;
          switch (c & 3) {
            case 0: sb = T::template sub<0>(wp[c >> 2], wq[c >> 2]); break;
            case 1: sb = T::template sub<1>(wp[c >> 2], wq[c >> 2]); break;
            case 2: sb = T::template sub<2>(wp[c >> 2], wq[c >> 2]); break;
            default: sb = T::template sub<3>(wp[c >> 2], wq[c >> 2]); break;
          }
          const V f = T::addmax(Fh[c], vgE, H[c]);                   // F̂
          const V y = C::ymax(diag, sb, C::fterm(f, vgIgE));         // Y
          e = T::addmax(e, vgEp, yl);                                // Ê
          const V hv = T::addmax(e, vgIgE, y);                       // H
          diag = H[c];
          H[c] = hv;
          Fh[c] = f;
          yl = y;
        }
        outY = yl;
        outE = e;
        // Row maximum of the lane (full-rate 2-input max tree).
        V m8[(K + 1) / 2];
#pragma unroll
        for (int c = 0; c < K / 2; ++c) m8[c] = T::max2(H[2 * c], H[2 * c + 1]);
        if constexpr (K & 1) m8[K / 2] = H[K - 1];
#pragma unroll
        for (int w = 1; w < (K + 1) / 2; w *= 2)
#pragma unroll
          for (int c = 0; c + w < (K + 1) / 2; c += 2 * w) m8[c] = T::max2(m8[c], m8[c + w]);
        const V rm = m8[0];
        // Running best of this lane: strict > keeps the first row.
        // With two pairs per lane (16-bit halves) the blend runs on every
        // step, improved or not: some lane of the warp improves on most
        // steps, and a branch around it cost more than it saved (measured
        // on B200: +1 % DNA, +3 % protein batches).  With one pair per
        // warp (s32 lanes) improvements are rarer and the branch pays
        // (the plain s32 kernel ran 16-20 % slower without it).
        const uint32_t keep = update_best(T{}, best, rm);
        if (NP == 2 || keep != 0xffffffffu) {
          const uint32_t ipk = (uint32_t)i * 0x00010001u;  // row in both halfwords
          brow = (brow & keep) | (ipk & ~keep);
#pragma unroll
          for (int c = 0; c < K; ++c) snap[c] = (V)(((uint32_t)snap[c] & keep) | ((uint32_t)H[c] & ~keep));
        }
        if (hasOut && lane == LANES - 1) scrOut[i] = make_int2((int)outY, (int)outE);
        if constexpr (HYB && NP == 2) bmax = T::max2(bmax, T::addmax(outE, vgIgE, outY));
      }
    };

    const int nsteps = rowsW + LANES - 1;
    bool gaveUp = false;
    int stopAt = nsteps;  // EARLY: end of the block after every pair is done
    for (int t0 = 0; t0 < nsteps; t0 += LANES) {
      if constexpr (EARLY) {
        if (t0 >= stopAt) break;
        if (stop.on && stopAt == nsteps) {
          // A pair is done once its group reached the target (before t0, so
          // the slowest lane passes that row within this block) or all
          // lanes are past its rows.  Warp-uniform.
          bool done = true;
#pragma unroll
          for (int h = 0; h < NP; ++h) {
            const bool found = (__ballot_sync(FULL, T::half(best, h) >= stop.target[h]) & gmask) != 0;
            done = done && (found || t0 - (LANES - 1) >= min(ps[h].blen, capRows[h]));
          }
          if (__all_sync(FULL, done)) stopAt = t0 + LANES;
        }
      }
      if constexpr (NP == 2) {
        if ((t0 & 31) == 0) {
          // A cell above s16Limit could overflow the next additions.
          const bool hi = T::half(best, 0) > lim || T::half(best, 1) > lim;
          if (__any_sync(FULL, hi)) {
            gaveUp = true;
            break;
          }
        }
      }
      if constexpr (TEAM) {
        // Another warp gave up: this pass's results are not used.
        if (__any_sync(FULL, *(volatile int*)team.abort != 0)) {
          teamGaveUp = true;
          break;
        }
      }
      if (t0 > 0) best = raise_to_group<T, LANES>(best);
      {
        const int w = (t0 + lane) & 63;
        s_bring[w] = s_bring[w + 64] = (uint16_t)bnext;
        if constexpr (NP == 2) s_bring[128 + w] = s_bring[192 + w] = (uint16_t)(bnext >> 16);
      }
      ringBase = (t0 - lane) & 63;
      bnext = fetch_letters(t0 + LANES + lane);
      __syncwarp();
      if (hasIn && t0 > 0) {
        if constexpr (TEAM) {
          if (!team_wait(strip - 1, min(t0 + 2 * LANES, rowsG))) {
            teamGaveUp = true;
            break;
          }
        }
        chunk = chunkNext;
        const int r = t0 + LANES + lane;
        chunkNext = (r < rowsG) ? bnd(r) : make_int2(0, 0);
      }
      if (t0 >= LANES - 1 && t0 + LANES - 1 < rowsMin) {
#pragma unroll kStepUnroll
        for (int k = 0; k < LANES; ++k) step(t0 + k, k, std::false_type{});
      } else {
#pragma unroll 1
        for (int k = 0; k < LANES; ++k) step(t0 + k, k, std::true_type{});
      }
      if constexpr (TEAM) {
        // Lane LANES - 1 wrote the boundary rows up to t0 (those below
        // rowsG): release them to the next strip's warp.
        if (hasOut && lane == LANES - 1) {
          __threadfence_block();
          *(volatile int*)(team.prog + team.warp) = (strip << 16) | min(t0 + 1, rowsG);
        }
      }
    }
    if constexpr (TEAM) {
      if (teamGaveUp) break;
    }

    if constexpr (NP == 2) {
      if (!gaveUp) gaveUp = __any_sync(FULL, T::half(best, 0) > lim || T::half(best, 1) > lim);
      if (gaveUp) {
        team_fail();
        return false;
      }
    }
    // Strip result: first column of the lane's snapshot that holds its best.
#pragma unroll
    for (int h = 0; h < NP; ++h) {
      const int bg = T::half(best, h);
      int s = bg;
      int jj = 0;
#pragma unroll
      for (int c = K - 1; c >= 0; --c)
        if (T::half(snap[c], h) == bg) jj = c;
      int ii = (NP == 1) ? (int)(brow & 0xffffu) : (int)((brow >> (16 * h)) & 0xffffu);
      int j = col0 + lane * K + jj;
      if (s <= 0) {
        s = 0;
        ii = 0;
        j = 0;
      }
      group_best_reduce<LANES>(s, ii, j);
      if (better(s, ii, j, out[h].s, out[h].i, out[h].j)) {
        out[h].s = s;
        out[h].i = ii;
        out[h].j = j;
      }
      if constexpr (EARLY) {
        if (stop.on && out[h].s >= stop.target[h]) capRows[h] = min(capRows[h], out[h].i);
      }
    }
    if (hasOut) {
      __threadfence_block();
      __syncwarp();
    }
  }
  if constexpr (TEAM) {
    if (teamGaveUp) return false;
  }
  return true;
}

}  // namespace ipuma_dev
