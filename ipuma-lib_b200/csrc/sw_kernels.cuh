// sw_kernels.cuh -- the __global__ kernels of the engine.
//
//   k_batched<T, K, LANES>  persistent kernel over a cost-ordered work list;
//                     each warp pulls work items (per group of LANES lanes one
//                     pair for s32 lanes, two for 16-bit halves) from an
//                     atomic queue head.  s16x2 items whose score could have
//                     left int16 are appended to an overflow list that a
//                     second k_batched<LaneS32, K> launch reruns.
//   k_plain<K>        the one-launch-per-batch kernel over the reference's
//                     wire buffer (Seqs || Meta, ipu_batch_affine.cpp:287) with
//                     results in its Scores || ARanges || BRanges layout; one
//                     warp per comparison slot in slot order, s32 lanes.
//   k_exact           one thread per pair with the recurrence written out
//                     cell by cell in int32; used for scoring configurations
//                     that the wavefront kernels do not cover (gI + gE >= 0 or
//                     gE > 0).
//   k_plain16<K>      the same wire-buffer kernel with two slots per warp in
//                     s16x2 halves (a slot that could leave int16 is redone
//                     in s32 by the same warp).
//   k_strips<K>       the strip-team kernel: the warps of a block share the
//                     strips of one item (two pairs in s16x2 halves), each
//                     strip waiting on the boundary rows of the one before
//                     (long pairs whose latency would end the launch).
//   k_bin_*           the cost-binning pre-pass that orders the work list:
//                     k_bin_total (batch cells), k_bin_bound (main-diagonal
//                     bounds of the long pairs, a warp per pair), k_bin_count
//                     (class and bucket of every pair), k_bin_scan (list
//                     offsets and class shares), k_bin_scatter (the list).
#pragma once
#include "sw_device.cuh"

namespace ipuma_dev {

// Pair descriptor of the batched API (matches ipuma_pair in ipuma_b200.h).
struct PairDesc {
  long long a_off;
  long long b_off;
  int a_len;
  int b_len;
};

// Packs (start, end) like codelet_batch_affine.cpp:117-123 (uint16 halves).
__device__ __forceinline__ int pack_range(int start, int end) {
  return (int)(((uint32_t)(uint16_t)start) | (((uint32_t)(uint16_t)end) << 16));
}

// Device-side status words (bounded error reporting, no traps).
struct DevStatus {
  int error;           // first error code seen by any warp (0 = none)
  int overflow_start;  // always 0: {overflow_start, overflow_count} is the
  int overflow_count;  // range of the overflow list for the s32 rerun
  int pad;
};

// Share of the GPU one class launch may use: blocks with blockIdx.x >=
// `blocks` exit at once, and the launch's strip scratch starts `base` int2
// into the scratch buffer.  Written on the device by the binning pre-pass
// (k_bin_scan) so that concurrent class launches split the SMs in
// proportion to their modelled work and never share scratch.
struct ClassAllot {
  long long base;
  int blocks;
  int pad;
};

constexpr int ERR_SCRATCH = 1;  // a pass needed more scratch rows than provided
constexpr int ERR_LENGTH = 2;   // a pair exceeded the stated maximum lengths
constexpr int ERR_RANGE = 3;    // a pair's offsets or lengths lie outside the code array
constexpr int ERR_WAIT = 4;     // a strip team's wait for a boundary ran out (kTeamWaitNs)

// What a kernel does with one pair descriptor of a device-resident batch,
// checked before any code is read (the same rules as the host-side check of
// the host-buffer calls): PAIR_OUT for a negative offset or length or a
// sequence reaching past the n_codes residues of the code array (error
// status, zero result), PAIR_EMPTY for an empty sequence (zero result),
// PAIR_LONG beyond the stated maxima (error status, zero result), PAIR_OK.
constexpr int PAIR_OK = 0, PAIR_EMPTY = 1, PAIR_LONG = 2, PAIR_OUT = 3;
__device__ __forceinline__ int pair_state(const PairDesc& d, long long n_codes, int max_a, int max_b) {
  if (d.a_len < 0 || d.b_len < 0 || d.a_off < 0 || d.b_off < 0 || d.a_off > n_codes - d.a_len ||
      d.b_off > n_codes - d.b_len)
    return PAIR_OUT;
  if (d.a_len == 0 || d.b_len == 0) return PAIR_EMPTY;
  if (d.a_len > max_a || d.b_len > max_b) return PAIR_LONG;
  return PAIR_OK;
}

// Records the error of a rejected pair (PAIR_LONG / PAIR_OUT) in the status
// word; the caller writes its zero result.
__device__ __forceinline__ void report_pair(int state, DevStatus* st) {
  if (state == PAIR_LONG) atomicCAS(&st->error, 0, ERR_LENGTH);
  if (state == PAIR_OUT) atomicCAS(&st->error, 0, ERR_RANGE);
}

// Shared-memory layout of the wavefront kernels.
// Per warp: 32 / LANES groups, each with its profile and B-letter ring.
template <class T, int K, int LANES>
struct SmemLayout {
  static constexpr int SW = LANES * K;
  static constexpr int GROUPS = 32 / LANES;
  // M = alphabet size (substitution table), P = letters of the profile.
  __host__ __device__ static int simp_bytes(int M) { return ((M * (M + 1)) + 15) & ~15; }
  __host__ __device__ static int prof_bytes(int P) { return T::NP * (P + 1) * LANES * ProfileWords<K>::KP; }
  __host__ __device__ static int ring_bytes() { return 128 * 2 * T::NP; }  // a doubled uint16 ring per pair
  __host__ __device__ static int group_bytes(int P) { return (prof_bytes(P) + ring_bytes() + 15) & ~15; }
  __host__ __device__ static int warp_bytes(int P) { return GROUPS * group_bytes(P); }
  __host__ __device__ static int total(int M, int P, int warps) { return simp_bytes(M) + warps * warp_bytes(P); }
};

// Loads the substitution table with its padding column: simp[a][x] =
// sim[a][x] for x < M, SUB_PAD for x == M.
__device__ __forceinline__ void load_simp(int8_t* s_simp, const int8_t* sim, const SwConst& sc) {
  const int M = sc.M;
  for (int k = threadIdx.x; k < M * (M + 1); k += blockDim.x) {
    const int a = k / (M + 1), x = k % (M + 1);
    s_simp[k] = (x < M) ? sim[a * M + x] : (int8_t)SUB_PAD;
  }
}

// Forward pass (+ reverse pass unless forwardOnly) for the NP pairs held
// by one lane group.  For 16-bit lanes a pair whose score exceeds the
// lane's limit (or any pair of a warp that gave up) is flagged in `ovf` and
// gets no reverse pass (the s32 rerun redoes it).
// MODE: 0 = by sc.forwardOnly at run time, 1 = forward only, 2 = with the
// reverse pass (a kernel specialised for one mode holds only its code, so
// the forward-only kernels keep their own register allocation).
template <class T, int K, int LANES, int MODE = 0>
__device__ __forceinline__ void align_pairs(const SwConst& sc, uint8_t* s_prof,
                                            const int8_t* s_simp, uint16_t* s_bring, const uint8_t* codes,
                                            const long long (&a0)[T::NP], const long long (&b0)[T::NP],
                                            const int (&alen)[T::NP], const int (&blen)[T::NP],
                                            int2* scr, long rowsCap, Best (&fw)[T::NP],
                                            Best (&rv)[T::NP], bool (&ovf)[T::NP]) {
  constexpr int NP = T::NP;
  PassSeq ps[NP];
#pragma unroll
  for (int h = 0; h < NP; ++h) {
    const bool empty = alen[h] <= 0 || blen[h] <= 0;
    ps[h] = PassSeq{codes, a0[h], b0[h], empty ? 0 : alen[h], empty ? 0 : blen[h], 1, 1};
  }
#pragma unroll
  for (int h = 0; h < NP; ++h) rv[h] = Best{0, 0, 0};
  if (MODE == 1 || (MODE == 0 && sc.forwardOnly)) {
    if constexpr (MODE != 2) {
      const bool done = sw_pass<T, K, LANES>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, fw);
#pragma unroll
      for (int h = 0; h < NP; ++h) ovf[h] = (NP == 2) && (!done || fw[h].s > Cell<T>::limit(sc));
    }
    return;
  }
  if constexpr (MODE != 1) {
  // With start coordinates both passes run through one copy of sw_pass: two
  // inlined copies alternating in the instruction cache slowed both down.
  // (A forward-only launch runs only the copy above.)  The reverse pass
  // stops early once every pair reached its forward score (PassStop).
  // Only the kernels specialised for full alignments (MODE 2) take the
  // early stop: it costs registers that the others keep.
  PassStop stop;
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    Best res[NP];
    const bool done = sw_pass<T, K, LANES, false, MODE == 2>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, res,
                                                              nullptr, stop);
    if (pass == 1) {
#pragma unroll
      for (int h = 0; h < NP; ++h) rv[h] = res[h];
      break;
    }
    bool any = false;
#pragma unroll
    for (int h = 0; h < NP; ++h) {
      fw[h] = res[h];
      ovf[h] = (NP == 2) && (!done || fw[h].s > Cell<T>::limit(sc));
      const bool run = !ovf[h] && fw[h].s > 0;
      any |= run;
      ps[h] = run ? PassSeq{codes, a0[h] + fw[h].j, b0[h] + fw[h].i, fw[h].j + 1, fw[h].i + 1, -1, -1}
                  : PassSeq{codes, a0[h], b0[h], 0, 0, 1, 1};
      stop.target[h] = run ? fw[h].s : 0;
    }
    stop.on = true;
    // Uniform across the warp: every group takes part in the shuffles.
    if (!__any_sync(FULL, any)) break;
  }
  }
}

// One pass of the hybrid class for the two pairs of a 32-lane group: s16x2
// while every strip is provably inside int16, then each pair alone in s32
// lanes from the first strip that is not (its half of the packed boundary
// column as input).  Returns false when the s16x2 part gave up anyway.
template <int K>
__device__ __forceinline__ bool hybrid_pass(const SwConst& sc, uint8_t* s_prof, const int8_t* s_simp,
                                            uint16_t* s_bring, const PassSeq (&ps)[2], int2* scr,
                                            long rowsCap, Best (&out)[2]) {
  PassCtl c16;
  if (!sw_pass<LaneHi, K, 32, true>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, out, &c16)) return false;
  if (c16.stoppedAt < 0) return true;
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    if (ps[h].alen <= c16.stoppedAt * 32 * K || ps[h].blen <= 0) continue;  // no strip left
    PassCtl c32;
    c32.strip0 = c16.stoppedAt;
    c32.bndHalf = h;
    c32.scrBase = c16.scrBase;
    const PassSeq one[1] = {ps[h]};
    Best o[1] = {out[h]};
    sw_pass<LaneS32, K, 32, true>(sc, s_prof, s_simp, s_bring, one, scr, rowsCap, o, &c32);
    out[h] = o[0];
  }
  return true;
}

// Forward (+ reverse) pass of the hybrid class; as align_pairs (MODE too).
template <int K, int MODE = 0>
__device__ __forceinline__ void align_pairs_hybrid(const SwConst& sc, uint8_t* s_prof, const int8_t* s_simp,
                                                   uint16_t* s_bring, const uint8_t* codes,
                                                   const long long (&a0)[2], const long long (&b0)[2],
                                                   const int (&alen)[2], const int (&blen)[2], int2* scr,
                                                   long rowsCap, Best (&fw)[2], Best (&rv)[2], bool (&ovf)[2]) {
  PassSeq ps[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const bool empty = alen[h] <= 0 || blen[h] <= 0;
    ps[h] = PassSeq{codes, a0[h], b0[h], empty ? 0 : alen[h], empty ? 0 : blen[h], 1, 1};
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) rv[h] = Best{0, 0, 0};
  if (MODE == 1 || (MODE == 0 && sc.forwardOnly)) {
    if constexpr (MODE != 2) {
      const bool done = hybrid_pass<K>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, fw);
      ovf[0] = ovf[1] = !done;
    }
    return;
  }
  if constexpr (MODE != 1) {
  // With start coordinates one copy of the hybrid pass serves both
  // directions (as align_pairs).
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    Best res[2];
    const bool done = hybrid_pass<K>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, res);
    if (pass == 1) {
      if (done) {
        rv[0] = res[0];
        rv[1] = res[1];
      } else {
        ovf[0] = ovf[1] = true;
      }
      break;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      fw[h] = res[h];
      ovf[h] = !done;
      ps[h] = fw[h].s > 0 ? PassSeq{codes, a0[h] + fw[h].j, b0[h] + fw[h].i, fw[h].j + 1, fw[h].i + 1, -1, -1}
                          : PassSeq{codes, a0[h], b0[h], 0, 0, 1, 1};
    }
    if (!done) break;
  }
  }
}

__device__ __forceinline__ void write_result(const SwConst& sc, const Best& fw, const Best& rv,
                                             int* score, int* arange, int* brange, long idx) {
  const int aend = fw.j, bend = fw.i;
  const int astart = sc.forwardOnly ? 0 : aend - rv.j;
  const int bstart = sc.forwardOnly ? 0 : bend - rv.i;
  score[idx] = fw.s;
  arange[idx] = pack_range(astart, aend);
  brange[idx] = pack_range(bstart, bend);
}

// Persistent batched kernel.  `list` holds pair ids in processing order;
// a warp takes items of 32 / LANES * NP consecutive entries (ids < 0 are
// padding), lane group g aligning entries [g * NP, g * NP + NP).
// Register budget: the forward-only kernels get at most 128 registers (4
// blocks of 128 threads per SM when the profile is small); the kernels
// with a reverse pass or a run-time mode (FWD false, or the hybrid class)
// up to 170 (3 blocks per SM, which their shared memory allows anyway), as
// at 128 they spilled.
template <class T, int K, int LANES, bool HYB = false, bool FWD = false>
__global__ void __launch_bounds__(128, (FWD && !HYB) ? 4 : 3) k_batched(SwConst sc, const int8_t* __restrict__ sim,
                                                 const uint8_t* __restrict__ codes,
                                                 const PairDesc* __restrict__ pairs,
                                                 const int* __restrict__ list,
                                                 const int* __restrict__ range, int* queue_head,
                                                 int2* scratch, long rowsCap, int* score,
                                                 int* arange, int* brange, int* overflow_list,
                                                 unsigned long long* rerun_cells, DevStatus* st,
                                                 const ClassAllot* __restrict__ allot,
                                                 unsigned long long* trace) {
  if ((int)blockIdx.x >= allot->blocks) return;  // outside this launch's share
  scratch += allot->base;
  // trace (option "trace"): {~first block start, last warp end} of the launch.
  if (trace && threadIdx.x == 0) atomicMax(&trace[0], ~global_ns());
  using L = SmemLayout<T, K, LANES>;
  constexpr int NP = T::NP;
  constexpr int GROUPS = L::GROUPS;
  constexpr int PER_ITEM = GROUPS * NP;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warps = blockDim.x >> 5;
  const int wib = threadIdx.x >> 5;
  const int lane32 = threadIdx.x & 31;
  const int group = lane32 / LANES;
  const int glane = lane32 & (LANES - 1);
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* gbase = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.P) + group * L::group_bytes(sc.P);
  uint8_t* s_prof = gbase;
  uint16_t* s_bring = reinterpret_cast<uint16_t*>(gbase + L::prof_bytes(sc.P));
  load_simp(s_simp, sim, sc);
  __syncthreads();

  // range = {first list entry, number of entries}, written by the binning
  // pre-pass (or the overflow counter) on the device.
  const int n = range[1];
  list += range[0];
  const int items = (n + PER_ITEM - 1) / PER_ITEM;
  const long gw = (long)blockIdx.x * warps + wib;
  constexpr int NBUF = HYB ? 3 : 2;  // strip-boundary buffers per group
  int2* scr = scratch + (gw * GROUPS + group) * NBUF * rowsCap;
  while (true) {
    int item = 0;
    if (lane32 == 0) item = atomicAdd(queue_head, 1);
    item = __shfl_sync(FULL, item, 0);
    if (item >= items) break;
    int pid[NP], alen[NP], blen[NP];
    long long a0[NP], b0[NP];
    bool tooLong = false;
#pragma unroll
    for (int h = 0; h < NP; ++h) {
      const int k = item * PER_ITEM + group * NP + h;
      pid[h] = (k < n) ? list[k] : -1;
      PairDesc d = (pid[h] >= 0) ? pairs[pid[h]] : PairDesc{0, 0, 0, 0};
      alen[h] = d.a_len;
      blen[h] = d.b_len;
      a0[h] = d.a_off;
      b0[h] = d.b_off;
      tooLong |= d.b_len > rowsCap;
    }
    if (__any_sync(FULL, tooLong)) {
      // The host sizes the scratch for the longest B; report, never trap.
      if (lane32 == 0) atomicCAS(&st->error, 0, ERR_SCRATCH);
      continue;
    }
    Best fw[NP], rv[NP];
    bool ovf[NP];
    if constexpr (HYB) {
      static_assert(NP == 2 && LANES == 32, "the hybrid class pairs two s16x2 pairs per 32-lane warp");
      // Mode chosen at run time: specialising the hybrid class made its
      // forward-only kernel spill and slowed the heavy-tailed protein batch.
      align_pairs_hybrid<K, 0>(sc, s_prof, s_simp, s_bring, codes, a0, b0, alen, blen, scr, rowsCap, fw, rv,
                               ovf);
    } else {
      // s16x2 classes: one kernel per mode (fewer registers, no spills for
      // forward-only; the early reverse stop for full alignments); the s32
      // class keeps the run-time choice for the same reason as the hybrid.
      constexpr int MODE = (T::NP == 1) ? 0 : (FWD ? 1 : 2);
      align_pairs<T, K, LANES, MODE>(sc, s_prof, s_simp, s_bring, codes, a0, b0, alen, blen, scr, rowsCap, fw, rv,
                                     ovf);
    }
    if (glane == 0) {
#pragma unroll
      for (int h = 0; h < NP; ++h) {
        if (pid[h] < 0) continue;
        if (ovf[h]) {
          const int slot = atomicAdd(&st->overflow_count, 1);
          overflow_list[slot] = pid[h];
          if (rerun_cells)
            atomicAdd(rerun_cells, (unsigned long long)alen[h] * (unsigned long long)blen[h]);
          continue;
        }
        write_result(sc, fw[h], rv[h], score, arange, brange, pid[h]);
      }
    }
  }
  if (trace && lane32 == 0) atomicMax(&trace[1], global_ns());
}

// Strip-team kernel: the blockDim.x / 32 warps of a block align one item
// (the two pairs of a 32-lane s16x2 group), taking its 32 * K wide strips
// round robin (sw_pass with TEAM), so a long pair finishes up to `warps`
// times sooner than on one warp.  Each warp keeps the best cell of its own
// strips; the block merges them with the first-strict-maximum order
// (better), the order-independent total order the one-warp pass applies
// strip by strip.  With start coordinates the team then runs the reverse
// pass the same way.  A team that gave up (a 16-bit overflow, or a wait
// past kTeamWaitNs, which also sets ERR_WAIT) sends both pairs to the s32
// rerun.  Block scratch: `warps` boundary columns of rowsCap rows.
constexpr int kTeamMaxWarps = 8;
template <int K>
__global__ void __launch_bounds__(256, 2) k_strips(SwConst sc, const int8_t* __restrict__ sim,
                                                   const uint8_t* __restrict__ codes,
                                                   const PairDesc* __restrict__ pairs,
                                                   const int* __restrict__ list, const int* __restrict__ range,
                                                   int* queue_head, int2* scratch, long rowsCap, int* score,
                                                   int* arange, int* brange, int* overflow_list,
                                                   unsigned long long* rerun_cells, DevStatus* st,
                                                   const ClassAllot* __restrict__ allot,
                                                   unsigned long long* trace) {
  if ((int)blockIdx.x >= allot->blocks) return;
  scratch += allot->base;
  if (trace && threadIdx.x == 0) atomicMax(&trace[0], ~global_ns());
  using T = LaneS16x2;
  using L = SmemLayout<T, K, 32>;
  constexpr int NP = 2;
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ int s_prog[kTeamMaxWarps];
  __shared__ int s_abort, s_item;
  __shared__ Best s_res[kTeamMaxWarps][NP];
  __shared__ Best s_best[2][NP];  // merged best of the forward / reverse pass
  __shared__ bool s_ovf[NP];
  const int warps = blockDim.x >> 5;
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* s_prof = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.P);
  uint16_t* s_bring = reinterpret_cast<uint16_t*>(s_prof + L::prof_bytes(sc.P));
  load_simp(s_simp, sim, sc);

  const int n = range[1];
  list += range[0];
  const int items = (n + NP - 1) / NP;
  int2* scr = scratch + (long)blockIdx.x * warps * rowsCap;
  const StripTeam team{s_prog, &s_abort, &st->error, ERR_WAIT, wib, warps};
  while (true) {
    __syncthreads();  // the previous item's merge is done; s_simp is loaded
    if (threadIdx.x == 0) {
      s_item = atomicAdd(queue_head, 1);
      s_abort = 0;
    }
    if (threadIdx.x < warps) s_prog[threadIdx.x] = -1;
    __syncthreads();
    const int item = s_item;
    if (item >= items) break;
    int pid[NP];
    PairDesc d[NP];
    bool tooLong = false;
#pragma unroll
    for (int h = 0; h < NP; ++h) {
      const int k = item * NP + h;
      pid[h] = (k < n) ? list[k] : -1;
      d[h] = (pid[h] >= 0) ? pairs[pid[h]] : PairDesc{0, 0, 0, 0};
      tooLong |= d[h].b_len > rowsCap;
    }
    if (tooLong) {
      // The host sizes the scratch for the longest B; report, never trap.
      if (threadIdx.x == 0) atomicCAS(&st->error, 0, ERR_SCRATCH);
      continue;
    }
    PassSeq ps[NP];
#pragma unroll
    for (int h = 0; h < NP; ++h) {
      const bool empty = d[h].a_len <= 0 || d[h].b_len <= 0;
      ps[h] = PassSeq{codes, d[h].a_off, d[h].b_off, empty ? 0 : d[h].a_len, empty ? 0 : d[h].b_len, 1, 1};
    }
    // Pass 0: forward.  Pass 1 (with start coordinates): the same pass over
    // the reversed reads from each pair's end cell (as align_pairs, without
    // the early stop), whose first strict maximum gives the start.  One
    // copy of sw_pass serves both.
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      Best out[NP];
      sw_pass<T, K, 32, false, false, true>(sc, s_prof, s_simp, s_bring, ps, scr, rowsCap, out, nullptr,
                                            PassStop{}, team);
      if (lane == 0) {
#pragma unroll
        for (int h = 0; h < NP; ++h) s_res[wib][h] = out[h];
      }
      __syncthreads();
      if (threadIdx.x < NP) {
        const int h = threadIdx.x;
        Best b = s_res[0][h];
        for (int w = 1; w < warps; ++w) {
          const Best c = s_res[w][h];
          if (better(c.s, c.i, c.j, b.s, b.i, b.j)) b = c;
        }
        s_best[pass][h] = b;
        // A team that gave up (in either pass) sends the pair to the rerun.
        if (pass == 0) {
          s_ovf[h] = s_abort != 0 || b.s > Cell<T>::limit(sc);
          s_best[1][h] = Best{0, 0, 0};  // the start of a pair without a reverse pass
        }
        if (pass == 1 && s_abort != 0) s_ovf[h] = true;
      }
      __syncthreads();
      if (pass == 1 || sc.forwardOnly) break;
      bool any = false;
#pragma unroll
      for (int h = 0; h < NP; ++h) {
        const Best fw = s_best[0][h];
        const bool run = pid[h] >= 0 && !s_ovf[h] && fw.s > 0;
        any |= run;
        ps[h] = run ? PassSeq{codes, d[h].a_off + fw.j, d[h].b_off + fw.i, fw.j + 1, fw.i + 1, -1, -1}
                    : PassSeq{codes, d[h].a_off, d[h].b_off, 0, 0, 1, 1};
      }
      if (!any) break;  // block-uniform: every thread read the same words
      // A fresh team for the reverse pass (after every warp read s_ovf).
      __syncthreads();
      if (threadIdx.x == 0) s_abort = 0;
      if (threadIdx.x < warps) s_prog[threadIdx.x] = -1;
      __syncthreads();
    }
    if (threadIdx.x < NP) {
      const int h = threadIdx.x;
      if (pid[h] >= 0) {
        if (s_ovf[h]) {
          const int slot = atomicAdd(&st->overflow_count, 1);
          overflow_list[slot] = pid[h];
          if (rerun_cells) atomicAdd(rerun_cells, (unsigned long long)d[h].a_len * (unsigned long long)d[h].b_len);
        } else {
          write_result(sc, s_best[0][h], s_best[1][h], score, arange, brange, pid[h]);
        }
      }
    }
  }
  if (trace && lane == 0) atomicMax(&trace[1], global_ns());
}

// One-launch-per-batch kernel over the reference wire buffer.
// Comparison slot g = tile * maxBatches + slot reads Meta[4g..4g+3] =
// {a_len, a_off, b_len, b_off}, byte offsets into the tile's Seqs region
// (ipu_batch_affine.cpp:164-167, 881-884), and writes Scores[g],
// ARanges[g], BRanges[g] of the output buffer (ipu_batch_affine.cpp:208-210,
// 288).  Warps take slots g = warp, warp + nwarps, ... in slot order.
template <int K>
__global__ void __launch_bounds__(128) k_plain(SwConst sc, const int8_t* __restrict__ sim,
                                               const int* __restrict__ inputs, long seqWordsPerTile,
                                               long metaOffset, int maxBatches, int totalSlots,
                                               int2* scratch, long rowsCap, int* results,
                                               DevStatus* st) {
  using T = LaneS32;
  using L = SmemLayout<T, K, 32>;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warps = blockDim.x >> 5;
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* wbase = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.P);
  uint8_t* s_prof = wbase;
  uint16_t* s_bring = reinterpret_cast<uint16_t*>(wbase + L::prof_bytes(sc.P));
  load_simp(s_simp, sim, sc);
  __syncthreads();
  const long gw = (long)blockIdx.x * warps + wib;
  const long nw = (long)gridDim.x * warps;
  int2* scr = scratch + gw * 2 * rowsCap;
  const int* meta = inputs + metaOffset;
  // Byte codes: residue offsets count bytes from the start of the buffer.
  const uint8_t* bytes = reinterpret_cast<const uint8_t*>(inputs);
  for (long g = gw; g < totalSlots; g += nw) {
    const long long tileBase = (long long)(g / maxBatches) * seqWordsPerTile * 4;
    const int alen = meta[4 * g + 0], aoff = meta[4 * g + 1];
    const int blen = meta[4 * g + 2], boff = meta[4 * g + 3];
    if (blen > rowsCap) {
      if (lane == 0) atomicCAS(&st->error, 0, ERR_SCRATCH);
      continue;
    }
    const long long a0[1] = {tileBase + aoff};
    const long long b0[1] = {tileBase + boff};
    const int al[1] = {alen}, bl[1] = {blen};
    Best fw[1], rv[1];
    bool ovf[1];
    align_pairs<T, K, 32>(sc, s_prof, s_simp, s_bring, bytes, a0, b0, al, bl, scr, rowsCap, fw, rv, ovf);
    if (lane == 0)
      write_result(sc, fw[0], rv[0], results, results + totalSlots, results + 2L * totalSlots, g);
  }
}

// The one-launch-per-batch kernel with s16x2 lanes: the same wire buffer,
// slot order and static stride as k_plain, but one warp aligns two
// consecutive comparison slots (2g, 2g + 1) in the halves of s16x2 lanes,
// whatever their lengths.  A slot whose score could have left int16 is
// redone by the same warp in s32 lanes, so the batch still takes one
// launch.  It isolates what the batched engine gains by sorting, binning
// and packing pairs from what it gains by the lane width.
template <int K>
__global__ void __launch_bounds__(128) k_plain16(SwConst sc, const int8_t* __restrict__ sim,
                                                 const int* __restrict__ inputs, long seqWordsPerTile,
                                                 long metaOffset, int maxBatches, int totalSlots,
                                                 int2* scratch, long rowsCap, int* results,
                                                 DevStatus* st) {
  using L = SmemLayout<Lane16, K, 32>;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warps = blockDim.x >> 5;
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* wbase = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.P);
  uint8_t* s_prof = wbase;  // the s32 redo uses the first half of it
  uint16_t* s_bring = reinterpret_cast<uint16_t*>(wbase + L::prof_bytes(sc.P));
  load_simp(s_simp, sim, sc);
  __syncthreads();
  const long gw = (long)blockIdx.x * warps + wib;
  const long nw = (long)gridDim.x * warps;
  int2* scr = scratch + gw * 2 * rowsCap;
  const int* meta = inputs + metaOffset;
  const uint8_t* bytes = reinterpret_cast<const uint8_t*>(inputs);
  for (long g0 = 2 * gw; g0 < totalSlots; g0 += 2 * nw) {
    long long a0[2], b0[2];
    int al[2], bl[2];
    bool tooLong = false;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long g = g0 + h;
      const bool have = g < totalSlots;
      const long long tileBase = have ? (long long)(g / maxBatches) * seqWordsPerTile * 4 : 0;
      al[h] = have ? meta[4 * g + 0] : 0;
      bl[h] = have ? meta[4 * g + 2] : 0;
      a0[h] = tileBase + (have ? meta[4 * g + 1] : 0);
      b0[h] = tileBase + (have ? meta[4 * g + 3] : 0);
      tooLong |= bl[h] > rowsCap;
    }
    if (tooLong) {  // warp-uniform: every lane read the same Meta words
      if (lane == 0) atomicCAS(&st->error, 0, ERR_SCRATCH);
      continue;
    }
    Best fw[2], rv[2];
    bool ovf[2];
    align_pairs<Lane16, K, 32>(sc, s_prof, s_simp, s_bring, bytes, a0, b0, al, bl, scr, rowsCap, fw, rv, ovf);
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      if (g0 + h >= totalSlots) break;
      if (ovf[h]) {  // uniform: the score is the 32-lane group's reduction
        const long long a1[1] = {a0[h]};
        const long long b1[1] = {b0[h]};
        const int al1[1] = {al[h]}, bl1[1] = {bl[h]};
        Best f1[1], r1[1];
        bool o1[1];
        align_pairs<LaneS32, K, 32>(sc, s_prof, s_simp, s_bring, bytes, a1, b1, al1, bl1, scr, rowsCap, f1, r1,
                                    o1);
        fw[h] = f1[0];
        rv[h] = r1[0];
      }
      if (lane == 0)
        write_result(sc, fw[h], rv[h], results, results + totalSlots, results + 2L * totalSlots, g0 + h);
    }
  }
}

// Exact per-thread kernel: one thread per pair, the recurrence written out
// cell by cell in int32 (codelet_batch_affine.cpp:65-115) with C and F rows
// in global scratch (2 * maxA int per thread).  Covers every scoring
// configuration.  A[j] = residue a0 + j * da, B[i] = residue b0 + i * db of
// `codes` (sc.bits per residue).
static __device__ void exact_pass(const uint8_t* codes, int bits, long long a0, int alen, int da, long long b0,
                                  int blen, int db, const int8_t* sim, int M, int gI, int gE, int* C, int* F,
                                  Best& out) {
  int s = 0, bi = 0, bj = 0;
  for (int j = 0; j < alen; ++j) {
    C[j] = 0;
    F[j] = 0;
  }
  for (int i = 0; i < blen; ++i) {
    const int bc = code_at(codes, b0 + (long long)i * db, bits);
    int e = gI, hl = 0, diag = 0;
    for (int j = 0; j < alen; ++j) {
      const int ac = code_at(codes, a0 + (long long)j * da, bits);
      e = max(hl + gI + gE, e + gE);
      const int f = max(C[j] + gI + gE, F[j] + gE);
      F[j] = f;
      int h = max(diag + (int)sim[ac * M + bc], e);
      h = max(max(h, f), 0);
      diag = C[j];
      C[j] = h;
      hl = h;
      if (h > s) {
        s = h;
        bi = i;
        bj = j;
      }
    }
  }
  out = Best{s, bi, bj};
}

// Pairs are checked with pair_state against n_codes and the stated maxima
// (maxA, maxB) before any code is read.
static __global__ void k_exact(SwConst sc, const int8_t* __restrict__ sim, const uint8_t* __restrict__ codes,
                        long long n_codes, const PairDesc* __restrict__ pairs, int n, int* cf_scratch, long maxA,
                        int maxB, int* score, int* arange, int* brange, DevStatus* st) {
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nt = (long)gridDim.x * blockDim.x;
  int* C = cf_scratch + tid * 2 * maxA;
  int* F = C + maxA;
  for (long p = tid; p < n; p += nt) {
    const PairDesc d = pairs[p];
    const int state = pair_state(d, n_codes, (int)maxA, maxB);
    report_pair(state, st);
    const int alen = state == PAIR_OK ? d.a_len : 0;
    const int blen = state == PAIR_OK ? d.b_len : 0;
    const long long a = state == PAIR_OK ? d.a_off : 0;
    const long long b = state == PAIR_OK ? d.b_off : 0;
    Best fw{0, 0, 0}, rv{0, 0, 0};
    if (alen > 0 && blen > 0 && alen <= maxA) {
      exact_pass(codes, sc.bits, a, alen, 1, b, blen, 1, sim, sc.M, sc.gI, sc.gE, C, F, fw);
      if (!sc.forwardOnly)
        exact_pass(codes, sc.bits, a + fw.j, fw.j + 1, -1, b + fw.i, fw.i + 1, -1, sim, sc.M, sc.gI, sc.gE, C, F,
                   rv);
    }
    write_result(sc, fw, rv, score, arange, brange, p);
  }
}

// -------------------------------------------------------------------------
// Cost-binned work list.  Every pair gets a key = class * NBUCKET + bucket,
// where the class picks the kernel (lane type, lanes per pair, columns per
// lane: |A| decides it) and the bucket orders by descending |B| on a
// log-linear scale; a counting sort over the keys yields the processing
// order: longest first inside each class (the long tail starts early) and
// neighbours of near-equal rows, which share a warp.  Empty pairs get their
// zero result here and are not listed.
// -------------------------------------------------------------------------
constexpr int NROWB = 256;    // row buckets (16 per power of two)
constexpr int NSTRIPB = 16;   // strip-count buckets
constexpr int NBUCKET = NROWB * NSTRIPB;
constexpr int NCLASS_MAX = 24;

// Log-linear bucket of |B| (16 sub-buckets per power of two): pairs that
// share a bucket differ by at most 1/16 in rows, so the groups of a warp
// finish their wavefronts together.
__device__ __forceinline__ int rows_bucket(int b) {
  if (b < 16) return b;
  const int lg = 31 - __clz(b);
  return min(NROWB - 1, (lg - 3) * 16 + ((b >> (lg - 4)) & 15));
}

struct BinParams {
  int nclass;
  int cls_s32;             // class index of the exact-32-bit kernel
  int cls_hi;              // class of pairs the diagonal bound sends to 32 bits:
                           // the hybrid class (or cls_s32 when it is off)
  int s16_max_len;         // min(|A|,|B|) above which s16x2 could overflow
  int s16_limit;           // scores above this need s32 lanes
  int lanes[NCLASS_MAX];   // lanes per group of each class
  int width[NCLASS_MAX];   // strip width (lanes * K) of each class
  float slot_ps[NCLASS_MAX];   // time per cell slot of a strip (autotuned)
  float strip_ps[NCLASS_MAX];  // fixed time per strip (autotuned)
  // Latency bound: one warp item of class c advances one step (row) every
  // step_ps[c] when the GPU is full, so a pair of `strips` strips takes
  // strips * (|B| + lanes) * step_ps[c].  A class is not chosen for a pair
  // whose item would take longer than lat_share * (modelled batch time =
  // cells of the batch * batch_ps_per_cell), when that batch time is at
  // least lat_min_ps: a few such items would end their launch alone.
  float step_ps[NCLASS_MAX];
  float batch_ps_per_cell;
  float lat_share;
  float lat_min_ps;
  int long_a;                  // |A| above which the widest class is used
  int widest;                  // that class
  int forced_class;        // >= 0: every s16x2 pair goes to this class
  int team_cls;            // strip-team class (-1: none in this batch)
  int team_warps;          // warps per team
  int n_s16_classes;
  int max_a, max_b;        // stated maxima (violations set ERR_LENGTH)
  long long n_codes;       // residues in the code array (pairs past it set ERR_RANGE)
  int bits;                // bits per residue of the code array (code_at)
  int M;                   // alphabet size of `sim`
  int force_s32;           // 1: every pair goes to the s32 class
  // Per-thread class (k_thread): one thread per two pairs, so a pair's time
  // is long.  A pair may use it only when |B| <= thr_max_rows and its cells
  // stay below thr_cap_scale * (cells of the whole batch): that bounds its
  // latency to a fraction of the batch's time (thr_cap_scale = fraction /
  // pair slots the class keeps resident).
  // Concurrent class launches (k_bin_scan turns modelled costs into block
  // shares): full-occupancy grid and strip scratch (int2) per block of
  // each class, and the scratch available.
  unsigned int enabled;    // bit c: class c may be chosen by cost (and is launched)
  int concurrent;          // 0 sequential, 1 shares, 2 two alternating streams
  int slot_of[NCLASS_MAX + 1];  // mode 2: scratch region (0 / 1) of each class
  long long region;             // mode 2: int2 per region
  int grid[NCLASS_MAX + 1];
  long long scr_per_block[NCLASS_MAX + 1];
  long long scr_cap;
  int thr_cls;             // class index
  int thr_on;              // 0: the class is never chosen (unless forced)
  int thr_k;               // columns per strip
  int thr_max_rows;
  float thr_cap_scale;
  const unsigned long long* total_cells;  // written by k_bin_total
};

// Buckets of the per-thread class: exact strip counts up to 24 (then one
// bucket), rows log-linear with 16 sub-buckets per octave (< 144 for rows
// up to 2048); both descending.
constexpr int THR_NSB = 25;
constexpr int THR_NRB = 144;
static_assert(THR_NSB * THR_NRB <= NBUCKET, "per-thread buckets");

// Best ungapped score along the main diagonal (a lower bound of the local
// alignment score): pairs that surely pass the s16 limit go to the hybrid
// (or s32) class instead of giving up half way in s16x2.  One warp per
// pair: lane l takes the l-th of 32 consecutive segments of the diagonal
// and summarises it as {sum, best prefix, best suffix, best run} (all >= 0
// but the sum); an ordered tree of shuffles joins the summaries, the best
// run of the whole diagonal ending in lane 0 (the maximum-subarray score
// that max(run + s, 0) computes sequentially).
struct DiagRun {
  int sum, pre, suf, best;
};

__device__ __forceinline__ DiagRun join_runs(const DiagRun& l, const DiagRun& r) {
  return DiagRun{l.sum + r.sum, max(l.pre, l.sum + r.pre), max(r.suf, r.sum + l.suf),
                 max(max(l.best, r.best), l.suf + r.pre)};
}

static __device__ int warp_diagonal_bound(const uint8_t* codes, int bits, long long a, long long b, int n,
                                          const int8_t* sim, int M) {
  const int lane = threadIdx.x & 31;
  const int seg = (n + 31) / 32;
  const int k0 = min(n, lane * seg), k1 = min(n, k0 + seg);
  DiagRun r{0, 0, 0, 0};
  int run = 0;
  auto take = [&](int s) {
    r.sum += s;
    r.pre = max(r.pre, r.sum);
    run = max(run + s, 0);
    r.best = max(r.best, run);
  };
  // A code outside the alphabet (no row of the matrix) counts 0 here.
  auto score = [&](int x, int y) { return (x < M && y < M) ? (int)sim[x * M + y] : 0; };
  if (k0 < k1) {
    if (bits == 8) {
      for (int k = k0; k < k1; ++k) take(score(codes[a + k], codes[b + k]));
    } else {
      PackedStream sa(codes, a + k0, bits), sb(codes, b + k0, bits);
      for (int k = k0; k < k1; ++k) {
        const int x = sa.next(), y = sb.next();
        take(score(x, y));
      }
    }
  }
  r.suf = run;  // best sum of a suffix (empty allowed)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    DiagRun o;
    o.sum = __shfl_down_sync(FULL, r.sum, off);
    o.pre = __shfl_down_sync(FULL, r.pre, off);
    o.suf = __shfl_down_sync(FULL, r.suf, off);
    o.best = __shfl_down_sync(FULL, r.best, off);
    if ((lane & (2 * off - 1)) == 0 && lane + off < 32) r = join_runs(r, o);
  }
  return __shfl_sync(FULL, r.best, 0);
}

// Steps a team warp starts behind the warp before it: it reads boundary
// rows two blocks of 32 ahead, which that warp publishes a block later.
constexpr float kTeamLagSteps = 96.f;
// Share of the batch's modelled time above which a pair's one-warp latency
// sends it to a strip team (measured on B200: a 500,000-pair heavy-tailed
// protein batch, whose 8,000-residue pairs take about a third of its time
// on one warp, ran 10 % slower with them in teams; batches of a few hundred
// long pairs ran 3.7-5.6 times faster).
constexpr float kTeamLatencyShare = 0.5f;

// Class of a pair: the kernel with the lowest modelled time
//   strips * ((|B| + lanes) * width * slot_ps + strip_ps)
// where strips * width covers |A|, |B| + lanes counts the fill and drain of
// each strip's wavefront, and slot_ps / strip_ps are the per-class rates
// the autotuner measured.  Key = class, then strip count (descending), then
// rows (descending).
__device__ __forceinline__ int pair_key(const BinParams& bp, int alen, int blen, bool s32, float thr_cap,
                                        float* cost_out = nullptr) {
  int cls;
  if (bp.force_s32) {
    cls = bp.cls_s32;
  } else if (s32) {
    cls = bp.cls_hi;
  } else if (bp.forced_class >= 0) {
    cls = bp.forced_class;
  } else {
    const float batch_ps = bp.total_cells ? (float)(*bp.total_cells) * bp.batch_ps_per_cell : 0.f;
    float bestLat = -1.f;  // one-warp latency of the class picked below
    if (alen > bp.long_a) {
      // Very long pairs are few and each keeps one warp busy for long: their
      // latency, not throughput, sets the end of the launch, and the widest
      // strips finish a pair in the fewest steps.
      cls = bp.widest;
      bestLat = (float)((alen + bp.width[cls] - 1) / bp.width[cls]) * (float)(blen + bp.lanes[cls]) *
                bp.step_ps[cls];
    } else {
      cls = 0;
      float bestCost = -1.f;
      int latCls = 0;
      const bool thr_ok = bp.thr_on && blen <= bp.thr_max_rows && (float)alen * (float)blen <= thr_cap;
      const float lat_cap = batch_ps >= bp.lat_min_ps ? bp.lat_share * batch_ps : 3.0e38f;
      for (int c = 0; c < bp.n_s16_classes; ++c) {
        if (!((bp.enabled >> c) & 1u)) continue;
        if (c == bp.thr_cls && !thr_ok) continue;
        const int strips = (alen + bp.width[c] - 1) / bp.width[c];
        const float lat = (float)strips * (float)(blen + bp.lanes[c]) * bp.step_ps[c];
        if (bestLat < 0.f || lat < bestLat) {
          bestLat = lat;
          latCls = c;
        }
        if (lat > lat_cap) continue;
        const float cost =
            (float)strips * ((float)(blen + bp.lanes[c]) * (float)bp.width[c] * bp.slot_ps[c] + bp.strip_ps[c]);
        if (bestCost < 0.f || cost < bestCost) {
          bestCost = cost;
          cls = c;
        }
      }
      if (bestCost < 0.f) {
        cls = latCls;  // every class is too slow: the fastest
      } else {
        bestLat = 0.f;  // a class keeps the pair under the latency cap
      }
    }
    // A strip team, when even the fastest warp would take a large share of
    // the whole batch's modelled time (kTeamLatencyShare: below it the
    // other pairs' work hides the pair, and a team's fill and idle warps
    // only cost throughput) and the team finishes the pair sooner.  Its
    // warps take the strips round robin, each starting about kTeamLagSteps
    // behind the warp before it.
    const int tc = bp.team_cls;
    if (tc >= 0 && bestLat > kTeamLatencyShare * batch_ps) {
      const int strips = (alen + bp.width[tc] - 1) / bp.width[tc];
      if (strips >= 2) {
        const int rounds = (strips + bp.team_warps - 1) / bp.team_warps;
        const float lat = ((float)rounds * (float)(blen + bp.lanes[tc]) +
                           kTeamLagSteps * (float)(min(strips, bp.team_warps) - 1)) *
                          bp.step_ps[tc];
        if (lat < bestLat) cls = tc;
      }
    }
  }
  const int strips = (alen + bp.width[cls] - 1) / bp.width[cls];
  if (cost_out)
    *cost_out = (float)strips *
                ((float)(blen + bp.lanes[cls]) * (float)bp.width[cls] * bp.slot_ps[cls] + bp.strip_ps[cls]);
  if (cls == bp.thr_cls) {
    const int sb = THR_NSB - 1 - min(strips - 1, THR_NSB - 1);
    return cls * NBUCKET + sb * THR_NRB + (THR_NRB - 1 - min(rows_bucket(blen), THR_NRB - 1));
  }
  const int sb = NSTRIPB - 1 - min(strips - 1, NSTRIPB - 1);
  return cls * NBUCKET + sb * NROWB + (NROWB - 1 - rows_bucket(blen));
}

// Latency cap of the per-thread class for this batch (cells per pair).
__device__ __forceinline__ float thread_cap(const BinParams& bp) {
  return (bp.thr_on && bp.total_cells) ? (float)(*bp.total_cells) * bp.thr_cap_scale : 0.f;
}

// Sum of |A| * |B| over the pairs the pipeline will align (the batch size
// the per-thread class's latency cap is measured against).
static __global__ void k_bin_total(BinParams bp, const PairDesc* __restrict__ pairs, int n,
                                   unsigned long long* total) {
  unsigned long long local = 0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const PairDesc d = pairs[p];
    if (pair_state(d, bp.n_codes, bp.max_a, bp.max_b) != PAIR_OK) continue;
    local += (unsigned long long)d.a_len * (unsigned long long)d.b_len;
  }
  for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(FULL, local, off);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(total, local);
}

// A pair whose diagonal bound decides its class: both sequences longer than
// the longest pair that cannot pass the s16 limit.
__device__ __forceinline__ bool bound_candidate(const BinParams& bp, const PairDesc& d) {
  return !bp.force_s32 && min(d.a_len, d.b_len) > bp.s16_max_len &&
         pair_state(d, bp.n_codes, bp.max_a, bp.max_b) == PAIR_OK;
}

// s32_flag of every candidate pair (k_bin_count reads it): warps take 32
// pairs at a time and compute the diagonal bound of each candidate among
// them together (warp_diagonal_bound).  blockDim.x is a multiple of 32.
static __global__ void k_bin_bound(BinParams bp, const uint8_t* __restrict__ codes,
                                   const int8_t* __restrict__ sim, const PairDesc* __restrict__ pairs, int n,
                                   uint8_t* s32_flag) {
  __shared__ int8_t s_sim[32 * 32];
  const bool smemSim = bp.M <= 32;
  if (smemSim)
    for (int k = threadIdx.x; k < bp.M * bp.M; k += blockDim.x) s_sim[k] = sim[k];
  __syncthreads();
  const int8_t* simT = smemSim ? s_sim : sim;
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x / 32);
  for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32 * 32; base < n; base += warps * 32) {
    const long p = base + lane;
    const bool cand = p < n && bound_candidate(bp, pairs[p]);
    unsigned m = __ballot_sync(FULL, cand);
    while (m) {
      const long q = base + __ffs(m) - 1;
      m &= m - 1;
      const PairDesc d = pairs[q];
      const int bound =
          warp_diagonal_bound(codes, bp.bits, d.a_off, d.b_off, min(d.a_len, d.b_len), simT, bp.M);
      if (lane == 0) s32_flag[q] = bound > bp.s16_limit ? 1 : 0;
    }
  }
}

static __global__ void k_bin_count(BinParams bp, const uint8_t* __restrict__ codes, const int8_t* __restrict__ sim,
                            const PairDesc* __restrict__ pairs, int n, int* hist, uint8_t* s32_flag,
                            unsigned long long* class_cells, unsigned long long* class_cost, DevStatus* st,
                            int* score, int* arange, int* brange) {
  // Per-class sums of the block, added to the global ones once at the end
  // (a batch has a handful of classes: one global address per class would
  // take every pair's atomic).
  __shared__ unsigned long long s_cells[NCLASS_MAX + 1], s_cost[NCLASS_MAX + 1];
  for (int k = threadIdx.x; k <= NCLASS_MAX; k += blockDim.x) {
    s_cells[k] = 0;
    s_cost[k] = 0;
  }
  __syncthreads();
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const PairDesc d = pairs[p];
    const int state = pair_state(d, bp.n_codes, bp.max_a, bp.max_b);
    if (state != PAIR_OK) {
      // Empty, too long or outside the code array: zero result, not listed.
      report_pair(state, st);
      score[p] = 0;
      arange[p] = 0;
      brange[p] = 0;
      continue;
    }
    // Candidates (both sequences longer than s16_max_len) got their flag
    // from k_bin_bound.
    bool s32 = false;
    if (bound_candidate(bp, d)) s32 = s32_flag[p] != 0;
    s32_flag[p] = s32 ? 1 : 0;
    float cost = 0.f;
    const int key = pair_key(bp, d.a_len, d.b_len, s32, thread_cap(bp), &cost);
    // One histogram update per distinct key among the warp's lanes.
    const unsigned same = __match_any_sync(__activemask(), key);
    if ((int)(threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&hist[key], __popc(same));
    atomicAdd(&s_cells[key / NBUCKET], (unsigned long long)d.a_len * (unsigned long long)d.b_len);
    atomicAdd(&s_cost[key / NBUCKET], (unsigned long long)fmaxf(cost, 1.f));
  }
  __syncthreads();
  for (int k = threadIdx.x; k < bp.nclass; k += blockDim.x) {
    if (s_cells[k]) atomicAdd(&class_cells[k], s_cells[k]);
    if (s_cost[k]) atomicAdd(&class_cost[k], s_cost[k]);
  }
}

__device__ __forceinline__ int run_total(const int* hist, const int* offs, int nkeys) {
  return offs[nkeys - 1] + hist[nkeys - 1];
}

// Single block (blockDim.x a multiple of 32): exclusive scan of the
// histogram into `offs`, and per class the {start, count} range consumed by
// k_batched.  The keys go tile by tile (blockDim.x keys, coalesced, kTiles
// tiles of loads in flight), each tile scanned across the block and offset
// by the running total of the tiles before.
static __global__ void k_bin_scan(BinParams bp, int nkeys, const int* hist, int* offs, int* class_range,
                                  const unsigned long long* class_cost, ClassAllot* allot, DevStatus* st) {
  constexpr int kTiles = 8;
  __shared__ int s_warp[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  int carry = 0;
  for (int base = 0; base < nkeys; base += kTiles * blockDim.x) {
    int v[kTiles];
#pragma unroll
    for (int j = 0; j < kTiles; ++j) {
      const int k = base + j * blockDim.x + tid;
      v[j] = k < nkeys ? hist[k] : 0;
    }
#pragma unroll
    for (int j = 0; j < kTiles; ++j) {
      int x = v[j];  // inclusive prefix within the warp
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(FULL, x, off);
        if (lane >= off) x += y;
      }
      if (lane == 31) s_warp[wid] = x;
      __syncthreads();
      if (wid == 0) {
        int w = lane < nw ? s_warp[lane] : 0;  // inclusive prefix of the warp totals
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(FULL, w, off);
          if (lane >= off) w += y;
        }
        if (lane < nw) s_warp[lane] = w;
      }
      __syncthreads();
      const int k = base + j * blockDim.x + tid;
      if (k < nkeys) offs[k] = carry + (wid > 0 ? s_warp[wid - 1] : 0) + x - v[j];
      carry += s_warp[nw - 1];
      __syncthreads();  // s_warp is rewritten by the next tile
    }
  }
  if (tid < nkeys / NBUCKET) {
    const int c = tid;
    class_range[2 * c] = offs[c * NBUCKET];
    class_range[2 * c + 1] = ((c + 1) * NBUCKET < nkeys ? offs[(c + 1) * NBUCKET] : run_total(hist, offs, nkeys)) -
                             offs[c * NBUCKET];
  }
  __syncthreads();
  if (tid == 0) {
    // Block shares: sequential launches each take the whole GPU; concurrent
    // ones split it by modelled cost, scratch regions laid end to end.
    const int nc = nkeys / NBUCKET;
    double total = 0.0;
    for (int c = 0; c < nc; ++c)
      if (class_range[2 * c + 1] > 0) total += (double)class_cost[c];
    long long base = 0;
    for (int c = 0; c < nc; ++c) {
      int blocks = 0;
      if (class_range[2 * c + 1] > 0) {
        blocks = bp.grid[c];
        if (bp.concurrent == 1 && total > 0.0)
          blocks = min(bp.grid[c], max(1, (int)ceil((double)class_cost[c] / total * bp.grid[c])));
      }
      const long long start = bp.concurrent == 1 ? base : bp.concurrent == 2 ? bp.slot_of[c] * bp.region : 0;
      const long long need = (long long)blocks * bp.scr_per_block[c];
      if (start + need > bp.scr_cap) {
        // Never reached when the host sized the scratch for these shares.
        blocks = bp.scr_per_block[c] > 0 ? (int)max(0ll, (bp.scr_cap - start) / bp.scr_per_block[c]) : blocks;
        if (blocks == 0 && class_range[2 * c + 1] > 0) atomicCAS(&st->error, 0, ERR_SCRATCH);
      }
      allot[c].blocks = blocks;
      allot[c].base = start;
      if (bp.concurrent == 1) base += (long long)blocks * bp.scr_per_block[c];
    }
    // The s32 rerun runs alone after every class: the whole GPU, base 0.
    allot[nc].blocks = bp.grid[bp.cls_s32];
    allot[nc].base = 0;
  }
}

static __global__ void k_bin_scatter(BinParams bp, const PairDesc* __restrict__ pairs, int n,
                              const uint8_t* __restrict__ s32_flag, int* offs, int* list) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const PairDesc d = pairs[p];
    if (pair_state(d, bp.n_codes, bp.max_a, bp.max_b) != PAIR_OK) continue;
    const int key = pair_key(bp, d.a_len, d.b_len, s32_flag[p] != 0, thread_cap(bp));
    // One atomic per distinct key among the warp's lanes; each lane takes
    // the slot of its rank in the group.
    const unsigned act = __activemask();
    const unsigned same = __match_any_sync(act, key);
    const int lane = (int)(threadIdx.x & 31), leader = __ffs(same) - 1;
    int pos0 = 0;
    if (lane == leader) pos0 = atomicAdd(&offs[key], __popc(same));
    pos0 = __shfl_sync(act, pos0, leader);
    list[pos0 + __popc(same & ((1u << lane) - 1u))] = (int)p;
  }
}

// Synthetic calibration batch for the autotuner: n pairs of |A| = alen,
// |B| = blen; A uniform over `letters`, B = A with 1 in 8 residues
// substituted, then random letters past |A|.
static __global__ void k_synth_pairs(uint8_t* codes, PairDesc* pairs, int n, int alen, int blen,
                                     const uint8_t* __restrict__ letters, int nletters, uint32_t seed) {
  const long per = (long)alen + blen;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < (long)n * per;
       k += (long)gridDim.x * blockDim.x) {
    const long p = k / per, i = k % per;
    auto hash = [&](long x) {
      uint32_t h = (uint32_t)x * 0x9E3779B1u ^ seed;
      h ^= h >> 15;
      h *= 0x85EBCA77u;
      h ^= h >> 13;
      h *= 0xC2B2AE3Du;
      return h ^ (h >> 16);
    };
    uint8_t v;
    if (i < alen) {
      v = letters[hash(p * 131071 + i) % nletters];
    } else {
      const long j = i - alen;
      const uint32_t r = hash(p * 524287 + j + 7);
      v = (j < alen && (r & 7)) ? letters[hash(p * 131071 + j) % nletters] : letters[(r >> 3) % nletters];
    }
    codes[k] = v;
    if (i == 0) pairs[p] = PairDesc{p * per, p * per + alen, alen, blen};
  }
}

// Validates the Meta section of a device-resident wire buffer: lengths and
// offsets must stay inside their tile.  info = {maxA, maxB, bad slots}.
static __global__ void k_wire_check(const int* __restrict__ inputs, long metaOffset, long tileBytes,
                             int totalSlots, int* info, unsigned long long* cells) {
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < totalSlots;
       g += (long)gridDim.x * blockDim.x) {
    const int* m = inputs + metaOffset + 4 * g;
    const int al = m[0], ao = m[1], bl = m[2], bo = m[3];
    if (al == 0 || bl == 0) continue;
    if (al < 0 || bl < 0 || ao < 0 || bo < 0 || (long)ao + al > tileBytes || (long)bo + bl > tileBytes) {
      atomicAdd(&info[2], 1);
      continue;
    }
    atomicMax(&info[0], al);
    atomicMax(&info[1], bl);
    atomicAdd(cells, (unsigned long long)al * (unsigned long long)bl);
  }
}

// Wire buffer -> pair list: slot g of tile g / maxBatches, offsets made
// absolute in bytes from the start of the input buffer.
static __global__ void k_wire_to_pairs(const int* __restrict__ inputs, long seqWordsPerTile, long metaOffset,
                                int maxBatches, int totalSlots, PairDesc* pairs) {
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < totalSlots;
       g += (long)gridDim.x * blockDim.x) {
    const int* m = inputs + metaOffset + 4 * g;
    const long base = (g / maxBatches) * seqWordsPerTile * 4;
    pairs[g] = PairDesc{base + m[1], base + m[3], m[0], m[2]};
  }
}

}  // namespace ipuma_dev
