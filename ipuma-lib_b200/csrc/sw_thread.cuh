// sw_thread.cuh -- the per-thread kernel class k_thread<K>: one thread
// aligns two pairs in s16x2 halves (pair P low, pair Q high) over the whole
// matrix, column strip by column strip, with no communication between
// threads.  It reads one byte per residue (the engine never launches it on
// packed codes).
//
// Same recurrence, frames and tie-break as the wavefront kernels
// (sw_device.cuh, after src/codelets/codelet_batch_affine.cpp:65-85): per
// cell F̂ = viaddmax(F̂, gE, Hup), Y = viaddmax_relu(Hdiag, sub, F̂ + gIgE),
// Ê = viaddmax(Ê, gE', Yleft), H = viaddmax(Ê, gIgE, Y).  A thread owns K
// consecutive columns of a strip and walks all rows of the pair through
// them; the (Y, Ê) of the strip's last column of every row is the next
// strip's left boundary.  The boundary column lives in global scratch laid
// out row-major over the launch's threads (row r of thread g at
// r * nthreads + g), so every row's loads and stores are coalesced across
// the warp, and it is updated in place: row r of strip s + 1 reads what
// row r of strip s wrote and overwrites it.
//
// Compared with the wavefront kernels this removes the per-step shuffles,
// the lane-0 boundary selection, the fill and drain steps of every strip
// and most column padding (a strip is K columns, not lanes * K), at the
// price of one global load and store of 8 bytes per row and strip and a
// longer time per pair; the class is therefore only used for pairs that
// are small relative to the batch (the binning pre-pass bounds their size).
//
// Query profile: per thread and strip, prof[x][h] = K int8 values
// sim[A_h[col]][x] for the thread's K columns (SUB_PAD past |A| and for the
// padding letter x = M).  In shared memory the entries of the 32 threads of
// a warp are interleaved (row x, pair h, thread t at ((x * 2 + h) * 32 + t)
// * K bytes), so the 16-byte profile loads of a warp are free of bank
// conflicts whatever letters its threads read.
#pragma once
#include "sw_kernels.cuh"

namespace ipuma_dev {

template <int K>
struct ThreadSmem {
  static_assert(K == 8 || K == 16, "k_thread columns per strip");
  __host__ __device__ static int simp_bytes(int M) { return ((M * (M + 1)) + 15) & ~15; }
  __host__ __device__ static int warp_bytes(int M) { return (M + 1) * 2 * 32 * K; }
  __host__ __device__ static int total(int M, int warps) { return simp_bytes(M) + warps * warp_bytes(M); }
};

// Builds this thread's profile slice for the strip starting at col0.
template <int K>
__device__ __forceinline__ void thread_profile(uint8_t* s_warp, const int8_t* s_simp, int M,
                                               const PassSeq (&ps)[2], int col0, int t) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int acode[K];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      const int col = col0 + c;
      acode[c] = (col < ps[h].alen) ? (int)ps[h].base[ps[h].a + (long long)col * ps[h].da] * (M + 1) : -1;
    }
    uint8_t* dst = s_warp + (h * 32 + t) * K;
    for (int x = 0; x <= M; ++x) {
      uint32_t w[K / 4];
#pragma unroll
      for (int q = 0; q < K / 4; ++q) {
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int a = acode[4 * q + b];
          const int v = (a >= 0) ? (int)s_simp[a + x] : SUB_PAD;
          word |= ((uint32_t)(uint8_t)(int8_t)v) << (8 * b);
        }
        w[q] = word;
      }
      uint8_t* row = dst + x * (2 * 32 * K);
      if constexpr (K == 16) {
        *reinterpret_cast<uint4*>(row) = make_uint4(w[0], w[1], w[2], w[3]);
      } else {
        *reinterpret_cast<uint2*>(row) = make_uint2(w[0], w[1]);
      }
    }
  }
}

// One pass (forward or reverse) of one thread over its two pairs.
//   s_warp : the warp's profile area ((M + 1) * 2 * 32 * K bytes)
//   scr    : this thread's boundary column, row stride `stride` (int2)
//   out    : best cell per pair in pass coordinates
//   over   : set per pair when its best passed sc.s16Limit (the pair is
//            rerun in s32 lanes; its values past that point are not used)
template <int K>
__device__ __forceinline__ void thread_pass(const SwConst& sc, uint8_t* s_warp, const int8_t* s_simp,
                                            const PassSeq (&ps)[2], int2* scr, long stride, int t,
                                            Best (&out)[2], bool (&over)[2]) {
  using T = LaneS16x2;
  using V = uint32_t;
  const int M = sc.M;
  const int rows = max(ps[0].blen, ps[1].blen);
  const int nstrips = (max(ps[0].alen, ps[1].alen) + K - 1) / K;
  const V vgE = T::splat(sc.gE);
  const V vgEp = T::splat(max(sc.gE, sc.gIgE));
  const V vgIgE = T::splat(sc.gIgE);
  const V vE0 = T::splat(-max(sc.gE, sc.gIgE));
  const V vF0 = T::splat(-sc.gIgE);
  const V vZero = T::splat(0);
  const uint8_t* prof0 = s_warp + t * K;
  const uint8_t* prof1 = s_warp + (32 + t) * K;
  constexpr int RSTRIDE = 2 * 32 * K;  // bytes between letters of the profile
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    out[h] = Best{0, 0, 0};
    over[h] = false;
  }
  if (rows <= 0) return;
  const int lim = sc.s16Limit;

  // B letters stream through aligned 32-bit words (a word that holds at
  // least one byte of the sequence lies in the sequence's page, so no load
  // leaves valid memory).  Row block j (rows 4j .. 4j+3) of pair h is
  //   forward: funnel(U_j, U_{j+1}) with U_k = word k from b & ~3
  //   reverse: byte-reversed funnel(U_{j+1}, U_j) with U_k = word 1 - k
  //            from (b - 3) & ~3
  // shifted by the sequence's misalignment; bytes past |B| become M.
  const uint32_t* wbase[2];
  int wstep[2], wshift[2], wfirst[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uintptr_t bp = (uintptr_t)(ps[h].base + ps[h].b);
    const uintptr_t p = (ps[h].db > 0) ? bp : bp - 3;
    wshift[h] = 8 * (int)(p & 3);
    wbase[h] = reinterpret_cast<const uint32_t*>(p & ~(uintptr_t)3) + (ps[h].db > 0 ? 0 : 1);
    wstep[h] = ps[h].db > 0 ? 1 : -1;
    // Row of the first byte of U_k is 4k - shift/8 (forward) or
    // 4k - 4 + shift/8 (reverse); U_k holds a sequence byte iff that row
    // is below |B| and its last row is >= 0.
    wfirst[h] = ps[h].db > 0 ? -(int)(p & 3) : (int)(p & 3) - 4;
  }
  const uint32_t padw = (uint32_t)M * 0x01010101u;
  auto word = [&](int h, int k) -> uint32_t {
    const int r0 = 4 * k + wfirst[h];
    return (r0 < ps[h].blen && r0 + 3 >= 0) ? __ldg(wbase[h] + (long)k * wstep[h]) : 0u;
  };
  // Letters of rows 4j .. 4j+3 of pair h from U_j (u0) and U_{j+1} (u1).
  auto block_letters = [&](int h, int j, uint32_t u0, uint32_t u1) -> uint32_t {
    uint32_t v = ps[h].db > 0 ? __funnelshift_r(u0, u1, wshift[h]) : prmt(__funnelshift_r(u1, u0, wshift[h]), 0u, 0x0123u);
    const int valid = ps[h].blen - 4 * j;
    if (valid < 4) {
      const uint32_t keep = valid <= 0 ? 0u : (0xffffffffu >> (32 - 8 * valid));
      v = (v & keep) | (padw & ~keep);
    }
    return v;
  };

  for (int strip = 0; strip < nstrips; ++strip) {
    const int col0 = strip * K;
    const bool hasIn = strip > 0;
    const bool hasOut = strip + 1 < nstrips;
    thread_profile<K>(s_warp, s_simp, M, ps, col0, t);

    V H[K], Fh[K], snap[K];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      H[c] = vZero;
      Fh[c] = vF0;
      snap[c] = vZero;
    }
    V best = vZero, diagIn = vZero;
    uint32_t brow = 0;

    auto row = [&](int i, uint32_t lt, int2 bnd, int2* out) {
      uint32_t wp[K / 4], wq[K / 4];
      load_profile_row<K>(wp, prof0 + prmt(lt, 0u, 0x4440u) * RSTRIDE);
      load_profile_row<K>(wq, prof1 + prmt(lt, 0u, 0x4441u) * RSTRIDE);
      V yl = (V)bnd.x;
      V e = (V)bnd.y;
      V diag = diagIn;
      diagIn = T::addmax(e, vgIgE, yl);  // H of the boundary cell of row i
#pragma unroll
      for (int c = 0; c < K; ++c) {
        V sb;
        switch (c & 3) {
          case 0: sb = T::template sub<0>(wp[c >> 2], wq[c >> 2]); break;
          case 1: sb = T::template sub<1>(wp[c >> 2], wq[c >> 2]); break;
          case 2: sb = T::template sub<2>(wp[c >> 2], wq[c >> 2]); break;
          default: sb = T::template sub<3>(wp[c >> 2], wq[c >> 2]); break;
        }
        const V f = T::addmax(Fh[c], vgE, H[c]);                 // F̂
        const V y = T::addmax_relu(diag, sb, T::add(f, vgIgE));  // Y
        e = T::addmax(e, vgEp, yl);                              // Ê
        const V hv = T::addmax(e, vgIgE, y);                     // H
        diag = H[c];
        H[c] = hv;
        Fh[c] = f;
        yl = y;
      }
      if (hasOut) *out = make_int2((int)yl, (int)e);
      V m8[K / 2];
#pragma unroll
      for (int c = 0; c < K / 2; ++c) m8[c] = T::max2(H[2 * c], H[2 * c + 1]);
#pragma unroll
      for (int w = 1; w < K / 2; w *= 2)
#pragma unroll
        for (int c = 0; c + w < K / 2; c += 2 * w) m8[c] = T::max2(m8[c], m8[c + w]);
      const V rm = m8[0];
      const uint32_t keep = keep_mask(T{}, rm, best);
      best = T::max2(best, rm);
      if (keep != 0xffffffffu) {
        const uint32_t ipk = (uint32_t)i * 0x00010001u;
        brow = (brow & keep) | (ipk & ~keep);
#pragma unroll
        for (int c = 0; c < K; ++c) snap[c] = (snap[c] & keep) | (H[c] & ~keep);
      }
    };

    // Rows in blocks of four; the letter words and boundary values of the
    // next block are loaded while the current one computes.
    const int2 bnd0 = make_int2((int)vZero, (int)vE0);
    uint32_t ua[2], ub[2], uc[2];  // U_j, U_{j+1}, U_{j+2} per pair
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      ua[h] = word(h, 0);
      ub[h] = word(h, 1);
    }
    int2 bc[4], bn[4];
    const int2* rin = scr;
#pragma unroll
    for (int k = 0; k < 4; ++k) bc[k] = (hasIn && k < rows) ? rin[k * stride] : bnd0;
    int2* rout = scr;
    for (int i0 = 0, j = 0; i0 < rows; i0 += 4, ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) uc[h] = word(h, j + 2);
      rin += 4 * stride;
#pragma unroll
      for (int k = 0; k < 4; ++k) bn[k] = (hasIn && i0 + 4 + k < rows) ? rin[k * stride] : bnd0;
      const uint32_t LP = block_letters(0, j, ua[0], ub[0]);
      const uint32_t LQ = block_letters(1, j, ua[1], ub[1]);
      if (i0 + 4 <= rows) {
#pragma unroll
        for (int k = 0; k < 4; ++k) row(i0 + k, prmt(LP, LQ, (uint32_t)(k | ((k + 4) << 4))), bc[k], rout + k * stride);
      } else {
#pragma unroll 1
        for (int k = 0; k < rows - i0; ++k) {
          // tail block: pick entry k without dynamic register indexing
          int2 b = bc[0];
          if (k == 1) b = bc[1];
          if (k == 2) b = bc[2];
          if (k == 3) b = bc[3];
          row(i0 + k, prmt(LP, LQ, (uint32_t)(k | ((k + 4) << 4))), b, rout + k * stride);
        }
      }
      rout += 4 * stride;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        ua[h] = ub[h];
        ub[h] = uc[h];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) bc[k] = bn[k];
    }

    // Strip result per pair: first column of the snapshot holding the best.
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int bg = T::half(best, h);
      if (bg > lim) over[h] = true;
      int jj = 0;
#pragma unroll
      for (int c = K - 1; c >= 0; --c)
        if (T::half(snap[c], h) == bg) jj = c;
      const int ii = (int)((brow >> (16 * h)) & 0xffffu);
      if (bg > 0 && better(bg, ii, col0 + jj, out[h].s, out[h].i, out[h].j)) out[h] = Best{bg, ii, col0 + jj};
    }
  }
}

// Persistent per-thread kernel over a cost-ordered work list: a warp takes
// items of 64 consecutive list entries, thread t aligning entries 2t and
// 2t + 1.  Pairs whose score passed the s16 limit go to the overflow list
// for the s32 rerun (no reverse pass here).
template <int K>
__global__ void __launch_bounds__(128, 3) k_thread(SwConst sc, const int8_t* __restrict__ sim,
                                                const uint8_t* __restrict__ codes,
                                                const PairDesc* __restrict__ pairs,
                                                const int* __restrict__ list,
                                                const int* __restrict__ range, int* queue_head,
                                                int2* scratch, long rowsCap, int* score, int* arange,
                                                int* brange, int* overflow_list,
                                                unsigned long long* rerun_cells, DevStatus* st,
                                                const ClassAllot* __restrict__ allot) {
  if ((int)blockIdx.x >= allot->blocks) return;  // outside this launch's share
  scratch += allot->base;
  using L = ThreadSmem<K>;
  extern __shared__ __align__(16) uint8_t smem[];
  const int wib = threadIdx.x >> 5;
  const int t = threadIdx.x & 31;
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* s_warp = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.M);
  load_simp(s_simp, sim, sc);
  __syncthreads();

  const int n = range[1];
  list += range[0];
  const int items = (n + 63) / 64;
  const long stride = (long)allot->blocks * blockDim.x;
  int2* scr = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
  while (true) {
    int item = 0;
    if (t == 0) item = atomicAdd(queue_head, 1);
    item = __shfl_sync(FULL, item, 0);
    if (item >= items) break;
    int pid[2];
    PassSeq ps[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = item * 64 + 2 * t + h;
      pid[h] = (k < n) ? list[k] : -1;
      const PairDesc d = (pid[h] >= 0) ? pairs[pid[h]] : PairDesc{0, 0, 0, 0};
      const bool empty = d.a_len <= 0 || d.b_len <= 0;
      ps[h] = PassSeq{codes, d.a_off, d.b_off, empty ? 0 : d.a_len, empty ? 0 : d.b_len, 1, 1};
    }
    // Only a thread with more than one strip touches the boundary scratch,
    // for all of its rows.
    if (max(ps[0].alen, ps[1].alen) > K && max(ps[0].blen, ps[1].blen) > rowsCap) {
      // The host sizes the scratch for the longest B; report, never trap.
      atomicCAS(&st->error, 0, ERR_SCRATCH);
      continue;
    }
    Best fw[2], rv[2];
    bool over[2];
    thread_pass<K>(sc, s_warp, s_simp, ps, scr, stride, t, fw, over);
    rv[0] = rv[1] = Best{0, 0, 0};
    if (!sc.forwardOnly) {
      PassSeq rs[2];
      bool any = false;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const bool run = !over[h] && fw[h].s > 0;
        any |= run;
        rs[h] = run ? PassSeq{codes, ps[h].a + fw[h].j, ps[h].b + fw[h].i, fw[h].j + 1, fw[h].i + 1, -1, -1}
                    : PassSeq{codes, ps[h].a, ps[h].b, 0, 0, 1, 1};
      }
      bool dummy[2];
      if (any) thread_pass<K>(sc, s_warp, s_simp, rs, scr, stride, t, rv, dummy);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (pid[h] < 0) continue;
      if (over[h]) {
        const int slot = atomicAdd(&st->overflow_count, 1);
        overflow_list[slot] = pid[h];
        if (rerun_cells)
          atomicAdd(rerun_cells, (unsigned long long)ps[h].alen * (unsigned long long)ps[h].blen);
        continue;
      }
      write_result(sc, fw[h], rv[h], score, arange, brange, pid[h]);
    }
  }
}

}  // namespace ipuma_dev
