// engine.cu -- the C ABI of include/ipuma_b200.h: engine lifecycle, device
// buffers, the cost-binned scheduling pipeline and the kernel launches.
//
// One engine = one CUDA device + one stream.  Calls on an engine are
// serialised by its mutex; device buffers grow on demand and are reused.
// Jobs (ipuma_gpu_submit_buffer) are stream-ordered and tracked by events.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "errors.h"
#include "ipuma_b200.h"
#include "sw_kernels.cuh"
#include "sw_thread.cuh"
#include "../host/swatlib/encoding.h"
#include "../host/swatlib/similarity.h"

using namespace ipuma_dev;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace ipuma_internal {
int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
}  // namespace ipuma_internal

namespace {
using ipuma_internal::fail;

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return fail(IPUMA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(_e));       \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes, cudaStream_t s) {
    if (bytes <= cap && p) return IPUMA_OK;
    const size_t old = cap;
    if (p) {
      cudaStreamSynchronize(s);
      cudaFree(p);
      p = nullptr;
      cap = 0;
    }
    // Geometric growth: a stream of slowly growing batches reallocates
    // (and synchronises the device in cudaFree) only a few times.
    size_t want = std::max<size_t>({bytes, (size_t)256, old + old / 2});
    want = (want + (1u << 20) - 1) & ~(size_t)((1u << 20) - 1);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(IPUMA_ERR_NO_MEMORY, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    cap = want;
    return IPUMA_OK;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Kernel classes of the batched pipeline.  s16x2 classes by |A| (columns
// per strip = lanes * K), then the s32 class; the rerun reuses the s32
// kernel.
// lanes = lanes per pair group (0: the per-thread class, no wavefront),
// k = columns per lane, width = columns per strip.
struct ClassDef {
  int lanes, k, kind, width;
};
constexpr int kNumS16 = 21;     // s16x2 classes chosen by cost
constexpr int kNumClasses = kNumS16 + 3;  // + the s32 class, the hybrid class, the strip-team class
constexpr ClassDef kClasses[kNumClasses] = {
    {16, 4, IPUMA_KERNEL_S16_L16_K4, 64},    {16, 8, IPUMA_KERNEL_S16_L16_K8, 128},
    {16, 12, IPUMA_KERNEL_S16_L16_K12, 192}, {16, 16, IPUMA_KERNEL_S16_L16_K16, 256},
    {32, 12, IPUMA_KERNEL_S16_L32_K12, 384}, {32, 16, IPUMA_KERNEL_S16_L32_K16, 512},
    {0, 16, IPUMA_KERNEL_S16_T_K16, 16},     {16, 6, IPUMA_KERNEL_S16_L16_K6, 96},
    {16, 10, IPUMA_KERNEL_S16_L16_K10, 160}, {16, 14, IPUMA_KERNEL_S16_L16_K14, 224},
    {16, 5, IPUMA_KERNEL_S16_L16_K5, 80},    {16, 7, IPUMA_KERNEL_S16_L16_K7, 112},
    {16, 9, IPUMA_KERNEL_S16_L16_K9, 144},   {16, 11, IPUMA_KERNEL_S16_L16_K11, 176},
    {16, 13, IPUMA_KERNEL_S16_L16_K13, 208}, {16, 15, IPUMA_KERNEL_S16_L16_K15, 240},
    {8, 8, IPUMA_KERNEL_S16_L8_K8, 64},      {8, 10, IPUMA_KERNEL_S16_L8_K10, 80},
    {8, 12, IPUMA_KERNEL_S16_L8_K12, 96},    {8, 14, IPUMA_KERNEL_S16_L8_K14, 112},
    {8, 16, IPUMA_KERNEL_S16_L8_K16, 128},
    {32, 16, IPUMA_KERNEL_S32_K16, 512},     {32, 16, IPUMA_KERNEL_S16_HYBRID, 512},
    {32, 16, IPUMA_KERNEL_S16_TEAM, 512},
};
constexpr int kClsWidest = 5;  // widest wavefront class (very long |A|)
constexpr int kMaxTimed = IPUMA_MAX_TIMED;  // launches timed per call (time_launches)
constexpr int kClsThread = 6;  // per-thread class k_thread<16>
constexpr int kClsS32 = kNumS16;
// Hybrid class: pairs whose score can pass int16 (main-diagonal bound) run
// their safe strips in s16x2 and the rest in s32 (option "hybrid").
constexpr int kClsHi = kNumS16 + 1;
// Strip-team class (k_strips<16>): the warps of a block share one item's
// 512-column strips, so a long pair finishes up to `warps` times sooner.
// Chosen for pairs of at least two strips whose one-warp latency the batch
// cannot hide (pair_key).  Warps per team: option "team_warps" (0 = off), capped by the
// batch's strip count.
constexpr int kClsTeam = kNumS16 + 2;
constexpr int kTeamWarpsDefault = 8;
// Per-thread class: rows it accepts (its boundary scratch is rows x threads)
// and the share of the batch's time one of its pairs may take.
constexpr int kThrMaxRows = 2048;
constexpr float kThrLatencyShare = 0.5f;
// Latency bound of every class (BinParams::lat_share): an item may take at
// most this share of the batch's modelled time (cells x fastest slot time
// / packing efficiency).  In small batches that sends pairs to the class
// that finishes them soonest: there one long pair, not throughput, sets the
// batch's time.
constexpr float kLatencyShare = 0.06f;  // measured best of 0.03-0.25 on the protein workloads
constexpr float kPackingEfficiency = 0.85f;
constexpr float kLatencyMinBatchPs = 0.f;
// Option "concurrent" = 3 (default) picks the launch mode by batch size:
// smaller batches leave most class launches with fewer items than resident
// warps, so the classes share the SMs (mode 1); larger ones alternate two
// streams (mode 2), which keeps one class per SM.
constexpr int kShareModeMaxPairs = 48000;
// The 16-lane classes at 16-column steps (every K from 4 to 16) cut column
// padding on large batches; a smaller batch uses the 64-column steps only
// (K = 4, 8, 12, 16), since every class launch costs a few microseconds
// even when empty.
constexpr int kFineClassMinPairs = 150000;
constexpr unsigned kCoarseClasses = (1u << 0) | (1u << 1) | (1u << 2) | (1u << 3) | (1u << 4) | (1u << 5);
// 8-lane groups for the five narrowest strip widths (64 to 128 columns):
// twice the columns per lane over a wavefront half as deep, so the per-step
// work of a lane covers twice the cells.  Their profiles take twice the
// shared memory per warp, so they replace the 16-lane classes of the same
// widths only with the four-row profile of 2-bit codes (measured on B200:
// 1M DNA 3383 -> 3546 GCUPS; 200k protein with 25-row profiles 2960 -> 2855,
// from half the resident warps).
// {16-lane class, 8-lane class of the same width}: 64, 80, 96, 112, 128 columns.
constexpr int kNarrowPairs[5][2] = {{0, 16}, {10, 17}, {7, 18}, {11, 19}, {1, 20}};
constexpr unsigned kFineClasses = (1u << 7) | (1u << 8) | (1u << 9) | (1u << 10) | (1u << 11) | (1u << 12) |
                                  (1u << 13) | (1u << 14) | (1u << 15);
constexpr int kWarpsPerBlock = 4;
// Chunked upload/compute overlap of ipuma_gpu_compare.
constexpr int kMaxChunks = 8;
constexpr int kChunkMinPairs = 250000;        // automatic chunking from 2 x this many pairs
// Pairs per automatic chunk: each chunk adds ~0.9 ms of launches and tails
// while more chunks expose less of the first upload (1M DNA pairs, B200: 3
// chunks 19.9 ms, 4 chunks 20.4 ms, 6 chunks 22.6 ms with 4-bit codes).
constexpr int kChunkPairs = 333334;
constexpr int kValidateMaxThreads = 16;       // host threads checking pair descriptors
constexpr int kValidatePairsPerThread = 65536;
constexpr size_t kChunkMinBytes = 32u << 20;  // and the batch uploads at least this much
constexpr int kThreads = 32 * kWarpsPerBlock;

// Status of one wire-buffer job, copied from its control block to pinned
// host memory by the job's own stream before any later job can clear it.
struct JobStatus {
  DevStatus st;
};

// One asynchronous wire-buffer batch (ipuma_gpu_submit_buffer).
struct Job {
  cudaEvent_t ev[3] = {};       // start, inputs uploaded, kernels done
  cudaEvent_t done = nullptr;   // after the job's last copy (timing too)
  JobStatus* status = nullptr;  // pinned, from the engine's pool
  int32_t* staged = nullptr;    // pinned results staging (pageable destination)
  size_t staged_bytes = 0;
  int32_t* results = nullptr;   // the caller's results buffer
  size_t n_results = 0;
  ipuma_stats stats{};
};

// Buffers and stream of one in-flight wire batch.  Wire jobs alternate
// between two such sets, so one batch's upload and result copy overlap the
// previous batch's kernels.
struct WireBufs {
  DevBuf inputs, results, pairs, ctl, list, scratch, ovf, flag;
};

}  // namespace

struct ipuma_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nsm = 0;
  ipuma_sw_config sw{};
  ipuma_algo_config algo{};
  std::vector<int8_t> sim;
  int M = 0;
  int maxSub = 0;
  SwConst sc{};
  bool fast_ok = false;  // wavefront kernels valid for this scoring
  bool s16_ok = false;   // s16x2 lanes valid for this scoring
  int s16_max_len = 0;

  // options
  int scheduler = 0;
  int plain_s16 = 0;  // option "plain_lanes" = 16: the plain kernel in s16x2 lanes (k_plain16)
  int trace = 0;      // option "trace": first start / last end of every class launch
  int graphs = 0;
  int tile_k = 0;
  int team_warps = kTeamWarpsDefault;  // option "team_warps": warps of a strip team (0 = no team class)
  int smem_optin = 0;                  // shared memory a block may opt in to
  int time_launches = 0;
  // option "thread_class": the per-thread class may be chosen.  Off by
  // default: on the benchmark batches its divergence between pairs of
  // different lengths made it slower than the wavefront classes.
  int thread_class = 0;

  // autotuned per-class rates of the class choice (BinParams)
  float slot_ps[NCLASS_MAX] = {};
  float strip_ps[NCLASS_MAX] = {};
  bool tuned = false;
  int autotune = 1;  // tune lazily before the first batched launch
  int long_a = 3072; // |A| above which pairs take the widest class
  std::string tune_source = "defaults";

  // per-launch timing of the current call (time_launches)
  cudaEvent_t tev[2 * kMaxTimed] = {};
  int n_timed = 0;
  int timed_kind[kMaxTimed] = {};
  int timed_cls[kMaxTimed] = {};

  DevBuf d_sim, d_codes, d_pairs, d_list, d_res, d_scratch, d_cf, d_ovf, d_ctl, d_inputs, d_wres, d_flag;
  DevBuf d_packed;  // 4-bit codes of ipuma_gpu_compare_packed before expansion
  // Second buffer set and streams of the chunked host-to-host path
  // (ipuma_gpu_compare): chunks alternate between `stream` and `stream2`
  // while `copy_stream` uploads the next chunks.
  DevBuf x_list, x_scratch, x_ovf, x_flag;
  // One stream per kernel class: the class launches of a batch run
  // concurrently, each on its share of the SMs (option "concurrent").
  cudaStream_t cls_stream[NCLASS_MAX] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[NCLASS_MAX] = {};
  int concurrent = 3;
  int hybrid = 1;  // option "hybrid": high-scoring pairs run s16x2 strips while provably safe
  float latency_share = kLatencyShare;  // option "latency_share" (per mille)
  cudaStream_t stream2 = nullptr, copy_stream = nullptr;
  cudaEvent_t cev[2 * kMaxChunks + 2] = {};
  int chunks = 0;  // option "chunks": 0 automatic, 1 off, n fixed
  std::map<std::pair<const void*, int>, int> grid_cache;  // {kernel, smem} -> grid
  // Captured pipelines of compare_device, by shape and buffers (option "graphs").
  std::map<std::vector<uint64_t>, cudaGraphExec_t> graphs_cache;
  std::map<cudaGraphExec_t, int> graph_launches;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  ipuma_stats stats{};
  std::mutex mu;
  std::map<uint64_t, Job> jobs;
  uint64_t next_job = 1;
  // Second wire-buffer set and its stream (the first set is the engine's
  // main buffers on `stream`); wire jobs alternate between the two.
  WireBufs w1;
  cudaStream_t wstream1 = nullptr;
  uint64_t wire_jobs = 0;
  // Recycled per-job resources: timing events, pinned status slots and
  // pinned result staging buffers (by size).
  std::vector<cudaEvent_t> free_events;
  std::vector<JobStatus*> free_status;
  std::multimap<size_t, int32_t*> free_staging;
  std::vector<void*> pinned_blocks;  // every pinned allocation, freed at destroy
};

namespace {

// Layout of the control block (ints): status, class ranges, queue heads,
// histogram, offsets.
constexpr int CTL_STATUS = 0;                       // DevStatus (4 ints)
constexpr int CTL_RANGES = 4;                       // 2 * NCLASS_MAX
constexpr int CTL_HEADS = CTL_RANGES + 2 * NCLASS_MAX;  // NCLASS_MAX + 1
constexpr int CTL_INFO = CTL_HEADS + NCLASS_MAX + 1;    // wire check {maxA, maxB, bad} (+1 pad)
constexpr int CTL_CELLS = ((CTL_INFO + 4) + 1) & ~1;    // 8-byte aligned: NCELLS uint64
constexpr int NCELLS = NCLASS_MAX + 3;              // per class, rerun, wire check, batch total
constexpr int CTL_COST = CTL_CELLS + 2 * NCELLS;    // modelled cost per class (uint64, ps)
constexpr int CTL_ALLOT = CTL_COST + 2 * NCLASS_MAX;  // ClassAllot per class + rerun (4 ints each)
static_assert(CTL_COST % 2 == 0 && CTL_ALLOT % 2 == 0, "8-byte aligned control block fields");
constexpr int CTL_TRACE = CTL_ALLOT + 4 * (NCLASS_MAX + 1);  // {~start, end} ns per class + rerun (uint64)
static_assert(CTL_TRACE % 2 == 0, "8-byte aligned trace");
constexpr int CTL_HIST = CTL_TRACE + 4 * (NCLASS_MAX + 1);  // NCLASS_MAX * NBUCKET
constexpr int CTL_OFFS = CTL_HIST + NCLASS_MAX * NBUCKET;
constexpr int CTL_INTS = CTL_OFFS + NCLASS_MAX * NBUCKET;
constexpr int CELLS_RERUN = NCLASS_MAX;             // index of the rerun cells
constexpr int CELLS_WIRE = NCLASS_MAX + 1;          // cells found by the wire check
constexpr int CELLS_TOTAL = NCLASS_MAX + 2;         // cells of the batch (k_bin_total)

// A kernel's dynamic shared memory limit is one process-wide attribute per
// device, shared by every engine: engines with different alphabets need
// different sizes and may run concurrently on several threads, so the limit
// only ever grows (lowering it would break another engine's launches).
template <class K>
void raise_smem_limit(int device, K kernel, int smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> limit;
  if (smem <= 48 * 1024) return;
  std::lock_guard<std::mutex> lock(mu);
  int& cur = limit[{device, reinterpret_cast<const void*>(kernel)}];
  if (smem > cur && cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
                        cudaSuccess)
    cur = smem;
}

// Persistent grid of a kernel: resident blocks per SM times SMs.  Computed
// once per kernel and engine (engine creation warms the cache, so no
// occupancy query or attribute change happens during a graph capture).
template <class K>
int occupancy_grid(ipuma_engine* e, K kernel, int smem, int threads = kThreads) {
  // Key: the kernel and its shared memory (and block size, when not kThreads).
  const auto key =
      std::make_pair(reinterpret_cast<const void*>(kernel), smem + (threads == kThreads ? 0 : threads << 20));
  auto it = e->grid_cache.find(key);
  if (it != e->grid_cache.end()) return it->second;
  int nb = 0;
  raise_smem_limit(e->device, kernel, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem);
  if (nb < 1) nb = 1;
  e->grid_cache[key] = nb * e->nsm;
  return nb * e->nsm;
}

// Letters of the query profile for codes of `bits` bits: 2-bit codes are
// A/C/G/T (codes 1..4), so their profile needs four rows, not one per
// letter of the alphabet -- less shared memory, more resident blocks.
int prof_letters(const ipuma_engine* e, int bits) { return (bits == 2 && e->M >= 5) ? 4 : e->M; }

// Shared memory of a wavefront launch whose profile has P letters (P < 0:
// one per letter of the alphabet).
template <class T, int K, int LANES>
int smem_for(const ipuma_engine* e, int P = -1) {
  return SmemLayout<T, K, LANES>::total(e->M, P < 0 ? e->M : P, kWarpsPerBlock);
}

// Grid of a k_batched<T, K, LANES, HYB> launch (the instantiation for the
// engine's forwardOnly, which is fixed at creation) with a P-letter profile.
template <class T, int K, int LANES, bool HYB = false>
int batched_grid(ipuma_engine* e, int P) {
  return e->sc.forwardOnly ? occupancy_grid(e, k_batched<T, K, LANES, HYB, true>, smem_for<T, K, LANES>(e, P))
                           : occupancy_grid(e, k_batched<T, K, LANES, HYB, false>, smem_for<T, K, LANES>(e, P));
}

int team_smem(const ipuma_engine* e, int P, int warps) {
  return SmemLayout<Lane16, 16, 32>::total(e->M, P, warps);
}

// Static shared memory of k_strips (progress words, merge slots) plus slack.
constexpr int kTeamStaticSmem = 1024;

// Warps of a strip team for a batch whose longest A is maxA, with a
// P-letter profile: the engine's team_warps, but no more than the strips
// of that A (a warp without a strip would idle for the whole item; two at
// least) and no more than the shared memory holds.  0: no team (the option
// is 0, or two warps do not fit).
int team_warps_for(const ipuma_engine* e, int P, int maxA) {
  const int strips = (std::max(maxA, 1) + kClasses[kClsTeam].width - 1) / kClasses[kClsTeam].width;
  int w = std::min({e->team_warps, std::max(strips, 2), kTeamMaxWarps});
  while (w >= 2 && team_smem(e, P, w) + kTeamStaticSmem > e->smem_optin) --w;
  return w >= 2 ? w : 0;
}

// Grid of a k_strips<16> launch with `warps` warps per block.
int team_grid(ipuma_engine* e, int P, int warps) {
  return occupancy_grid(e, k_strips<16>, team_smem(e, P, warps), 32 * warps);
}

template <int K>
int thread_smem(const ipuma_engine* e) {
  return ThreadSmem<K>::total(e->M, kWarpsPerBlock);
}

// Threads of a k_thread<K> launch (one boundary column each).
template <int K>
long thread_threads(ipuma_engine* e) {
  return (long)occupancy_grid(e, k_thread<K>, thread_smem<K>(e)) * kThreads;
}

// Lane groups (one scratch slice each) of the widest batched launch (either
// profile size).
int max_batched_groups(ipuma_engine* e) {
  int g = 0;
  for (int P : {e->M, prof_letters(e, 2)}) {
    g = std::max(g, batched_grid<Lane16, 4, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 8, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 12, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 16, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 6, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 10, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 14, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 5, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 7, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 9, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 11, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 13, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 15, 16>(e, P) * 2);
    g = std::max(g, batched_grid<Lane16, 8, 8>(e, P) * 4);
    g = std::max(g, batched_grid<Lane16, 10, 8>(e, P) * 4);
    g = std::max(g, batched_grid<Lane16, 12, 8>(e, P) * 4);
    g = std::max(g, batched_grid<Lane16, 14, 8>(e, P) * 4);
    g = std::max(g, batched_grid<Lane16, 16, 8>(e, P) * 4);
    g = std::max(g, batched_grid<Lane16, 12, 32>(e, P));
    g = std::max(g, batched_grid<Lane16, 16, 32>(e, P));
    g = std::max(g, batched_grid<LaneS32, 16, 32>(e, P));
    g = std::max(g, batched_grid<LaneHi, 16, 32, true>(e, P));
    // Warm the cache of the team grids (no occupancy query during a capture).
    for (int w = 2; w <= std::min(e->team_warps, kTeamMaxWarps); ++w)
      if (team_smem(e, P, w) + kTeamStaticSmem <= e->smem_optin) team_grid(e, P, w);
  }
  return g * kWarpsPerBlock;
}

// Device buffers of one run of the batched pipeline: the control block and
// the per-run work lists and strip scratch.  Two runs may execute at once
// (on two streams) only with disjoint sets.
struct RunBufs {
  int* ctl;  // CTL_INTS ints, cleared before the run
  DevBuf* scratch;
  DevBuf* list;
  DevBuf* ovf;
  DevBuf* flag;
  // First of the two class streams of alternating launches (0 or 2): a
  // second buffer set runs its classes on streams of its own, so its
  // launches fill the tails of a run on the first set instead of queueing
  // behind them.
  int cls_base = 0;
};

// The engine's default set (control block at the start of d_ctl).
RunBufs main_bufs(ipuma_engine* e) {
  return RunBufs{e->d_ctl.as<int>(), &e->d_scratch, &e->d_list, &e->d_ovf, &e->d_flag};
}

// Brackets one alignment-kernel launch with events when time_launches is set.
int timed_begin(ipuma_engine* e, cudaStream_t s, int kind, int cls) {
  if (!e->time_launches || e->n_timed >= kMaxTimed) return IPUMA_OK;
  if (!e->tev[2 * e->n_timed]) {
    CUDA_TRY(cudaEventCreate(&e->tev[2 * e->n_timed]));
    CUDA_TRY(cudaEventCreate(&e->tev[2 * e->n_timed + 1]));
  }
  e->timed_kind[e->n_timed] = kind;
  e->timed_cls[e->n_timed] = cls;
  CUDA_TRY(cudaEventRecord(e->tev[2 * e->n_timed], s));
  return IPUMA_OK;
}

int timed_end(ipuma_engine* e, cudaStream_t s) {
  if (!e->time_launches || e->n_timed >= kMaxTimed) return IPUMA_OK;
  CUDA_TRY(cudaEventRecord(e->tev[2 * e->n_timed + 1], s));
  e->n_timed++;
  return IPUMA_OK;
}

// allot_idx = entry of the control block's ClassAllot table (the class, or
// NCLASS_MAX for the s32 rerun).
template <class T, int K, int LANES, bool HYB = false>
int launch_batched(ipuma_engine* e, const SwConst& sc, const RunBufs& rb, cudaStream_t s, const uint8_t* codes,
                   const PairDesc* pairs, const int* list, const int* range, int* head, long rowsCap,
                   int* score, int* arange, int* brange, int kind, int cls, int allot_idx) {
  const int smem = smem_for<T, K, LANES>(e, sc.P);
  const int grid = batched_grid<T, K, LANES, HYB>(e, sc.P);
  int* ctl = rb.ctl;
  auto* cells = reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS);
  int rc;
  if ((rc = timed_begin(e, s, kind, cls))) return rc;
  auto* kern = e->sc.forwardOnly ? k_batched<T, K, LANES, HYB, true> : k_batched<T, K, LANES, HYB, false>;
  kern<<<grid, kThreads, smem, s>>>(
      sc, e->d_sim.as<int8_t>(), codes, pairs, list, range, head, rb.scratch->as<int2>(),
      rowsCap, score, arange, brange, rb.ovf->as<int>(), cells + CELLS_RERUN,
      reinterpret_cast<DevStatus*>(ctl + CTL_STATUS),
      reinterpret_cast<const ClassAllot*>(ctl + CTL_ALLOT) + allot_idx,
      e->trace ? reinterpret_cast<unsigned long long*>(ctl + CTL_TRACE) + 2 * allot_idx : nullptr);
  CUDA_TRY(cudaGetLastError());
  return timed_end(e, s);
}

// Launches the strip-team class (`warps` warps per block) over its list range.
int launch_team(ipuma_engine* e, const SwConst& sc, const RunBufs& rb, cudaStream_t s, const uint8_t* codes,
                const PairDesc* pairs, const int* list, const int* range, int* head, long rowsCap, int* score,
                int* arange, int* brange, int warps) {
  const int smem = team_smem(e, sc.P, warps);
  const int grid = team_grid(e, sc.P, warps);
  int* ctl = rb.ctl;
  auto* cells = reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS);
  int rc;
  if ((rc = timed_begin(e, s, kClasses[kClsTeam].kind, kClsTeam))) return rc;
  k_strips<16><<<grid, 32 * warps, smem, s>>>(
      sc, e->d_sim.as<int8_t>(), codes, pairs, list, range, head, rb.scratch->as<int2>(), rowsCap, score, arange,
      brange, rb.ovf->as<int>(), cells + CELLS_RERUN, reinterpret_cast<DevStatus*>(ctl + CTL_STATUS),
      reinterpret_cast<const ClassAllot*>(ctl + CTL_ALLOT) + kClsTeam,
      e->trace ? reinterpret_cast<unsigned long long*>(ctl + CTL_TRACE) + 2 * kClsTeam : nullptr);
  CUDA_TRY(cudaGetLastError());
  return timed_end(e, s);
}

// Launches the per-thread class over its list range; rowsCap = rows of
// the boundary scratch per thread.
template <int K>
int launch_thread(ipuma_engine* e, const RunBufs& rb, cudaStream_t s, const uint8_t* codes,
                  const PairDesc* pairs, const int* list, const int* range, int* head, long rowsCap,
                  int* score, int* arange, int* brange, int cls) {
  const int smem = thread_smem<K>(e);
  const int grid = occupancy_grid(e, k_thread<K>, smem);
  int* ctl = rb.ctl;
  auto* cells = reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS);
  int rc;
  if ((rc = timed_begin(e, s, kClasses[cls].kind, cls))) return rc;
  k_thread<K><<<grid, kThreads, smem, s>>>(e->sc, e->d_sim.as<int8_t>(), codes, pairs, list, range, head,
                                           rb.scratch->as<int2>(), rowsCap, score, arange, brange,
                                           rb.ovf->as<int>(), cells + CELLS_RERUN,
                                           reinterpret_cast<DevStatus*>(ctl + CTL_STATUS),
                                           reinterpret_cast<const ClassAllot*>(ctl + CTL_ALLOT) + cls);
  CUDA_TRY(cudaGetLastError());
  return timed_end(e, s);
}

// Grows every buffer run_batched uses for a batch of this shape, so that
// the pipeline itself allocates nothing (graph capture).
// Rows of the per-thread class's boundary scratch (0 when no pair of the
// batch can need a second strip there).  The class only takes pairs of at
// most kThrMaxRows rows, unless option tile_k forces every pair into it.
long thread_rows(const ipuma_engine* e, int maxA, int maxB) {
  if (maxA <= kClasses[kClsThread].width) return 0;
  return e->tile_k == kClsThread + 1 ? maxB : std::min(maxB, kThrMaxRows);
}

// Strip-boundary scratch (int2) of one run: the wavefront classes need two
// columns of rowsCap per lane group, the per-thread class one column of
// thread_rows per thread.
// Full-occupancy grid and strip scratch (int2) per block of every class,
// for a P-letter profile.
void class_grids(ipuma_engine* e, int P, int maxA, int maxB, int* grid, long long* spb) {
  const long long rowsCap = std::max(1, maxB);
  for (int c = 0; c < kNumClasses; ++c) {
    switch (c) {
      case kClsHi: grid[c] = batched_grid<LaneHi, 16, 32, true>(e, P); break;
      case 0: grid[c] = batched_grid<Lane16, 4, 16>(e, P); break;
      case 1: grid[c] = batched_grid<Lane16, 8, 16>(e, P); break;
      case 2: grid[c] = batched_grid<Lane16, 12, 16>(e, P); break;
      case 3: grid[c] = batched_grid<Lane16, 16, 16>(e, P); break;
      case 4: grid[c] = batched_grid<Lane16, 12, 32>(e, P); break;
      case 5: grid[c] = batched_grid<Lane16, 16, 32>(e, P); break;
      case kClsThread: grid[c] = (int)(thread_threads<16>(e) / kThreads); break;
      case 7: grid[c] = batched_grid<Lane16, 6, 16>(e, P); break;
      case 8: grid[c] = batched_grid<Lane16, 10, 16>(e, P); break;
      case 9: grid[c] = batched_grid<Lane16, 14, 16>(e, P); break;
      case 10: grid[c] = batched_grid<Lane16, 5, 16>(e, P); break;
      case 11: grid[c] = batched_grid<Lane16, 7, 16>(e, P); break;
      case 12: grid[c] = batched_grid<Lane16, 9, 16>(e, P); break;
      case 13: grid[c] = batched_grid<Lane16, 11, 16>(e, P); break;
      case 14: grid[c] = batched_grid<Lane16, 13, 16>(e, P); break;
      case 15: grid[c] = batched_grid<Lane16, 15, 16>(e, P); break;
      case 16: grid[c] = batched_grid<Lane16, 8, 8>(e, P); break;
      case 17: grid[c] = batched_grid<Lane16, 10, 8>(e, P); break;
      case 18: grid[c] = batched_grid<Lane16, 12, 8>(e, P); break;
      case 19: grid[c] = batched_grid<Lane16, 14, 8>(e, P); break;
      case 20: grid[c] = batched_grid<Lane16, 16, 8>(e, P); break;
      case kClsTeam: {
        const int w = team_warps_for(e, P, maxA);
        grid[c] = w ? team_grid(e, P, w) : 0;
        spb[c] = (long long)w * rowsCap;  // one boundary column per warp of a team
        continue;
      }
      default: grid[c] = batched_grid<LaneS32, 16, 32>(e, P); break;
    }
    if (c == kClsThread)
      spb[c] = (long long)kThreads * thread_rows(e, maxA, maxB);
    else
      spb[c] = (long long)kWarpsPerBlock * (32 / kClasses[c].lanes) * (c == kClsHi ? 3 : 2) * rowsCap;
  }
}

// Scratch for any split of the GPU between the classes: shares are
// fractions f_c of each class's full grid with sum f_c = 1, rounded up.
// With two alternating streams (option concurrent = 2) two full-grid
// launches may run at once: two regions of the largest full grid.
size_t scratch_int2(ipuma_engine* e, int maxA, int maxB) {
  int grid[NCLASS_MAX + 1];
  long long spb[NCLASS_MAX + 1];
  long long full = 0, round = 0;
  for (int P : {e->M, prof_letters(e, 2)}) {  // the smaller profile may fit more blocks
    class_grids(e, P, maxA, maxB, grid, spb);
    long long r = 0;
    for (int c = 0; c < kNumClasses; ++c) {
      full = std::max(full, (long long)grid[c] * spb[c]);
      r += spb[c];
    }
    round = std::max(round, r);
  }
  return (size_t)std::max(full + round, 2 * full);
}

// Launch order of the classes (longest-tail classes first) and, for two
// alternating streams, the stream (and scratch region) of each.
// The hybrid class and the widest class (the long pairs of a heavy-tailed
// batch) come first and land on different streams, so the widest class's
// blocks start on the SMs the hybrid class frees during its tail.
constexpr int kLaunchOrder[kNumClasses] = {23, 22, 5, 21, 4, 6, 3, 15, 9, 14, 2, 13, 8, 12, 1, 20, 11, 19, 7, 18, 10, 17, 0, 16};

int reserve_bufs(ipuma_engine* e, const RunBufs& rb, cudaStream_t s, int n, int maxA, int maxB) {
  int rc;
  if ((rc = rb.scratch->ensure(sizeof(int2) * scratch_int2(e, maxA, maxB), s))) return rc;
  if ((rc = rb.list->ensure(sizeof(int) * (size_t)n + 64, s))) return rc;
  if ((rc = rb.ovf->ensure(sizeof(int) * (size_t)n + 64, s))) return rc;
  if ((rc = rb.flag->ensure((size_t)n + 64, s))) return rc;
  return IPUMA_OK;
}

int reserve_batched(ipuma_engine* e, cudaStream_t s, int n, int maxA, int maxB) {
  int rc;
  if ((rc = e->d_ctl.ensure(sizeof(int) * CTL_INTS, s))) return rc;
  return reserve_bufs(e, main_bufs(e), s, n, maxA, maxB);
}

// Runs the persistent cost-binned pipeline over n device-resident pairs.
// Results land at score[p], arange[p], brange[p].
// n_codes = residues the code array holds: pairs reaching past it are
// rejected on the device (status ERR_RANGE) before any code is read.
// bits = bits per residue of `codes` (8: bytes; 2, 4, 5: packed, code_at).
int run_batched(ipuma_engine* e, const RunBufs& rb, cudaStream_t s, const uint8_t* codes, size_t n_codes,
                int bits, const PairDesc* pairs, int n, int maxA, int maxB, int* score, int* arange,
                int* brange, int* launches) {
  int rc;
  if (n <= 0) return IPUMA_OK;
  int* ctl = rb.ctl;
  DevStatus* st = reinterpret_cast<DevStatus*>(ctl + CTL_STATUS);
  SwConst sc = e->sc;
  sc.bits = bits;
  sc.P = prof_letters(e, bits);
  sc.pshift = sc.P == e->M ? 0 : 1;

  if (!e->fast_ok) {
    // Exact per-thread kernel; C and F rows in global scratch.
    const long maxAcap = std::max(1, maxA);
    long threads = std::min<long>(n, std::max<long>(1024, (512l << 20) / (8 * maxAcap)));
    threads = ((threads + 127) / 128) * 128;
    if ((rc = e->d_cf.ensure(sizeof(int) * 2 * maxAcap * threads, s))) return rc;
    if ((rc = timed_begin(e, s, IPUMA_KERNEL_EXACT, -1))) return rc;
    k_exact<<<(int)(threads / 128), 128, 0, s>>>(sc, e->d_sim.as<int8_t>(), codes, (long long)n_codes, pairs, n,
                                                  e->d_cf.as<int>(), maxAcap, maxB, score, arange, brange, st);
    CUDA_TRY(cudaGetLastError());
    if ((rc = timed_end(e, s))) return rc;
    *launches += 1;
    return IPUMA_OK;
  }

  // Scratch for strip boundaries and the lists.
  const long rowsCap = std::max(1, maxB);
  if ((rc = rb.scratch->ensure(sizeof(int2) * scratch_int2(e, maxA, maxB), s))) return rc;
  if ((rc = rb.list->ensure(sizeof(int) * (size_t)n + 64, s))) return rc;
  if ((rc = rb.ovf->ensure(sizeof(int) * (size_t)n + 64, s))) return rc;

  BinParams bp{};
  bp.n_s16_classes = kNumS16;
  bp.cls_s32 = kClsS32;
  bp.cls_hi = e->hybrid ? kClsHi : kClsS32;
  bp.nclass = kNumClasses;
  bp.s16_max_len = e->s16_max_len;
  bp.force_s32 = e->s16_ok ? 0 : 1;
  for (int c = 0; c < kNumClasses; ++c) {
    bp.lanes[c] = kClasses[c].lanes;
    bp.width[c] = kClasses[c].width;
    bp.slot_ps[c] = e->slot_ps[c];
    bp.strip_ps[c] = e->strip_ps[c];
  }
  bp.widest = kClsWidest;
  const long thrThreads = thread_threads<16>(e);
  bp.thr_cls = kClsThread;
  bp.thr_on = e->thread_class && bits == 8;
  bp.thr_k = kClasses[kClsThread].width;
  bp.thr_max_rows = kThrMaxRows;
  bp.thr_cap_scale = kThrLatencyShare / (2.0f * (float)thrThreads);
  bp.total_cells = reinterpret_cast<const unsigned long long*>(ctl + CTL_CELLS) + CELLS_TOTAL;
  // Concurrent class launches, except when every launch is timed alone.
  const int mode = e->time_launches ? 0
                   : e->concurrent == 3 ? (n < kShareModeMaxPairs ? 1 : 2)
                                        : e->concurrent;
  const bool conc = mode != 0;
  bp.concurrent = mode;
  // Classes this batch may use (the others are not launched).
  unsigned enabled = kCoarseClasses | (1u << kClsS32);
  if (e->hybrid) enabled |= 1u << kClsHi;
  if (n >= kFineClassMinPairs) enabled |= kFineClasses;
  if (e->thread_class && bits == 8) enabled |= 1u << kClsThread;  // k_thread reads bytes only
  if (sc.P < e->M) {
    // Four-row profiles: the narrow widths in 8-lane groups.
    for (const auto& w : kNarrowPairs)
      if ((enabled >> w[0]) & 1u) enabled = (enabled & ~(1u << w[0])) | (1u << w[1]);
  }
  // Strip teams: batches with pairs of two strips or more, unless tile_k
  // forces another class (then no pair could reach a team).
  const bool teamForced = e->tile_k == kClsTeam + 1;
  const int teamW = e->team_warps >= 2 ? team_warps_for(e, sc.P, maxA) : 0;
  if (teamForced && teamW < 2)
    return fail(IPUMA_ERR_INVALID_ARG, "tile_k %d (strip teams) needs team_warps >= 2 and room for two warps",
                kClsTeam + 1);
  if (teamW >= 2 && maxA > kClasses[kClsTeam].width && e->tile_k == 0) enabled |= 1u << kClsTeam;
  if (e->tile_k > 0) enabled |= 1u << (e->tile_k - 1);
  bp.enabled = enabled;
  bp.team_cls = ((enabled >> kClsTeam) & 1u) ? kClsTeam : -1;
  bp.team_warps = std::max(teamW, 1);
  class_grids(e, sc.P, maxA, maxB, bp.grid, bp.scr_per_block);
  bp.scr_cap = (long long)(rb.scratch->cap / sizeof(int2));
  float slot_min = 1e30f;
  for (int c = 0; c < kNumS16; ++c) {
    // cell slots one warp step covers: 32 lanes x k columns x 2 pairs
    // (the per-thread class: 32 threads x 16 columns x 2 pairs per row)
    bp.step_ps[c] = e->slot_ps[c] * 64.f * (float)kClasses[c].k * (float)(bp.grid[c] * kWarpsPerBlock);
    if (c != kClsThread) slot_min = std::min(slot_min, e->slot_ps[c]);
  }
  // A warp of a team steps like one of the widest class's warps.
  bp.step_ps[kClsTeam] =
      e->slot_ps[kClsTeam] * 64.f * (float)kClasses[kClsTeam].k * (float)(bp.grid[kClsTeam] * bp.team_warps);
  bp.batch_ps_per_cell = slot_min / kPackingEfficiency;
  bp.lat_share = e->latency_share;
  bp.lat_min_ps = kLatencyMinBatchPs;
  bp.region = 0;
  for (int c = 0; c < kNumClasses; ++c) bp.region = std::max(bp.region, (long long)bp.grid[c] * bp.scr_per_block[c]);
  // Two alternating streams: stream (and scratch region) by position
  // among the launched classes.
  for (int k = 0, pos = 0; k < kNumClasses; ++k) {
    const int c = kLaunchOrder[k];
    bp.slot_of[c] = pos & 1;
    if ((enabled >> c) & 1u) ++pos;
  }
  bp.long_a = e->long_a;
  // tile_k > 0 forces one s16x2 class: every pair uses the chosen kernel,
  // long A crossing several strips.
  bp.forced_class = e->tile_k > 0 ? e->tile_k - 1 : -1;
  bp.max_a = maxA;
  bp.max_b = maxB;
  bp.n_codes = (long long)n_codes;
  bp.bits = bits;
  bp.M = e->M;
  bp.s16_limit = e->sc.s16Limit;
  if ((rc = rb.flag->ensure((size_t)n + 64, s))) return rc;
  const int nkeys = bp.nclass * NBUCKET;
  const int tb = 256;
  const int gb = std::min<int>((n + tb - 1) / tb, e->nsm * 8);
  k_bin_total<<<gb, tb, 0, s>>>(bp, pairs, n,
                                reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS) + CELLS_TOTAL);
  k_bin_bound<<<gb, tb, 0, s>>>(bp, codes, e->d_sim.as<int8_t>(), pairs, n, rb.flag->as<uint8_t>());
  k_bin_count<<<gb, tb, 0, s>>>(bp, codes, e->d_sim.as<int8_t>(), pairs, n, ctl + CTL_HIST,
                                rb.flag->as<uint8_t>(),
                                reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS),
                                reinterpret_cast<unsigned long long*>(ctl + CTL_COST), st, score,
                                arange, brange);
  k_bin_scan<<<1, 1024, 0, s>>>(bp, nkeys, ctl + CTL_HIST, ctl + CTL_OFFS, ctl + CTL_RANGES,
                                reinterpret_cast<const unsigned long long*>(ctl + CTL_COST),
                                reinterpret_cast<ClassAllot*>(ctl + CTL_ALLOT), st);
  k_bin_scatter<<<gb, tb, 0, s>>>(bp, pairs, n, rb.flag->as<uint8_t>(), ctl + CTL_OFFS,
                                  rb.list->as<int>());
  CUDA_TRY(cudaGetLastError());
  *launches += 5;

  int* list = rb.list->as<int>();
  int* heads = ctl + CTL_HEADS;
  // Class launches: concurrently on the class streams (each on the share
  // of the SMs k_bin_scan gave it, so every class starts its longest items
  // at once and the classes finish together), or one after the other on
  // `s`, longest-tail classes first.
  if (conc) CUDA_TRY(cudaEventRecord(e->fork_ev, s));
  // Stream of a class: its own (shares) or one of two by launch position.
  auto stream_of = [&](int cls) -> int {
    if (mode == 2) return rb.cls_base + bp.slot_of[cls];
    return cls;
  };
  auto on = [&](int cls) -> cudaStream_t {
    if (!conc) return s;
    cudaStream_t cs = e->cls_stream[stream_of(cls)];
    cudaStreamWaitEvent(cs, e->fork_ev, 0);
    return cs;
  };
  auto done = [&](int cls) -> int {
    if (!conc) return IPUMA_OK;
    cudaStream_t cs = e->cls_stream[stream_of(cls)];
    CUDA_TRY(cudaEventRecord(e->join_ev[cls], cs));
    CUDA_TRY(cudaStreamWaitEvent(s, e->join_ev[cls], 0));
    return IPUMA_OK;
  };
  const int* R = ctl + CTL_RANGES;
#define IPUMA_LAUNCH(T, K, L, cls)                                                                     \
  if ((enabled >> (cls)) & 1u) {                                                                       \
    cudaStream_t cs = on(cls);                                                                         \
    if ((rc = launch_batched<T, K, L>(e, sc, rb, cs, codes, pairs, list, R + 2 * (cls), heads + (cls), \
                                      rowsCap, score, arange, brange, kClasses[cls].kind, cls, cls)))  \
      return rc;                                                                                       \
    if ((rc = done(cls))) return rc;                                                                   \
    ++*launches;                                                                                       \
  }
  if ((enabled >> kClsTeam) & 1u) {
    cudaStream_t cs = on(kClsTeam);
    if ((rc = launch_team(e, sc, rb, cs, codes, pairs, list, R + 2 * kClsTeam, heads + kClsTeam, rowsCap, score,
                          arange, brange, teamW)))
      return rc;
    if ((rc = done(kClsTeam))) return rc;
    ++*launches;
  }
  if ((enabled >> kClsHi) & 1u) {
    cudaStream_t cs = on(kClsHi);
    if ((rc = launch_batched<LaneHi, 16, 32, true>(e, sc, rb, cs, codes, pairs, list, R + 2 * kClsHi,
                                                      heads + kClsHi, rowsCap, score, arange, brange,
                                                      kClasses[kClsHi].kind, kClsHi, kClsHi)))
      return rc;
    if ((rc = done(kClsHi))) return rc;
    ++*launches;
  }
  IPUMA_LAUNCH(LaneS32, 16, 32, kClsS32)
  IPUMA_LAUNCH(Lane16, 16, 32, 5)
  IPUMA_LAUNCH(Lane16, 12, 32, 4)
  if ((enabled >> kClsThread) & 1u) {
    cudaStream_t cs = on(kClsThread);
    if ((rc = launch_thread<16>(e, rb, cs, codes, pairs, list, R + 2 * kClsThread, heads + kClsThread,
                                thread_rows(e, maxA, maxB), score, arange, brange, kClsThread)))
      return rc;
    if ((rc = done(kClsThread))) return rc;
    ++*launches;
  }
  IPUMA_LAUNCH(Lane16, 16, 16, 3)
  IPUMA_LAUNCH(Lane16, 15, 16, 15)
  IPUMA_LAUNCH(Lane16, 14, 16, 9)
  IPUMA_LAUNCH(Lane16, 13, 16, 14)
  IPUMA_LAUNCH(Lane16, 12, 16, 2)
  IPUMA_LAUNCH(Lane16, 11, 16, 13)
  IPUMA_LAUNCH(Lane16, 10, 16, 8)
  IPUMA_LAUNCH(Lane16, 9, 16, 12)
  IPUMA_LAUNCH(Lane16, 8, 16, 1)
  IPUMA_LAUNCH(Lane16, 16, 8, 20)
  IPUMA_LAUNCH(Lane16, 7, 16, 11)
  IPUMA_LAUNCH(Lane16, 14, 8, 19)
  IPUMA_LAUNCH(Lane16, 6, 16, 7)
  IPUMA_LAUNCH(Lane16, 12, 8, 18)
  IPUMA_LAUNCH(Lane16, 5, 16, 10)
  IPUMA_LAUNCH(Lane16, 10, 8, 17)
  IPUMA_LAUNCH(Lane16, 4, 16, 0)
  IPUMA_LAUNCH(Lane16, 8, 8, 16)
#undef IPUMA_LAUNCH
  // Exact 32-bit rerun of the s16x2 pairs whose score may have overflowed
  // (after every class: it reads their overflow list).
  if ((rc = launch_batched<LaneS32, 16, 32>(e, sc, rb, s, codes, pairs, rb.ovf->as<int>(), ctl + CTL_STATUS + 1,
                                            heads + NCLASS_MAX, rowsCap, score, arange, brange,
                                            IPUMA_KERNEL_S32_RERUN, CELLS_RERUN, NCLASS_MAX)))
    return rc;
  *launches += 1;
  return IPUMA_OK;
}

// Clears the control block at the start of every call.
int reset_ctl(ipuma_engine* e, cudaStream_t s) {
  int rc;
  if ((rc = e->d_ctl.ensure(sizeof(int) * CTL_INTS, s))) return rc;
  CUDA_TRY(cudaMemsetAsync(e->d_ctl.p, 0, sizeof(int) * CTL_INTS, s));
  e->n_timed = 0;
  return IPUMA_OK;
}

// Forward-pass cells counted for class c (or the rerun) over `nblk` runs.
template <size_t N>
unsigned long long cells_of(const unsigned long long (*cells)[N], int nblk, int c) {
  unsigned long long v = 0;
  for (int k = 0; k < nblk; ++k) v += cells[k][c];
  return v;
}

// Waits for the stream and reads the status of the call's runs: `nblk`
// consecutive control blocks at the start of d_ctl (one per run; errors,
// overflow reruns and per-class cells are summed).
int check_status(ipuma_engine* e, cudaStream_t s, int nblk = 1) {
  DevStatus st{};
  unsigned long long cells[NCELLS] = {};
  DevStatus stk[kMaxChunks];
  unsigned long long cellsk[kMaxChunks][NCELLS];
  unsigned long long tracek[kMaxChunks][2 * (NCLASS_MAX + 1)];
  int rangesk[kMaxChunks][2 * NCLASS_MAX];
  nblk = std::max(1, std::min(nblk, kMaxChunks));
  for (int k = 0; k < nblk; ++k) {
    const int* ctl = e->d_ctl.as<int>() + (size_t)k * CTL_INTS;
    CUDA_TRY(cudaMemcpyAsync(&stk[k], ctl + CTL_STATUS, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(cellsk[k], ctl + CTL_CELLS, sizeof(cellsk[k]), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(rangesk[k], ctl + CTL_RANGES, sizeof(rangesk[k]), cudaMemcpyDeviceToHost, s));
    if (e->trace)
      CUDA_TRY(cudaMemcpyAsync(tracek[k], ctl + CTL_TRACE, sizeof(tracek[k]), cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  e->stats.n_trace = 0;
  if (e->trace) {
    // Per class (and the rerun): earliest block start and latest warp end
    // over the call's runs, in ms from the call's earliest start.
    unsigned long long t0 = ~0ull;
    unsigned long long st0[NCLASS_MAX + 1], en[NCLASS_MAX + 1];
    for (int c = 0; c <= NCLASS_MAX; ++c) {
      st0[c] = ~0ull;
      en[c] = 0;
      for (int k = 0; k < nblk; ++k) {
        if (!tracek[k][2 * c + 1]) continue;
        st0[c] = std::min(st0[c], ~tracek[k][2 * c]);
        en[c] = std::max(en[c], tracek[k][2 * c + 1]);
      }
      if (en[c]) t0 = std::min(t0, st0[c]);
    }
    for (int c = 0; c <= NCLASS_MAX && e->stats.n_trace < IPUMA_MAX_TIMED; ++c) {
      if (!en[c]) continue;
      const int i = e->stats.n_trace++;
      e->stats.trace_kind[i] = c < kNumClasses ? kClasses[c].kind : IPUMA_KERNEL_S32_RERUN;
      e->stats.trace_start_ms[i] = (double)(st0[c] - t0) * 1e-6;
      e->stats.trace_end_ms[i] = (double)(en[c] - t0) * 1e-6;
      e->stats.trace_cells[i] = (int64_t)cells_of(cellsk, nblk, c < kNumClasses ? c : CELLS_RERUN);
    }
  }
  for (int k = 0; k < nblk; ++k) {
    if (!st.error) st.error = stk[k].error;
    st.overflow_count += stk[k].overflow_count;
    for (int c = 0; c < NCELLS; ++c) cells[c] += cellsk[k][c];
  }
  e->stats.overflow_reruns = st.overflow_count;
  // Pairs the binning sent to the s32 and hybrid classes ({start, count}
  // list ranges per class).
  e->stats.s32_pairs = 0;
  for (int k = 0; k < nblk; ++k)
    e->stats.s32_pairs += (int64_t)rangesk[k][2 * kClsS32 + 1] + (int64_t)rangesk[k][2 * kClsHi + 1];
  e->stats.n_timed = e->n_timed;
  for (int k = 0; k < e->n_timed; ++k) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e->tev[2 * k], e->tev[2 * k + 1]);
    e->stats.timed_kind[k] = e->timed_kind[k];
    e->stats.timed_ms[k] = ms;
    const int c = e->timed_cls[k];
    e->stats.timed_cells[k] = (c >= 0 && c < NCELLS) ? (int64_t)cells[c] : 0;
  }
  e->n_timed = 0;
  if (st.error == ERR_LENGTH) return fail(IPUMA_ERR_TOO_LONG, "a pair exceeds the stated maximum length");
  if (st.error == ERR_RANGE)
    return fail(IPUMA_ERR_INVALID_ARG, "a pair lies outside the code array (negative or past n_codes)");
  if (st.error) return fail(IPUMA_ERR_DEVICE, "kernel status error %d", st.error);
  return IPUMA_OK;
}

int plain_k_for(int maxAB) {
  if (maxAB <= 128) return 4;
  if (maxAB <= 256) return 8;
  return 16;
}

// Launches the one-launch-per-batch kernel over a wire buffer on the device.
int run_plain_wire(ipuma_engine* e, const RunBufs& rb, cudaStream_t s, const int* d_inputs, long seqWordsPerTile,
                   long metaOffset, int maxBatches, int totalSlots, int maxB, int* d_results,
                   int* launches) {
  int rc;
  int* ctl = rb.ctl;
  DevStatus* st = reinterpret_cast<DevStatus*>(ctl + CTL_STATUS);
  const long rowsCap = std::max(1, maxB);
  const int K = plain_k_for(e->algo.max_ab);
  const bool s16 = e->plain_s16 && e->s16_ok;
  auto go = [&](auto kern, int smem) -> int {
    const int grid = occupancy_grid(e, kern, smem);
    const long warps = (long)grid * kWarpsPerBlock;
    int r;
    if ((r = rb.scratch->ensure(sizeof(int2) * 2 * rowsCap * warps, s))) return r;
    if ((r = timed_begin(e, s, s16 ? IPUMA_KERNEL_PLAIN_S16 : IPUMA_KERNEL_PLAIN, CELLS_WIRE))) return r;
    kern<<<grid, kThreads, smem, s>>>(e->sc, e->d_sim.as<int8_t>(), d_inputs, seqWordsPerTile,
                                      metaOffset, maxBatches, totalSlots, rb.scratch->as<int2>(),
                                      rowsCap, d_results, st);
    CUDA_TRY(cudaGetLastError());
    return timed_end(e, s);
  };
  if (s16) {
    if (K == 4) rc = go(k_plain16<4>, smem_for<Lane16, 4, 32>(e));
    else if (K == 8) rc = go(k_plain16<8>, smem_for<Lane16, 8, 32>(e));
    else rc = go(k_plain16<16>, smem_for<Lane16, 16, 32>(e));
  } else {
    if (K == 4) rc = go(k_plain<4>, smem_for<LaneS32, 4, 32>(e));
    else if (K == 8) rc = go(k_plain<8>, smem_for<LaneS32, 8, 32>(e));
    else rc = go(k_plain<16>, smem_for<LaneS32, 16, 32>(e));
  }
  *launches += 1;
  return rc;
}

int validate_algo(const ipuma_algo_config* a) {
  if (a->tiles_used < 0 || a->max_batches < 0 || a->bufsize < 0 || a->max_ab < 0)
    return fail(IPUMA_ERR_INVALID_ARG, "negative size in IPUAlgoConfig");
  if (a->transmission_programs != 1 && a->transmission_programs != 0)
    return fail(IPUMA_ERR_INVALID_ARG, "transmissionPrograms other than 1 is not supported");
  return IPUMA_OK;
}

// ---------------------------------------------------------------------------
// Autotuner.  The class choice (pair_key) models a pair's time in kernel
// class c as strips * ((|B| + lanes) * width * slot_ps[c] + strip_ps[c]).
// The two rates per class depend on the GPU and on the alphabet (profile
// size, occupancy), so they are measured: a synthetic batch of related pairs
// per class at one strip of 1024 rows and at eight strips of 128 rows, every
// pair forced through that class, gives two equations for the two unknowns.
// Results are kept per process (by GPU, alphabet and gaps) and optionally in
// a cache file of "key<TAB>slot_ps...<TAB>strip_ps..." lines.
// ---------------------------------------------------------------------------

// The s32 class is not tuned (it is chosen by the overflow rules, not by
// cost); for the GPU shares of concurrent launches it is modelled as the
// widest s16x2 class with one pair per lane group instead of two.
void set_s32_rates(ipuma_engine* e) {
  e->slot_ps[kClsS32] = 2.f * e->slot_ps[kClsWidest];
  e->strip_ps[kClsS32] = 2.f * e->strip_ps[kClsWidest];
  // Hybrid class: between the two; modelled like s32 (its pairs' later
  // strips run there).
  e->slot_ps[kClsHi] = e->slot_ps[kClsS32];
  e->strip_ps[kClsHi] = e->strip_ps[kClsS32];
  // Strip teams run the widest class's strips (plus the waits of a
  // pipeline that fills and drains once per item: modelled in pair_key).
  e->slot_ps[kClsTeam] = e->slot_ps[kClsWidest];
  e->strip_ps[kClsTeam] = e->strip_ps[kClsWidest];
}

void set_default_rates(ipuma_engine* e) {
  // Measured on B200 with the nucleic-acid alphabet (uniform related pairs).
  const float slot[kNumS16] = {0.385f, 0.286f, 0.263f, 0.25f, 0.3125f, 0.3125f, 0.3f,  0.33f, 0.27f, 0.25f, 0.36f,
                               0.31f,  0.28f,  0.26f,  0.25f, 0.25f,   0.3f,    0.29f, 0.27f, 0.26f, 0.25f};
  for (int c = 0; c < kNumS16; ++c) {
    e->slot_ps[c] = slot[c];
    e->strip_ps[c] = 0.f;
  }
  set_s32_rates(e);
  e->tuned = false;
  e->tune_source = "defaults";
}

std::mutex g_tune_mu;
std::map<std::string, std::vector<float>> g_tune_cache;

std::string tune_key(const ipuma_engine* e) {
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, e->device);
  char buf[512];
  // The rates are those of the engine's kernels, which differ by mode: a
  // full alignment (forward + reverse pass) takes longer per cell.
  snprintf(buf, sizeof(buf), "%s|sm%d%d|M=%d|sim=%d|gI=%d|gE=%d|fwd=%d|v7", prop.name, prop.major, prop.minor, e->M,
           e->sw.similarity, e->sw.gap_init, e->sw.gap_extend, e->sc.forwardOnly);
  for (char* c = buf; *c; ++c)
    if (*c == '\t' || *c == '\n') *c = ' ';
  return buf;
}

void apply_rates(ipuma_engine* e, const std::vector<float>& v, const char* source) {
  for (int c = 0; c < kNumS16; ++c) {
    e->slot_ps[c] = v[c];
    e->strip_ps[c] = v[kNumS16 + c];
  }
  set_s32_rates(e);
  e->tuned = true;
  e->tune_source = source;
}

bool load_cache_file(const char* path, const std::string& key, std::vector<float>& v) {
  if (!path || !*path) return false;
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    char* tab = strchr(line, '\t');
    if (!tab) continue;
    *tab = 0;
    if (key != line) continue;
    std::vector<float> vals;
    for (char* p = tab + 1; *p;) {
      char* end = nullptr;
      const float x = strtof(p, &end);
      if (end == p) {
        ++p;
        continue;
      }
      vals.push_back(x);
      p = end;
    }
    if ((int)vals.size() == 2 * kNumS16) {
      v = vals;
      found = true;
    }
  }
  fclose(f);
  return found;
}

void append_cache_file(const char* path, const std::string& key, const std::vector<float>& v) {
  if (!path || !*path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s\t", key.c_str());
  for (int c = 0; c < kNumS16; ++c) fprintf(f, "%s%.6g", c ? "," : "", v[c]);
  fprintf(f, "\t");
  for (int c = 0; c < kNumS16; ++c) fprintf(f, "%s%.6g", c ? "," : "", v[kNumS16 + c]);
  fprintf(f, "\n");
  fclose(f);
}

// Device time (ms) of the class-`cls` launch for n synthetic pairs.
int time_class(ipuma_engine* e, int cls, int n, int alen, int blen, const DevBuf& letters, int nletters,
               uint32_t seed, float* ms) {
  cudaStream_t s = e->stream;
  int rc;
  const size_t bytes = (size_t)n * (alen + blen);
  if ((rc = e->d_codes.ensure(bytes, s))) return rc;
  if ((rc = e->d_pairs.ensure(sizeof(PairDesc) * (size_t)n, s))) return rc;
  if ((rc = e->d_res.ensure(sizeof(int) * 3 * (size_t)n, s))) return rc;
  const int gb = (int)std::min<size_t>((bytes + 255) / 256, (size_t)e->nsm * 16);
  k_synth_pairs<<<gb, 256, 0, s>>>(e->d_codes.as<uint8_t>(), e->d_pairs.as<PairDesc>(), n, alen, blen,
                                   letters.as<uint8_t>(), nletters, seed);
  CUDA_TRY(cudaGetLastError());
  const int savedK = e->tile_k, savedT = e->time_launches;
  e->tile_k = cls + 1;
  e->time_launches = 1;
  int* out = e->d_res.as<int>();
  *ms = -1.f;
  for (int rep = 0; rep < 2 && rc == IPUMA_OK; ++rep) {
    int launches = 0;
    if ((rc = reset_ctl(e, s))) break;
    if ((rc = run_batched(e, main_bufs(e), s, e->d_codes.as<uint8_t>(), bytes, 8, e->d_pairs.as<PairDesc>(), n, alen,
                          blen,
                          out, out + n,
                          out + 2 * n, &launches)))
      break;
    if ((rc = check_status(e, s))) break;
    for (int k = 0; k < e->stats.n_timed; ++k)
      if (e->timed_cls[k] == cls) *ms = (float)e->stats.timed_ms[k];
  }
  e->tile_k = savedK;
  e->time_launches = savedT;
  return rc;
}

int run_autotune(ipuma_engine* e, const char* cache_path) {
  const std::string key = tune_key(e);
  std::vector<float> v;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      apply_rates(e, it->second, "process cache");
      return IPUMA_OK;
    }
  }
  if (load_cache_file(cache_path, key, v)) {
    apply_rates(e, v, "cache file");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = v;
    return IPUMA_OK;
  }
  if (!e->fast_ok || !e->s16_ok) return IPUMA_OK;  // nothing to choose between
  // Letters of the alphabet that real sequences use.
  std::vector<uint8_t> letters;
  if (e->sw.datatype == IPUMA_DT_NUCLEIC_ACID) {
    letters = {1, 2, 3, 4};
  } else {
    for (int x = 0; x < std::min(20, e->M); ++x) letters.push_back((uint8_t)x);
  }
  DevBuf dl;
  int rc;
  if ((rc = dl.ensure(letters.size(), e->stream))) return rc;
  CUDA_TRY(cudaMemcpy(dl.p, letters.data(), letters.size(), cudaMemcpyHostToDevice));
  v.assign(2 * kNumS16, 0.f);
  for (int c = 0; c < kNumS16 && rc == IPUMA_OK; ++c) {
    const int W = kClasses[c].width, L = kClasses[c].lanes;
    // Pairs per warp item; the per-thread class keeps 64 pairs per warp and
    // far more pairs resident, so two rounds of items suffice there.
    const int perItem = L > 0 ? (32 / L) * 2 : 64;
    const int rounds = L > 0 ? 6 : 2;
    int grid = 1;
    switch (c) {
      case 0: grid = batched_grid<Lane16, 4, 16>(e, e->M); break;
      case 1: grid = batched_grid<Lane16, 8, 16>(e, e->M); break;
      case 2: grid = batched_grid<Lane16, 12, 16>(e, e->M); break;
      case 3: grid = batched_grid<Lane16, 16, 16>(e, e->M); break;
      case 4: grid = batched_grid<Lane16, 12, 32>(e, e->M); break;
      case 5: grid = batched_grid<Lane16, 16, 32>(e, e->M); break;
      case 7: grid = batched_grid<Lane16, 6, 16>(e, e->M); break;
      case 8: grid = batched_grid<Lane16, 10, 16>(e, e->M); break;
      case 9: grid = batched_grid<Lane16, 14, 16>(e, e->M); break;
      case 10: grid = batched_grid<Lane16, 5, 16>(e, e->M); break;
      case 11: grid = batched_grid<Lane16, 7, 16>(e, e->M); break;
      case 12: grid = batched_grid<Lane16, 9, 16>(e, e->M); break;
      case 13: grid = batched_grid<Lane16, 11, 16>(e, e->M); break;
      case 14: grid = batched_grid<Lane16, 13, 16>(e, e->M); break;
      case 15: grid = batched_grid<Lane16, 15, 16>(e, e->M); break;
      case 16: grid = batched_grid<Lane16, 8, 8>(e, e->M); break;
      case 17: grid = batched_grid<Lane16, 10, 8>(e, e->M); break;
      case 18: grid = batched_grid<Lane16, 12, 8>(e, e->M); break;
      case 19: grid = batched_grid<Lane16, 14, 8>(e, e->M); break;
      case 20: grid = batched_grid<Lane16, 16, 8>(e, e->M); break;
      default: grid = (int)(thread_threads<16>(e) / kThreads); break;
    }
    const int minPairs = grid * kWarpsPerBlock * perItem * rounds;
    // (strips, rows) of the two calibration batches.  The per-thread class
    // passes a boundary column through global memory at every strip, so
    // its shapes have several strips and a boundary working set larger
    // than L2, as real batches do.
    const int shapes[2][2] = {{1, 1024}, {8, 128}};
    const int thr_shapes[2][2] = {{4, 1024}, {16, 512}};
    double tpp[2] = {0, 0};
    for (int sh = 0; sh < 2 && rc == IPUMA_OK; ++sh) {
      const int* shp = L > 0 ? shapes[sh] : thr_shapes[sh];
      const int alen = shp[0] * W, blen = shp[1];
      const int n = std::max(minPairs, (int)std::min(2.0e6, 1.5e9 / ((double)alen * blen)));
      float ms = -1.f;
      rc = time_class(e, c, n, alen, blen, dl, (int)letters.size(), 0x5eed0000u + 16 * c + sh, &ms);
      tpp[sh] = ms > 0 ? ms * 1e9 / n : 0;  // ps per pair
    }
    // tpp = strips * ((rows + L) * W * slot + strip)
    const int* s1 = L > 0 ? shapes[0] : thr_shapes[0];
    const int* s2 = L > 0 ? shapes[1] : thr_shapes[1];
    const double a1 = (double)s1[0] * (s1[1] + L) * W, a2 = (double)s2[0] * (s2[1] + L) * W;
    const double b1 = s1[0], b2 = s2[0];
    const double det = a1 * b2 - a2 * b1;
    double slot = (tpp[0] * b2 - tpp[1] * b1) / det;
    double strip = (a1 * tpp[1] - a2 * tpp[0]) / det;
    if (slot <= 0) slot = tpp[0] / a1;
    if (strip < 0) strip = 0;
    v[c] = (float)slot;
    v[kNumS16 + c] = (float)strip;
  }
  dl.release();
  if (rc) return rc;
  apply_rates(e, v, "measured");
  append_cache_file(cache_path, key, v);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = v;
  return IPUMA_OK;
}

int maybe_autotune(ipuma_engine* e) {
  if (e->tuned || !e->autotune) return IPUMA_OK;
  const char* path = getenv("IPUMA_TUNE_CACHE");
  return run_autotune(e, path);
}

// Byte ranges of the code array one chunk of pairs reads: its A range and
// its B range (empty pairs read nothing).
struct ChunkSpan {
  size_t lo[2] = {SIZE_MAX, SIZE_MAX};
  size_t hi[2] = {0, 0};
};

// Adds [lo, hi) to the sorted disjoint list `have` and appends the parts
// that were missing to `todo`.
void take_range(std::vector<std::pair<size_t, size_t>>& have, size_t lo, size_t hi,
                std::vector<std::pair<size_t, size_t>>& todo) {
  if (lo >= hi) return;
  size_t cur = lo;
  for (const auto& r : have) {
    if (r.second <= cur) continue;
    if (r.first >= hi) break;
    if (r.first > cur) todo.emplace_back(cur, r.first);
    cur = std::max(cur, r.second);
    if (cur >= hi) break;
  }
  if (cur < hi) todo.emplace_back(cur, hi);
  have.emplace_back(lo, hi);
  std::sort(have.begin(), have.end());
  std::vector<std::pair<size_t, size_t>> merged;
  for (const auto& r : have) {
    if (!merged.empty() && r.first <= merged.back().second)
      merged.back().second = std::max(merged.back().second, r.second);
    else
      merged.push_back(r);
  }
  have.swap(merged);
}

int chunk_count(const ipuma_engine* e, int32_t n, size_t n_codes) {
  // The exact kernel's row scratch is one engine buffer: its runs cannot
  // overlap on two streams.
  if (!e->fast_ok) return 1;
  if (e->chunks > 0) return std::min<int>(std::min(e->chunks, kMaxChunks), std::max(1, n));
  if (n < 2 * kChunkMinPairs || n_codes < kChunkMinBytes) return 1;
  return std::min(kMaxChunks, std::max(2, (n + kChunkPairs / 2) / kChunkPairs));
}

// Bounds check of pairs [lo, hi) (the kernels trust the descriptors), with
// their maxima, cells and the code ranges each chunk's pairs read.
struct PairScan {
  int32_t bad = -1;  // first pair outside the code array
  int maxA = 0, maxB = 0;
  int64_t cells = 0;
  ChunkSpan span[kMaxChunks];
};

void scan_pairs(const ipuma_pair* pairs, size_t n_codes, int32_t lo, int32_t hi, const int32_t* cbeg,
                int nch, PairScan& r) {
  // Chunk by chunk, branch-free over the pairs (local accumulators); a
  // chunk part with a bad pair is scanned again for the first one.
  for (int k = 0; k < nch; ++k) {
    const int32_t b0 = std::max(lo, cbeg[k]), b1 = std::min(hi, cbeg[k + 1]);
    if (b0 >= b1) continue;
    int maxA = r.maxA, maxB = r.maxB;
    int64_t cells = 0;
    uint64_t alo = UINT64_MAX, ahi = 0, blo = UINT64_MAX, bhi = 0;
    bool ok = true;
    for (int32_t p = b0; p < b1; ++p) {
      const ipuma_pair d = pairs[p];
      const uint64_t ae = (uint64_t)d.a_off + (uint64_t)(uint32_t)d.a_len;
      const uint64_t be = (uint64_t)d.b_off + (uint64_t)(uint32_t)d.b_len;
      ok &= (d.a_len >= 0) & (d.b_len >= 0) & (d.a_off >= 0) & (d.b_off >= 0) & (ae <= n_codes) & (be <= n_codes);
      maxA = std::max(maxA, d.a_len);
      maxB = std::max(maxB, d.b_len);
      cells += (int64_t)d.a_len * d.b_len;
      const bool used = (d.a_len > 0) & (d.b_len > 0);  // empty pairs read nothing
      alo = std::min(alo, used ? (uint64_t)d.a_off : UINT64_MAX);
      ahi = std::max(ahi, used ? ae : 0);
      blo = std::min(blo, used ? (uint64_t)d.b_off : UINT64_MAX);
      bhi = std::max(bhi, used ? be : 0);
    }
    if (!ok) {
      for (int32_t p = b0; p < b1; ++p) {
        const ipuma_pair& d = pairs[p];
        if (d.a_len < 0 || d.b_len < 0 || d.a_off < 0 || d.b_off < 0 ||
            (size_t)d.a_off + (size_t)d.a_len > n_codes || (size_t)d.b_off + (size_t)d.b_len > n_codes) {
          r.bad = p;
          return;
        }
      }
    }
    r.maxA = maxA;
    r.maxB = maxB;
    r.cells += cells;
    ChunkSpan& sp = r.span[k];
    sp.lo[0] = std::min(sp.lo[0], (size_t)alo);
    sp.hi[0] = std::max(sp.hi[0], (size_t)ahi);
    sp.lo[1] = std::min(sp.lo[1], (size_t)blo);
    sp.hi[1] = std::max(sp.hi[1], (size_t)bhi);
  }
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Bounds check of a wire buffer's Meta (the kernels trust offsets and
// lengths) with the maxima, the cells and the last slot holding any
// non-zero Meta word.
struct MetaScan {
  long bad = -1;  // first slot pointing outside its tile
  int maxA = 0, maxB = 0;
  int64_t cells = 0;
  long last = -1;
};

void scan_meta(const int32_t* meta, long lo, long hi, long tileBytes, MetaScan& r) {
  for (long g = lo; g < hi; ++g) {
    const int32_t al = meta[4 * g], ao = meta[4 * g + 1], bl = meta[4 * g + 2], bo = meta[4 * g + 3];
    if ((al | ao | bl | bo) != 0) r.last = g;
    if (al == 0 || bl == 0) continue;
    if (al < 0 || bl < 0 || ao < 0 || bo < 0 || (long)ao + al > tileBytes || (long)bo + bl > tileBytes) {
      r.bad = g;
      return;
    }
    r.maxA = std::max(r.maxA, (int)al);
    r.maxB = std::max(r.maxB, (int)bl);
    r.cells += (int64_t)al * bl;
  }
}

// Scans all slots, on several host threads for large buffers.
MetaScan scan_wire(const int32_t* meta, long totalSlots, long tileBytes) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nthr = (int)std::max<long>(1, std::min<long>({(long)kValidateMaxThreads, (long)hw,
                                                          totalSlots / (2 * kValidatePairsPerThread)}));
  std::vector<MetaScan> part(nthr);
  std::vector<std::thread> pool;
  for (int t = 1; t < nthr; ++t)
    pool.emplace_back(scan_meta, meta, totalSlots * t / nthr, totalSlots * (t + 1) / nthr, tileBytes,
                      std::ref(part[t]));
  scan_meta(meta, 0, totalSlots / nthr, tileBytes, part[0]);
  for (auto& th : pool) th.join();
  MetaScan r;
  for (const auto& p : part) {
    if (p.bad >= 0 && r.bad < 0) r.bad = p.bad;
    r.maxA = std::max(r.maxA, p.maxA);
    r.maxB = std::max(r.maxB, p.maxB);
    r.cells += p.cells;
    r.last = std::max(r.last, p.last);
  }
  return r;
}

// The buffers and stream of wire set k: 0 = the engine's main buffers on
// `stream`, 1 = the second set on `wstream1`.  `rb.ctl` is valid once
// `ctl` holds a control block.
struct WireSet {
  DevBuf *inputs, *results, *pairs, *ctl;
  RunBufs rb;
  cudaStream_t s;
};

WireSet wire_set(ipuma_engine* e, int k) {
  if (k == 0) return WireSet{&e->d_inputs, &e->d_wres, &e->d_pairs, &e->d_ctl, main_bufs(e), e->stream};
  WireBufs& w = e->w1;
  return WireSet{&w.inputs, &w.results, &w.pairs, &w.ctl,
                 RunBufs{w.ctl.as<int>(), &w.scratch, &w.list, &w.ovf, &w.flag, 2}, e->wstream1};
}

int take_event(ipuma_engine* e, cudaEvent_t* ev) {
  if (!e->free_events.empty()) {
    *ev = e->free_events.back();
    e->free_events.pop_back();
    return IPUMA_OK;
  }
  CUDA_TRY(cudaEventCreate(ev));
  return IPUMA_OK;
}

int take_status(ipuma_engine* e, JobStatus** out) {
  if (e->free_status.empty()) {
    constexpr int kSlots = 64;
    void* block = nullptr;
    CUDA_TRY(cudaHostAlloc(&block, sizeof(JobStatus) * kSlots, cudaHostAllocPortable));
    e->pinned_blocks.push_back(block);
    for (int i = 0; i < kSlots; ++i) e->free_status.push_back(static_cast<JobStatus*>(block) + i);
  }
  *out = e->free_status.back();
  e->free_status.pop_back();
  return IPUMA_OK;
}

// Pinned staging of at least `bytes`, reused when a free one is at most
// twice that size.
int take_staging(ipuma_engine* e, size_t bytes, int32_t** out, size_t* cap) {
  auto it = e->free_staging.lower_bound(bytes);
  if (it != e->free_staging.end() && it->first <= 2 * bytes) {
    *out = it->second;
    *cap = it->first;
    e->free_staging.erase(it);
    return IPUMA_OK;
  }
  void* p = nullptr;
  CUDA_TRY(cudaHostAlloc(&p, bytes, cudaHostAllocPortable));
  *out = static_cast<int32_t*>(p);
  *cap = bytes;
  return IPUMA_OK;
}

constexpr size_t kMaxFreeStaging = 8;

// Returns a finished (or abandoned) job's events, status slot and staging
// to the engine's pools.  Caller holds e->mu.
void recycle_job(ipuma_engine* e, Job& j) {
  for (auto& ev : j.ev)
    if (ev) e->free_events.push_back(ev);
  if (j.done) e->free_events.push_back(j.done);
  if (j.status) e->free_status.push_back(j.status);
  if (j.staged) {
    if (e->free_staging.size() < kMaxFreeStaging) e->free_staging.emplace(j.staged_bytes, j.staged);
    else cudaFreeHost(j.staged);
  }
  j = Job{};
}

}  // namespace

extern "C" {

const char* ipuma_last_error(void) { return g_last_error.c_str(); }

const char* ipuma_version(void) { return "ipuma-b200 0.1 (sm_100a)"; }

int32_t ipuma_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int ipuma_host_alloc(size_t bytes, void** out) {
  if (!out) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (bytes == 0) return IPUMA_OK;
  cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return fail(IPUMA_ERR_NO_MEMORY, "cudaHostAlloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  return IPUMA_OK;
}

void ipuma_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

int ipuma_encode(int32_t datatype, const char* s, size_t n, uint8_t* out) {
  if ((!s || !out) && n) return fail(IPUMA_ERR_INVALID_ARG, "null pointer");
  if (datatype < 0 || datatype > 2) return fail(IPUMA_ERR_INVALID_ARG, "invalid datatype %d", datatype);
  const auto enc = swatlib::getEncoder(static_cast<swatlib::DataType>(datatype));
  const auto table = enc.getCodeTable();
  for (size_t i = 0; i < n; ++i) {
    const unsigned char c = static_cast<unsigned char>(s[i]);
    const uint8_t v = c < 127 ? table[c] : enc.get_terminator();
    if (datatype == IPUMA_DT_NUCLEIC_ACID && v == 16)
      return fail(IPUMA_ERR_BAD_SEQUENCE, "character 0x%02x at %zu is not a nucleic-acid code", c, i);
    out[i] = v;
  }
  return IPUMA_OK;
}

int ipuma_pack_codes(const uint8_t* codes, size_t n, int32_t bits, uint8_t* out) {
  if ((!codes || !out) && n) return fail(IPUMA_ERR_INVALID_ARG, "null pointer");
  if (bits != 2 && bits != 4 && bits != 5) return fail(IPUMA_ERR_INVALID_ARG, "bits must be 2, 4 or 5, not %d", bits);
  // Groups of 8 residues fill `bits` whole bytes of the little-endian bit
  // stream; the last group writes only the bytes its residues reach.
  const size_t groups = (n + 7) / 8;
  const size_t bytes = (n * (size_t)bits + 7) / 8;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nthr = (int)std::max<size_t>(1, std::min<size_t>({(size_t)16, (size_t)hw, groups >> 20}));
  std::vector<size_t> bad(nthr, SIZE_MAX);
  auto work = [&](int t) {
    const size_t g0 = groups * t / nthr, g1 = groups * (t + 1) / nthr;
    for (size_t g = g0; g < g1; ++g) {
      uint64_t v = 0;
      for (size_t q = 0; q < 8; ++q) {
        const size_t i = 8 * g + q;
        if (i >= n) break;
        // 2 bits: code - 1 for A, T, C, G (1..4); 4 and 5 bits: the code.
        const uint32_t x = (bits == 2) ? (uint32_t)codes[i] - 1u : codes[i];
        if (x >= (1u << bits)) {
          bad[t] = i;
          return;
        }
        v |= (uint64_t)x << (bits * q);
      }
      for (size_t k = 0; k < (size_t)bits && (size_t)bits * g + k < bytes; ++k)
        out[(size_t)bits * g + k] = (uint8_t)(v >> (8 * k));
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthr; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  for (size_t b : bad)
    if (b != SIZE_MAX)
      return fail(IPUMA_ERR_BAD_SEQUENCE, "code %u at %zu does not fit %d bits", codes[b], b, bits);
  return IPUMA_OK;
}

int ipuma_select_matrix(int32_t similarity, int32_t match, int32_t mismatch, int32_t ambiguity,
                        int8_t* out, size_t out_cap, int32_t* m, int32_t* n) {
  try {
    auto mat = swatlib::selectMatrix(static_cast<swatlib::Similarity>(similarity), (int8_t)match,
                                     (int8_t)mismatch, (int8_t)ambiguity);
    auto [mm, nn] = mat.shape();
    if (m) *m = (int32_t)mm;
    if (n) *n = (int32_t)nn;
    if (out) {
      if (out_cap < mm * nn) return fail(IPUMA_ERR_INVALID_ARG, "output too small");
      std::memcpy(out, mat.data(), mm * nn);
    }
  } catch (const std::exception& ex) {
    return fail(IPUMA_ERR_INVALID_ARG, "%s", ex.what());
  }
  return IPUMA_OK;
}

int64_t ipuma_input_buffer_words(const ipuma_algo_config* a) {
  if (!a) return 0;
  const int64_t bufWords = (a->bufsize + 3) / 4;
  return (int64_t)a->tiles_used * bufWords + (int64_t)a->tiles_used * a->max_batches * 4;
}

int ipuma_gpu_create(const ipuma_sw_config* sw, const ipuma_algo_config* algo, int32_t device,
                     ipuma_engine** out) {
  if (!sw || !algo || !out) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  int rc;
  if ((rc = validate_algo(algo))) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(IPUMA_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(IPUMA_ERR_NO_DEVICE, "device %d out of range", device);
  std::unique_ptr<ipuma_engine> e(new ipuma_engine());
  e->device = device;
  e->sw = *sw;
  e->algo = *algo;
  CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(IPUMA_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                device, prop.major, prop.minor);
  e->nsm = prop.multiProcessorCount;
  e->smem_optin = (int)prop.sharedMemPerBlockOptin;
  CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  for (auto& ev : e->ev) CUDA_TRY(cudaEventCreate(&ev));
  // Class streams and their fork/join events (created here: no stream or
  // event is created while a stream is being captured).
  CUDA_TRY(cudaEventCreateWithFlags(&e->fork_ev, cudaEventDisableTiming));
  for (int c = 0; c < NCLASS_MAX; ++c) {
    CUDA_TRY(cudaStreamCreateWithFlags(&e->cls_stream[c], cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->join_ev[c], cudaEventDisableTiming));
  }

  // Substitution matrix (swatlib::selectMatrix, ipu_batch_affine.cpp:390).
  int32_t m = 0, n = 0;
  int8_t buf[32 * 32];
  if ((rc = ipuma_select_matrix(sw->similarity, sw->match_value, sw->mismatch_value,
                                sw->ambiguity_value, buf, sizeof(buf), &m, &n)))
    return rc;
  e->M = m;
  e->sim.assign(buf, buf + m * n);
  e->maxSub = 0;
  int minSub = 0;
  for (auto v : e->sim) {
    e->maxSub = std::max<int>(e->maxSub, v);
    minSub = std::min<int>(minSub, v);
  }
  if ((rc = e->d_sim.ensure(e->sim.size(), e->stream))) return rc;
  CUDA_TRY(cudaMemcpy(e->d_sim.p, e->sim.data(), e->sim.size(), cudaMemcpyHostToDevice));

  const int gI = sw->gap_init, gE = sw->gap_extend;
  e->sc.gI = gI;
  e->sc.gE = gE;
  e->sc.gIgE = gI + gE;
  e->sc.M = m;
  e->sc.forwardOnly = algo->forward_only ? 1 : 0;
  // Wavefront kernels: padding cells must stay below real ones (gI+gE < 0,
  // gE <= 0) and profile entries sim - (gI+gE) must fit int8.
  e->fast_ok = (gI + gE < 0) && (gE <= 0) && (e->maxSub - (gI + gE) <= 127) &&
               (minSub - (gI + gE) >= -128) && (gI + gE > -1000) && (gE > -1000);
  // 16-bit lanes: H <= limit guarantees no halfword leaves its range (signed
  // halves of the wavefront and per-thread classes: 32767 - maxSub; the
  // biased halves of the hybrid class: 65535 - bias - maxSub).  The binning
  // pass sends pairs whose main diagonal may pass the signed limit to the
  // hybrid class.
  e->sc.s16Limit = 32767 - std::max(0, e->maxSub);
  e->sc.u16Limit = 65535 - LaneB16x2::BIAS - std::max(0, e->maxSub);
  e->sc.maxSub = std::max(0, e->maxSub);
  e->sc.bits = 8;
  e->sc.P = m;
  e->sc.pshift = 0;
  e->s16_ok = e->fast_ok;
  e->s16_max_len = e->maxSub > 0 ? (e->sc.s16Limit / e->maxSub) : (1 << 30);
  set_default_rates(e.get());
  max_batched_groups(e.get());  // warm the grid cache
  thread_threads<16>(e.get());
  *out = e.release();
  return IPUMA_OK;
}

void ipuma_gpu_destroy(ipuma_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->wstream1) cudaStreamSynchronize(e->wstream1);
  for (auto& kv : e->jobs) recycle_job(e, kv.second);
  for (auto ev : e->free_events) cudaEventDestroy(ev);
  for (auto& kv : e->free_staging) cudaFreeHost(kv.second);
  for (void* p : e->pinned_blocks) cudaFreeHost(p);
  if (e->stream2) cudaStreamSynchronize(e->stream2);
  if (e->copy_stream) cudaStreamSynchronize(e->copy_stream);
  for (auto* b : {&e->d_sim, &e->d_codes, &e->d_packed, &e->d_pairs, &e->d_list, &e->d_res, &e->d_scratch, &e->d_cf,
                  &e->d_ovf, &e->d_ctl, &e->d_inputs, &e->d_wres, &e->d_flag, &e->x_list, &e->x_scratch,
                  &e->x_ovf, &e->x_flag, &e->w1.inputs, &e->w1.results, &e->w1.pairs, &e->w1.ctl, &e->w1.list,
                  &e->w1.scratch, &e->w1.ovf, &e->w1.flag})
    b->release();
  for (auto& ev : e->cev)
    if (ev) cudaEventDestroy(ev);
  for (int c = 0; c < NCLASS_MAX; ++c) {
    if (e->cls_stream[c]) cudaStreamSynchronize(e->cls_stream[c]);
    if (e->cls_stream[c]) cudaStreamDestroy(e->cls_stream[c]);
    if (e->join_ev[c]) cudaEventDestroy(e->join_ev[c]);
  }
  if (e->fork_ev) cudaEventDestroy(e->fork_ev);
  if (e->stream2) cudaStreamDestroy(e->stream2);
  if (e->wstream1) cudaStreamDestroy(e->wstream1);
  if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
  for (auto& ev : e->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : e->tev)
    if (ev) cudaEventDestroy(ev);
  for (auto& kv : e->graphs_cache) cudaGraphExecDestroy(kv.second);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

int ipuma_gpu_set_option(ipuma_engine* e, const char* name, int64_t value) {
  if (!e || !name) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  const std::string k(name);
  if (k == "scheduler") {
    if (value != 0 && value != 1) return fail(IPUMA_ERR_INVALID_ARG, "scheduler must be 0 or 1");
    e->scheduler = (int)value;
  } else if (k == "plain_lanes") {
    if (value != 16 && value != 32) return fail(IPUMA_ERR_INVALID_ARG, "plain_lanes must be 16 or 32");
    e->plain_s16 = value == 16 ? 1 : 0;
  } else if (k == "trace") {
    e->trace = value ? 1 : 0;
  } else if (k == "graphs") {
    e->graphs = value ? 1 : 0;
  } else if (k == "long_a") {
    if (value < 0) return fail(IPUMA_ERR_INVALID_ARG, "long_a must be >= 0");
    e->long_a = (int)std::min<int64_t>(value, 1 << 30);
  } else if (k == "autotune") {
    e->autotune = value ? 1 : 0;
  } else if (k == "time_launches") {
    e->time_launches = value ? 1 : 0;
  } else if (k == "latency_share") {
    if (value < 1 || value > 100000) return fail(IPUMA_ERR_INVALID_ARG, "latency_share is in per mille, 1..100000");
    e->latency_share = (float)value / 1000.f;
  } else if (k == "hybrid") {
    e->hybrid = value ? 1 : 0;
  } else if (k == "concurrent") {
    if (value < 0 || value > 3) return fail(IPUMA_ERR_INVALID_ARG, "concurrent must be 0, 1, 2 or 3");
    e->concurrent = (int)value;
  } else if (k == "thread_class") {
    e->thread_class = value ? 1 : 0;
  } else if (k == "chunks") {
    if (value < 0 || value > kMaxChunks)
      return fail(IPUMA_ERR_INVALID_ARG, "chunks must be 0 (automatic) .. %d", kMaxChunks);
    e->chunks = (int)value;
  } else if (k == "tile_k") {
    if (value < 0 || (value > kNumS16 && value != kClsTeam + 1))
      return fail(IPUMA_ERR_INVALID_ARG, "tile_k must be 0 (automatic), a kernel class 1..%d or %d (strip teams)",
                  kNumS16, kClsTeam + 1);
    e->tile_k = (int)value;
  } else if (k == "team_warps") {
    if (value != 0 && (value < 2 || value > kTeamMaxWarps))
      return fail(IPUMA_ERR_INVALID_ARG, "team_warps must be 0 (no strip teams) or 2..%d", kTeamMaxWarps);
    e->team_warps = (int)value;
  } else {
    return fail(IPUMA_ERR_INVALID_ARG, "unknown option '%s'", name);
  }
  return IPUMA_OK;
}

int ipuma_gpu_autotune(ipuma_engine* e, const char* cache_path) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  std::lock_guard<std::mutex> lk(e->mu);
  CUDA_TRY(cudaSetDevice(e->device));
  if (!cache_path) cache_path = getenv("IPUMA_TUNE_CACHE");
  return run_autotune(e, cache_path);
}

int ipuma_gpu_tuning(ipuma_engine* e, char* buf, size_t cap) {
  if (!e || !buf || cap == 0) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  std::string j = "{\"source\": \"" + e->tune_source + "\", \"classes\": [";
  char tmp[256];
  for (int c = 0; c < kNumS16; ++c) {
    snprintf(tmp, sizeof(tmp), "%s{\"lanes\": %d, \"k\": %d, \"slot_ps\": %.5g, \"strip_ps\": %.5g}", c ? ", " : "",
             kClasses[c].lanes, kClasses[c].k, e->slot_ps[c], e->strip_ps[c]);
    j += tmp;
  }
  j += "]}";
  if (j.size() + 1 > cap) return fail(IPUMA_ERR_INVALID_ARG, "buffer too small (%zu bytes needed)", j.size() + 1);
  memcpy(buf, j.c_str(), j.size() + 1);
  return IPUMA_OK;
}

int ipuma_gpu_last_stats(ipuma_engine* e, ipuma_stats* out) {
  if (!e || !out) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  *out = e->stats;
  return IPUMA_OK;
}

int ipuma_gpu_reserve(ipuma_engine* e, int32_t n, int32_t max_a_len, int32_t max_b_len) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  if (n < 0 || max_a_len < 0 || max_b_len < 0 || max_a_len > 65535 || max_b_len > 65535)
    return fail(IPUMA_ERR_INVALID_ARG, "bad reservation (%d pairs, %d x %d)", n, max_a_len, max_b_len);
  std::lock_guard<std::mutex> lk(e->mu);
  CUDA_TRY(cudaSetDevice(e->device));
  int rc;
  if ((rc = reserve_batched(e, e->stream, n, max_a_len, max_b_len))) return rc;
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return IPUMA_OK;
}

// Checks a packed-code request: the width fits the engine's alphabet and
// the per-thread class (byte codes only) is not forced.
static int check_bits(const ipuma_engine* e, int bits) {
  if (bits != 2 && bits != 4 && bits != 5) return fail(IPUMA_ERR_INVALID_ARG, "bits must be 2, 4 or 5, not %d", bits);
  // 2-bit codes are A, T, C, G = nucleic-acid codes 1..4.
  if (bits == 2 && e->sw.datatype != IPUMA_DT_NUCLEIC_ACID)
    return fail(IPUMA_ERR_INVALID_ARG, "2-bit codes are nucleic-acid codes");
  // 4 and 5 bits hold codes 0 .. 2^bits - 1: the alphabet must fit (2 bits
  // hold A, C, G, T of the nucleic-acid alphabet).
  if (bits != 2 && e->M > (1 << bits))
    return fail(IPUMA_ERR_INVALID_ARG, "%d-bit codes hold at most %d letters (this alphabet has %d)", bits, 1 << bits,
                e->M);
  if (e->tile_k == kClsThread + 1)
    return fail(IPUMA_ERR_INVALID_ARG, "the per-thread class (tile_k %d) reads one byte per residue", e->tile_k);
  return IPUMA_OK;
}

// Body of ipuma_gpu_compare_device (bits = 8) and
// ipuma_gpu_compare_device_packed (bits = 2, 4, 5).
static int compare_dev(ipuma_engine* e, const uint8_t* d_codes, size_t n_codes, int bits,
                       const ipuma_pair* d_pairs, int32_t n, int32_t max_a_len, int32_t max_b_len,
                       int32_t* d_score, int32_t* d_arange, int32_t* d_brange, void* stream) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  if (n < 0) return fail(IPUMA_ERR_INVALID_ARG, "negative pair count");
  if (n > 0 && (!d_codes || !d_pairs || !d_score || !d_arange || !d_brange))
    return fail(IPUMA_ERR_INVALID_ARG, "null buffer");
  if (bits != 8) {
    int rcb = check_bits(e, bits);
    if (rcb) return rcb;
    if (reinterpret_cast<uintptr_t>(d_codes) & 3)
      return fail(IPUMA_ERR_INVALID_ARG, "packed codes must start 4-byte aligned");
  }
  std::lock_guard<std::mutex> lk(e->mu);
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : e->stream;
  int rc;
  if ((rc = maybe_autotune(e))) return rc;
  e->stats = ipuma_stats{};
  int launches = 0;
  if (e->graphs && !e->time_launches && e->fast_ok && n > 0) {
    // Replay (or capture, then replay) the whole pipeline as one graph.
    if ((rc = reserve_batched(e, s, n, max_a_len, max_b_len))) return rc;
    const std::vector<uint64_t> key = {(uint64_t)(uintptr_t)d_codes, (uint64_t)n_codes, (uint64_t)bits,
                                       (uint64_t)(uintptr_t)d_pairs,
                                       (uint64_t)n,
                                       (uint64_t)max_a_len, (uint64_t)max_b_len, (uint64_t)(uintptr_t)d_score,
                                       (uint64_t)(uintptr_t)d_arange, (uint64_t)(uintptr_t)d_brange,
                                       (uint64_t)(uintptr_t)e->d_scratch.p, (uint64_t)e->d_scratch.cap,
                                       (uint64_t)(uintptr_t)e->d_list.p, (uint64_t)(uintptr_t)e->d_ctl.p,
                                       (uint64_t)(uintptr_t)e->d_ovf.p, (uint64_t)(uintptr_t)e->d_flag.p,
                                       (uint64_t)e->tile_k, (uint64_t)e->long_a, (uint64_t)e->thread_class,
                                       (uint64_t)e->concurrent, (uint64_t)e->hybrid, (uint64_t)e->trace,
                                       (uint64_t)(e->latency_share * 1e6f), (uint64_t)e->team_warps};
    auto it = e->graphs_cache.find(key);
    if (it == e->graphs_cache.end()) {
      if (e->graphs_cache.size() >= 16) {
        cudaGraphExecDestroy(e->graphs_cache.begin()->second);
        e->graphs_cache.erase(e->graphs_cache.begin());
      }
      cudaGraph_t g = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int crc = reset_ctl(e, s);
      if (!crc)
        crc = run_batched(e, main_bufs(e), s, d_codes, n_codes, bits, reinterpret_cast<const PairDesc*>(d_pairs), n,
                          max_a_len, max_b_len,
                          d_score, d_arange, d_brange, &launches);
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (crc) {
        if (g) cudaGraphDestroy(g);
        return crc;
      }
      if (ce != cudaSuccess) return fail(IPUMA_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
      cudaGraphExec_t ex = nullptr;
      ce = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return fail(IPUMA_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ce));
      it = e->graphs_cache.emplace(key, ex).first;
      e->graph_launches[ex] = launches;
    }
    launches = e->graph_launches[it->second];
    CUDA_TRY(cudaEventRecord(e->ev[1], s));
    CUDA_TRY(cudaGraphLaunch(it->second, s));
    e->stats.used_graph = 1;
  } else {
    if ((rc = reset_ctl(e, s))) return rc;
    CUDA_TRY(cudaEventRecord(e->ev[1], s));
    rc = run_batched(e, main_bufs(e), s, d_codes, n_codes, bits, reinterpret_cast<const PairDesc*>(d_pairs), n,
                     max_a_len,
                     max_b_len, d_score, d_arange, d_brange, &launches);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(e->ev[2], s));
  if ((rc = check_status(e, s))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, e->ev[1], e->ev[2]);
  e->stats.kernel_ms = ms;
  e->stats.total_ms = ms;
  e->stats.pairs = n;
  e->stats.launches = launches;
  return IPUMA_OK;
}

// Host-buffer compare of ipuma_gpu_compare (bits = 8: one byte per
// residue) and ipuma_gpu_compare_packed (bits = 4 or 2: two or four
// residues per byte, expanded on the device after each upload).
static int compare_host(ipuma_engine* e, const uint8_t* codes, size_t n_codes, int bits, const ipuma_pair* pairs,
                        int32_t n, int32_t* score, int32_t* arange, int32_t* brange) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  if (n < 0) return fail(IPUMA_ERR_INVALID_ARG, "negative pair count");
  if (n == 0) return IPUMA_OK;
  if (!codes || !pairs || !score || !arange || !brange) return fail(IPUMA_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(e->mu);
  const auto h0 = std::chrono::steady_clock::now();
  const int nch = e->time_launches ? 1 : chunk_count(e, n, n_codes);
  // Host-side bounds check of every pair (the kernels trust the
  // descriptors), with the code ranges each chunk of pairs reads; large
  // batches are checked on several threads.
  int32_t cbeg[kMaxChunks + 1];
  // Chunk k+1's upload overlaps chunk k's kernels, so chunks grow (weights
  // 1, 5.67, 11.3, ...: 6 %, 31 %, 63 % for three chunks) and the first one,
  // whose upload no kernel hides, is the smallest.  (1M DNA pairs, 2-bit
  // codes, B200: 16.9-17.5 ms per call against 17.7-18.0 with 10/30/60 %
  // chunks and 19.1-19.5 with equal ones.)
  {
    double w[kMaxChunks], tot = 0, acc = 0;
    for (int k = 0; k < nch; ++k) tot += (w[k] = k == 0 ? 1.0 : 5.67 * k);
    cbeg[0] = 0;
    for (int k = 1; k <= nch; ++k) {
      acc += w[k - 1];
      cbeg[k] = k == nch ? n : (int32_t)((double)n * acc / tot);
    }
  }
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nthr = std::max(1, std::min({kValidateMaxThreads, hw, n / kValidatePairsPerThread}));
  std::vector<PairScan> part(nthr);
  {
    std::vector<std::thread> pool;
    for (int t = 1; t < nthr; ++t)
      pool.emplace_back(scan_pairs, pairs, n_codes, (int32_t)((int64_t)n * t / nthr),
                        (int32_t)((int64_t)n * (t + 1) / nthr), cbeg, nch, std::ref(part[t]));
    scan_pairs(pairs, n_codes, 0, (int32_t)((int64_t)n / nthr), cbeg, nch, part[0]);
    for (auto& th : pool) th.join();
  }
  int maxA = 0, maxB = 0;
  int64_t cells = 0;
  ChunkSpan span[kMaxChunks];
  for (const PairScan& r : part) {
    if (r.bad >= 0) return fail(IPUMA_ERR_INVALID_ARG, "pair %d lies outside the code array", r.bad);
    maxA = std::max(maxA, r.maxA);
    maxB = std::max(maxB, r.maxB);
    cells += r.cells;
    for (int k = 0; k < nch; ++k)
      for (int q = 0; q < 2; ++q) {
        span[k].lo[q] = std::min(span[k].lo[q], r.span[k].lo[q]);
        span[k].hi[q] = std::max(span[k].hi[q], r.span[k].hi[q]);
      }
  }
  if (maxA > 65535 || maxB > 65535)
    return fail(IPUMA_ERR_TOO_LONG, "sequence longer than 65535 (ranges are uint16)");
  const auto h1 = std::chrono::steady_clock::now();
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t s = e->stream;
  int rc;
  if ((rc = maybe_autotune(e))) return rc;
  // Packed codes stay packed on the device (the kernels decode them, code_at):
  // the buffer covers the host's bytes rounded up to a word plus one word.
  const size_t hostBytes = bits == 8 ? n_codes : (n_codes * (size_t)bits + 7) / 8;
  DevBuf& dcodes = bits == 8 ? e->d_codes : e->d_packed;
  if ((rc = dcodes.ensure(std::max<size_t>(((hostBytes + 3) & ~(size_t)3) + 8, 16), s))) return rc;
  if ((rc = e->d_pairs.ensure(sizeof(ipuma_pair) * (size_t)n, s))) return rc;
  if ((rc = e->d_res.ensure(sizeof(int32_t) * 3 * (size_t)n, s))) return rc;
  // Puts the bytes holding residues [lo, hi) on the device, on stream `us`.
  auto upload = [&](size_t lo, size_t hi, cudaStream_t us) -> int {
    if (lo >= hi) return IPUMA_OK;
    const size_t blo = lo * (size_t)bits / 8, bhi = std::min(hostBytes, (hi * (size_t)bits + 7) / 8);
    CUDA_TRY(cudaMemcpyAsync(dcodes.as<uint8_t>() + blo, codes + blo, bhi - blo, cudaMemcpyHostToDevice, us));
    return IPUMA_OK;
  };
  e->stats = ipuma_stats{};
  int launches = 0;
  int32_t* d_score = e->d_res.as<int32_t>();
  int32_t* d_ar = d_score + n;
  int32_t* d_br = d_ar + n;
  if (nch == 1) {
    if ((rc = reset_ctl(e, s))) return rc;
    CUDA_TRY(cudaEventRecord(e->ev[0], s));
    if ((rc = upload(0, n_codes, s))) return rc;
    CUDA_TRY(cudaMemcpyAsync(e->d_pairs.p, pairs, sizeof(ipuma_pair) * (size_t)n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaEventRecord(e->ev[1], s));
    rc = run_batched(e, main_bufs(e), s, dcodes.as<uint8_t>(), n_codes, bits, e->d_pairs.as<PairDesc>(), n, maxA, maxB,
                     d_score, d_ar, d_br, &launches);
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(e->ev[2], s));
    CUDA_TRY(cudaMemcpyAsync(score, d_score, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(arange, d_ar, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(brange, d_br, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaEventRecord(e->ev[3], s));
    if ((rc = check_status(e, s))) return rc;
  } else {
    // Chunked: chunk k's code ranges and descriptors go up on copy_stream
    // while earlier chunks run; runs alternate between two streams with
    // their own buffer sets, so one chunk's launches fill the tail of the
    // previous one's.  Results come back per chunk when the host buffers
    // are pinned (pageable copies would block the issuing thread), else
    // once at the end.
    if (!e->stream2) CUDA_TRY(cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking));
    if (!e->copy_stream) CUDA_TRY(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
    for (auto& ev : e->cev)
      if (!ev) CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    int nmax = 0;
    for (int k = 0; k < nch; ++k) nmax = std::max(nmax, cbeg[k + 1] - cbeg[k]);
    const RunBufs rb1{nullptr, &e->x_scratch, &e->x_list, &e->x_ovf, &e->x_flag, 2};
    if ((rc = e->d_ctl.ensure(sizeof(int) * CTL_INTS * (size_t)nch, s))) return rc;
    if ((rc = reserve_bufs(e, main_bufs(e), s, nmax, maxA, maxB))) return rc;
    if ((rc = reserve_bufs(e, rb1, s, nmax, maxA, maxB))) return rc;
    const bool pinned_out = is_pinned(score) && is_pinned(arange) && is_pinned(brange);
    cudaStream_t run_s[2] = {s, e->stream2};
    CUDA_TRY(cudaEventRecord(e->ev[0], s));
    CUDA_TRY(cudaMemsetAsync(e->d_ctl.p, 0, sizeof(int) * CTL_INTS * (size_t)nch, s));
    e->n_timed = 0;
    CUDA_TRY(cudaEventRecord(e->ev[1], s));
    CUDA_TRY(cudaStreamWaitEvent(e->stream2, e->ev[1], 0));
    CUDA_TRY(cudaStreamWaitEvent(e->copy_stream, e->ev[1], 0));
    std::vector<std::pair<size_t, size_t>> have, todo;
    for (int k = 0; k < nch; ++k) {
      const int32_t off = cbeg[k], nk = cbeg[k + 1] - cbeg[k];
      todo.clear();
      for (int r = 0; r < 2; ++r)
        if (span[k].lo[r] < span[k].hi[r]) take_range(have, span[k].lo[r], span[k].hi[r], todo);
      for (const auto& r : todo)
        if ((rc = upload(r.first, r.second, e->copy_stream))) return rc;
      CUDA_TRY(cudaMemcpyAsync(e->d_pairs.as<ipuma_pair>() + off, pairs + off, sizeof(ipuma_pair) * (size_t)nk,
                               cudaMemcpyHostToDevice, e->copy_stream));
      CUDA_TRY(cudaEventRecord(e->cev[k], e->copy_stream));
      cudaStream_t rs = run_s[k & 1];
      CUDA_TRY(cudaStreamWaitEvent(rs, e->cev[k], 0));
      RunBufs rb = (k & 1) ? rb1 : main_bufs(e);
      rb.ctl = e->d_ctl.as<int>() + (size_t)k * CTL_INTS;
      if ((rc = run_batched(e, rb, rs, dcodes.as<uint8_t>(), n_codes, bits, e->d_pairs.as<PairDesc>() + off, nk, maxA,
                            maxB,
                            d_score + off, d_ar + off, d_br + off, &launches)))
        return rc;
      if (pinned_out) {
        CUDA_TRY(cudaMemcpyAsync(score + off, d_score + off, sizeof(int32_t) * nk, cudaMemcpyDeviceToHost, rs));
        CUDA_TRY(cudaMemcpyAsync(arange + off, d_ar + off, sizeof(int32_t) * nk, cudaMemcpyDeviceToHost, rs));
        CUDA_TRY(cudaMemcpyAsync(brange + off, d_br + off, sizeof(int32_t) * nk, cudaMemcpyDeviceToHost, rs));
      }
    }
    CUDA_TRY(cudaEventRecord(e->cev[kMaxChunks], e->stream2));
    CUDA_TRY(cudaStreamWaitEvent(s, e->cev[kMaxChunks], 0));
    CUDA_TRY(cudaEventRecord(e->ev[2], s));
    if (!pinned_out) {
      CUDA_TRY(cudaMemcpyAsync(score, d_score, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaMemcpyAsync(arange, d_ar, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaMemcpyAsync(brange, d_br, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaEventRecord(e->ev[3], s));
    if ((rc = check_status(e, s, nch))) return rc;
  }
  float kms = 0, tms = 0;
  cudaEventElapsedTime(&kms, e->ev[1], e->ev[2]);
  cudaEventElapsedTime(&tms, e->ev[0], e->ev[3]);
  e->stats.kernel_ms = kms;
  e->stats.total_ms = tms;
  e->stats.cells = cells;
  e->stats.pairs = n;
  e->stats.launches = launches;
  e->stats.chunks = nch;
  e->stats.host_check_ms = std::chrono::duration<double, std::milli>(h1 - h0).count();
  e->stats.host_wall_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
  return IPUMA_OK;
}

int ipuma_gpu_compare(ipuma_engine* e, const uint8_t* codes, size_t n_codes, const ipuma_pair* pairs,
                      int32_t n, int32_t* score, int32_t* arange, int32_t* brange) {
  return compare_host(e, codes, n_codes, 8, pairs, n, score, arange, brange);
}

int ipuma_gpu_compare_packed(ipuma_engine* e, const uint8_t* packed, size_t n_codes, int32_t bits,
                             const ipuma_pair* pairs, int32_t n, int32_t* score, int32_t* arange,
                             int32_t* brange) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  int rc = check_bits(e, bits);
  if (rc) return rc;
  return compare_host(e, packed, n_codes, bits, pairs, n, score, arange, brange);
}

int ipuma_gpu_compare_device(ipuma_engine* e, const uint8_t* d_codes, size_t n_codes, const ipuma_pair* d_pairs,
                             int32_t n, int32_t max_a_len, int32_t max_b_len, int32_t* d_score, int32_t* d_arange,
                             int32_t* d_brange, void* stream) {
  return compare_dev(e, d_codes, n_codes, 8, d_pairs, n, max_a_len, max_b_len, d_score, d_arange, d_brange, stream);
}

int ipuma_gpu_compare_device_packed(ipuma_engine* e, const uint8_t* d_packed, size_t n_codes, int32_t bits,
                                    const ipuma_pair* d_pairs, int32_t n, int32_t max_a_len, int32_t max_b_len,
                                    int32_t* d_score, int32_t* d_arange, int32_t* d_brange, void* stream) {
  // Only packed widths here: 8 would read one byte per residue from a
  // buffer the caller sized for packed codes.
  if (bits != 2 && bits != 4 && bits != 5)
    return fail(IPUMA_ERR_INVALID_ARG, "bits must be 2, 4 or 5, not %d", bits);
  return compare_dev(e, d_packed, n_codes, bits, d_pairs, n, max_a_len, max_b_len, d_score, d_arange, d_brange,
                     stream);
}

// Launches the alignment work of a wire buffer already on the device
// (plain kernel or wire -> pair list -> batched pipeline).
static int launch_wire(ipuma_engine* e, DevBuf* pairs, const RunBufs& rb, cudaStream_t s, const int* d_in,
                       int* d_res, int maxA, int maxB, int* launches) {
  const ipuma_algo_config& a = e->algo;
  const long seqWordsPerTile = (a.bufsize + 3) / 4;
  const long metaOffset = (long)a.tiles_used * seqWordsPerTile;
  const long totalSlots = (long)a.tiles_used * a.max_batches;
  int rc;
  if (totalSlots <= 0) return IPUMA_OK;
  if (e->scheduler == 1 && e->fast_ok) {
    return run_plain_wire(e, rb, s, d_in, seqWordsPerTile, metaOffset, a.max_batches, (int)totalSlots, maxB,
                          d_res, launches);
  }
  if ((rc = pairs->ensure(sizeof(PairDesc) * totalSlots, s))) return rc;
  const int gb = (int)std::min<long>((totalSlots + 255) / 256, e->nsm * 8);
  k_wire_to_pairs<<<gb, 256, 0, s>>>(d_in, seqWordsPerTile, metaOffset, a.max_batches, (int)totalSlots,
                                     pairs->as<PairDesc>());
  CUDA_TRY(cudaGetLastError());
  *launches += 1;
  // Pair offsets are absolute within the tiles' sequence words.
  return run_batched(e, rb, s, reinterpret_cast<const uint8_t*>(d_in), (size_t)metaOffset * 4, 8,
                     pairs->as<PairDesc>(), (int)totalSlots,
                     maxA, maxB, d_res, d_res + totalSlots, d_res + 2 * totalSlots, launches);
}

static int check_wire_sizes(const ipuma_algo_config& a, size_t n_inputs, size_t n_results) {
  const long totalSlots = (long)a.tiles_used * a.max_batches;
  if ((int64_t)n_inputs != ipuma_input_buffer_words(&a))
    return fail(IPUMA_ERR_INVALID_ARG, "input buffer has %zu words, config needs %lld", n_inputs,
                (long long)ipuma_input_buffer_words(&a));
  if ((long)n_results != 3 * totalSlots) return fail(IPUMA_ERR_INVALID_ARG, "Results buffer not 3 aligned.");
  if (totalSlots > 0x7fffffffL) return fail(IPUMA_ERR_INVALID_ARG, "too many comparison slots");
  return IPUMA_OK;
}

// Wire-buffer path of run/submit: validates Meta, then enqueues on the next
// wire set's stream the upload of the tiles in use (trailing tiles whose
// Meta is all zero are not copied: their Meta is cleared on the device),
// the kernels, the status copy and the results copy (straight into pinned
// results, else into pinned staging that the join copies out).
static int enqueue_buffer(ipuma_engine* e, const int32_t* inputs, size_t n_inputs, int32_t* results,
                          size_t n_results, Job& j) {
  const ipuma_algo_config& a = e->algo;
  const long seqWordsPerTile = (a.bufsize + 3) / 4;
  const long metaOffset = (long)a.tiles_used * seqWordsPerTile;
  const long totalSlots = (long)a.tiles_used * a.max_batches;
  int rc;
  if ((rc = check_wire_sizes(a, n_inputs, n_results))) return rc;
  const MetaScan m = scan_wire(inputs + metaOffset, totalSlots, seqWordsPerTile * 4);
  if (m.bad >= 0) return fail(IPUMA_ERR_INVALID_ARG, "Meta slot %ld points outside its tile", m.bad);
  if (m.maxA > 65535 || m.maxB > 65535)
    return fail(IPUMA_ERR_TOO_LONG, "sequence longer than 65535 (ranges are uint16)");

  // The second set needs the wavefront kernels (the exact kernel's row
  // scratch is one engine buffer); per-launch timing stays on one stream.
  const int k = (e->fast_ok && !e->time_launches) ? (int)(e->wire_jobs & 1) : 0;
  e->wire_jobs++;
  if (k == 1 && !e->wstream1) CUDA_TRY(cudaStreamCreateWithFlags(&e->wstream1, cudaStreamNonBlocking));
  WireSet w = wire_set(e, k);
  cudaStream_t s = w.s;
  if ((rc = w.inputs->ensure(sizeof(int32_t) * std::max<size_t>(n_inputs, 1), s))) return rc;
  if ((rc = w.results->ensure(sizeof(int32_t) * std::max<size_t>(n_results, 1), s))) return rc;
  if ((rc = w.ctl->ensure(sizeof(int) * CTL_INTS, s))) return rc;
  w.rb.ctl = w.ctl->as<int>();
  for (auto& ev : j.ev)
    if ((rc = take_event(e, &ev))) return rc;
  if ((rc = take_event(e, &j.done))) return rc;
  if ((rc = take_status(e, &j.status))) return rc;
  j.results = results;
  j.n_results = n_results;
  const size_t resBytes = sizeof(int32_t) * n_results;
  if (resBytes && !is_pinned(results) && (rc = take_staging(e, resBytes, &j.staged, &j.staged_bytes)))
    return rc;

  CUDA_TRY(cudaEventRecord(j.ev[0], s));
  CUDA_TRY(cudaMemsetAsync(w.rb.ctl, 0, sizeof(int) * CTL_INTS, s));
  e->n_timed = 0;
  int32_t* d_in = w.inputs->as<int32_t>();
  const long usedTiles = m.last < 0 ? 0 : m.last / std::max(1, a.max_batches) + 1;
  const size_t seqWords = (size_t)usedTiles * seqWordsPerTile;
  const size_t metaWords = (size_t)usedTiles * a.max_batches * 4;
  const size_t metaTotal = (size_t)totalSlots * 4;
  if (seqWords)
    CUDA_TRY(cudaMemcpyAsync(d_in, inputs, sizeof(int32_t) * seqWords, cudaMemcpyHostToDevice, s));
  if (metaWords)
    CUDA_TRY(cudaMemcpyAsync(d_in + metaOffset, inputs + metaOffset, sizeof(int32_t) * metaWords,
                             cudaMemcpyHostToDevice, s));
  if (metaTotal > metaWords)
    CUDA_TRY(cudaMemsetAsync(d_in + metaOffset + metaWords, 0, sizeof(int32_t) * (metaTotal - metaWords), s));
  CUDA_TRY(cudaEventRecord(j.ev[1], s));
  int launches = 1;
  int* d_res = w.results->as<int>();
  if ((rc = launch_wire(e, w.pairs, w.rb, s, d_in, d_res, m.maxA, m.maxB, &launches))) return rc;
  CUDA_TRY(cudaEventRecord(j.ev[2], s));
  CUDA_TRY(cudaMemcpyAsync(&j.status->st, w.rb.ctl + CTL_STATUS, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
  if (resBytes)
    CUDA_TRY(cudaMemcpyAsync(j.staged ? j.staged : results, d_res, resBytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaEventRecord(j.done, s));
  j.stats.cells = m.cells;
  j.stats.pairs = totalSlots;
  j.stats.launches = launches;
  j.stats.chunks = 1;
  return IPUMA_OK;
}

int ipuma_gpu_run_buffer_device(ipuma_engine* e, const int32_t* d_inputs, size_t n_inputs, int32_t* d_results,
                                size_t n_results, void* stream) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  if ((n_inputs && !d_inputs) || (n_results && !d_results)) return fail(IPUMA_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(e->mu);
  CUDA_TRY(cudaSetDevice(e->device));
  const ipuma_algo_config& a = e->algo;
  int rc;
  if ((rc = check_wire_sizes(a, n_inputs, n_results))) return rc;
  if (e->scheduler == 0 && (rc = maybe_autotune(e))) return rc;
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : e->stream;
  const long seqWordsPerTile = (a.bufsize + 3) / 4;
  const long metaOffset = (long)a.tiles_used * seqWordsPerTile;
  const long totalSlots = (long)a.tiles_used * a.max_batches;
  e->stats = ipuma_stats{};
  if ((rc = reset_ctl(e, s))) return rc;
  int* ctl = e->d_ctl.as<int>();
  auto* cells = reinterpret_cast<unsigned long long*>(ctl + CTL_CELLS);
  // Device-side validation of Meta; the host needs maxA/maxB for scratch.
  const int gb = (int)std::max<long>(1, std::min<long>((totalSlots + 255) / 256, e->nsm * 8));
  k_wire_check<<<gb, 256, 0, s>>>(d_inputs, metaOffset, seqWordsPerTile * 4, (int)totalSlots, ctl + CTL_INFO,
                                  cells + CELLS_WIRE);
  CUDA_TRY(cudaGetLastError());
  int info[3] = {0, 0, 0};
  unsigned long long wcells = 0;
  CUDA_TRY(cudaMemcpyAsync(info, ctl + CTL_INFO, sizeof(info), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&wcells, cells + CELLS_WIRE, sizeof(wcells), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (info[2]) return fail(IPUMA_ERR_INVALID_ARG, "%d Meta slots point outside their tile", info[2]);
  if (info[0] > 65535 || info[1] > 65535)
    return fail(IPUMA_ERR_TOO_LONG, "sequence longer than 65535 (ranges are uint16)");
  int launches = 1;
  CUDA_TRY(cudaEventRecord(e->ev[1], s));
  if ((rc = launch_wire(e, &e->d_pairs, main_bufs(e), s, d_inputs, d_results, info[0], info[1], &launches)))
    return rc;
  CUDA_TRY(cudaEventRecord(e->ev[2], s));
  if ((rc = check_status(e, s))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, e->ev[1], e->ev[2]);
  e->stats.kernel_ms = ms;
  e->stats.total_ms = ms;
  e->stats.cells = (int64_t)wcells;
  e->stats.pairs = totalSlots;
  e->stats.launches = launches;
  return IPUMA_OK;
}

int ipuma_gpu_run_buffer(ipuma_engine* e, const int32_t* inputs, size_t n_inputs, int32_t* results,
                         size_t n_results) {
  uint64_t job = 0;
  int rc = ipuma_gpu_submit_buffer(e, inputs, n_inputs, results, n_results, &job);
  if (rc) return rc;
  return ipuma_gpu_join(e, job, -1);
}

int ipuma_gpu_submit_buffer(ipuma_engine* e, const int32_t* inputs, size_t n_inputs,
                            int32_t* results, size_t n_results, uint64_t* job) {
  if (!e || !job) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  if ((n_inputs && !inputs) || (n_results && !results)) return fail(IPUMA_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(e->mu);
  CUDA_TRY(cudaSetDevice(e->device));
  int rc;
  if (e->scheduler == 0 && (rc = maybe_autotune(e))) return rc;
  Job j;
  rc = enqueue_buffer(e, inputs, n_inputs, results, n_results, j);
  if (rc) {
    // Nothing of a failed submission is joined: wait for what it enqueued
    // before its resources go back to the pools.
    if (j.done || j.ev[0]) {
      cudaStreamSynchronize(e->stream);
      if (e->wstream1) cudaStreamSynchronize(e->wstream1);
    }
    recycle_job(e, j);
    return rc;
  }
  e->stats = j.stats;
  *job = e->next_job++;
  e->jobs[*job] = j;
  return IPUMA_OK;
}

int ipuma_gpu_poll(ipuma_engine* e, uint64_t job, int32_t* done) {
  if (!e || !done) return fail(IPUMA_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  auto it = e->jobs.find(job);
  if (it == e->jobs.end()) return fail(IPUMA_ERR_UNKNOWN_JOB, "unknown job %llu", (unsigned long long)job);
  cudaError_t q = cudaEventQuery(it->second.done);
  if (q == cudaSuccess) {
    *done = 1;
  } else if (q == cudaErrorNotReady) {
    *done = 0;
  } else {
    return fail(IPUMA_ERR_CUDA, "job %llu failed: %s", (unsigned long long)job, cudaGetErrorString(q));
  }
  return IPUMA_OK;
}

int ipuma_gpu_join_stats(ipuma_engine* e, uint64_t job, int64_t timeout_ms, ipuma_stats* out) {
  if (!e) return fail(IPUMA_ERR_INVALID_ARG, "null engine");
  cudaEvent_t ev;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job);
    if (it == e->jobs.end()) return fail(IPUMA_ERR_UNKNOWN_JOB, "unknown job %llu", (unsigned long long)job);
    ev = it->second.done;
  }
  CUDA_TRY(cudaSetDevice(e->device));
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) return fail(IPUMA_ERR_CUDA, "job failed: %s", cudaGetErrorString(q));
    if (timeout_ms >= 0 &&
        std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
      return fail(IPUMA_ERR_TIMEOUT, "job %llu not finished after %lld ms", (unsigned long long)job,
                  (long long)timeout_ms);
    if (timeout_ms < 0) {
      CUDA_TRY(cudaEventSynchronize(ev));
      break;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  Job j;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job);
    if (it == e->jobs.end()) return fail(IPUMA_ERR_UNKNOWN_JOB, "job %llu already joined", (unsigned long long)job);
    j = it->second;
    e->jobs.erase(it);
  }
  // Everything the job enqueued has finished: its staging, status and
  // events are only read here.
  if (j.staged) std::memcpy(j.results, j.staged, sizeof(int32_t) * j.n_results);
  float kms = 0, tms = 0;
  cudaEventElapsedTime(&kms, j.ev[1], j.ev[2]);
  cudaEventElapsedTime(&tms, j.ev[0], j.done);
  j.stats.kernel_ms = kms;
  j.stats.total_ms = tms;
  j.stats.overflow_reruns = j.status->st.overflow_count;
  const int err = j.status->st.error;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->stats = j.stats;
    if (out) *out = j.stats;
    recycle_job(e, j);
  }
  if (err == ERR_LENGTH) return fail(IPUMA_ERR_TOO_LONG, "a pair exceeds the stated maximum length");
  if (err) return fail(IPUMA_ERR_DEVICE, "kernel status error %d", err);
  return IPUMA_OK;
}

int ipuma_gpu_join(ipuma_engine* e, uint64_t job, int64_t timeout_ms) {
  return ipuma_gpu_join_stats(e, job, timeout_ms, nullptr);
}

}  // extern "C"
