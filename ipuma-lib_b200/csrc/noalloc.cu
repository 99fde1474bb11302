// noalloc.cu -- ipuma_gpu_compare_noalloc, the entry point that allocates
// no memory at all.
//
// Some callers cannot call cudaMalloc: host programs that hand every byte
// of device memory to their own pool (a framework's caching allocator that
// reserved the GPU up front) and forbid other allocations, or
// latency-critical paths that cannot afford the device-wide
// synchronisation cudaMalloc and cudaFree imply.  For them this entry point
// aligns pairs whose inputs and outputs the caller already holds in device
// memory, without an engine and without any allocation.
//
// It runs a variant of the s32 wavefront kernel (k_batched<LaneS32, 16, 32>):
// the one scratch buffer that kernel needs -- the last column of a
// 512-column strip, handed to the next strip for A longer than 512 -- lives
// in the file-scope array g_noalloc_scratch (16 MiB, held by every GPU that
// loads the library until the process exits), and the status word in
// g_noalloc_status.  The substitution matrix travels in the kernel
// parameters.  Pairs are taken in a static stride instead of from a queue.
//
// Host code must not use those arrays' names as device addresses: the first
// call on a device looks their addresses up with cudaGetSymbolAddress (with
// that device current) and caches them; that first call should therefore
// happen before any stream capture begins.  Every call shares the arrays and
// they keep the last call's contents: the status word is cleared at the
// start of each call; the scratch needs no clearing (each strip writes the
// rows the next strip reads).  Calls that overlap on the GPU (different
// streams, or host threads racing) share the scratch and race; issue them
// one after another.
//
// Each pair descriptor is checked on the device before any code is read:
// a negative offset or length, or a sequence reaching past n_codes, sets
// the status to a range error; |A| > 65535 or |B| > max_b_len sets it to a
// length error; such pairs and empty ones get a zero result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "errors.h"
#include "ipuma_b200.h"
#include "sw_kernels.cuh"

using namespace ipuma_dev;

namespace {

constexpr long kScratchInt2 = 2L << 20;  // 2 Mi int2 = 16 MiB
constexpr int kMaxLen = 65535;           // ranges are uint16
constexpr int kWarps = 2;                // warps per block
constexpr int kMaxDevices = 64;

__device__ __align__(256) int2 g_noalloc_scratch[kScratchInt2];
__device__ __align__(256) DevStatus g_noalloc_status;

struct SimParam {
  int8_t v[32 * 32];
};

template <int K>
__global__ void __launch_bounds__(64) k_noalloc(SwConst sc, SimParam sim, const uint8_t* __restrict__ codes,
                                                long long n_codes, const PairDesc* __restrict__ pairs, int n,
                                                int2* scratch, long rowsCap, DevStatus* status, int* score,
                                                int* arange, int* brange) {
  using T = LaneS32;
  using L = SmemLayout<T, K, 32>;
  extern __shared__ __align__(16) uint8_t smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int8_t* s_simp = reinterpret_cast<int8_t*>(smem);
  uint8_t* wbase = smem + L::simp_bytes(sc.M) + wib * L::warp_bytes(sc.P);
  uint8_t* s_prof = wbase;
  uint16_t* s_bring = reinterpret_cast<uint16_t*>(wbase + L::prof_bytes(sc.P));
  const int M = sc.M;
  for (int k = threadIdx.x; k < M * (M + 1); k += blockDim.x) {
    const int a = k / (M + 1), x = k % (M + 1);
    s_simp[k] = (x < M) ? sim.v[a * M + x] : (int8_t)SUB_PAD;
  }
  __syncthreads();
  const long gw = (long)blockIdx.x * kWarps + wib;
  const long nw = (long)gridDim.x * kWarps;
  int2* scr = scratch + gw * 2 * rowsCap;
  for (long p = gw; p < n; p += nw) {
    const PairDesc d = pairs[p];
    const int state = pair_state(d, n_codes, kMaxLen, (int)rowsCap);
    if (state != PAIR_OK) {
      if (lane == 0) {
        report_pair(state, status);
        score[p] = 0;
        arange[p] = 0;
        brange[p] = 0;
      }
      continue;
    }
    const long long a0[1] = {d.a_off};
    const long long b0[1] = {d.b_off};
    const int al[1] = {d.a_len}, bl[1] = {d.b_len};
    Best fw[1], rv[1];
    bool ovf[1];
    align_pairs<T, K, 32>(sc, s_prof, s_simp, s_bring, codes, a0, b0, al, bl, scr, rowsCap, fw, rv, ovf);
    if (lane == 0) write_result(sc, fw[0], rv[0], score, arange, brange, p);
  }
}

struct DeviceSymbols {
  bool ready = false;
  int2* scratch = nullptr;
  DevStatus* status = nullptr;
  int nsm = 0;
};
DeviceSymbols g_symbols[kMaxDevices];
std::mutex g_symbols_mutex;

using ipuma_internal::fail;

}  // namespace

extern "C" int ipuma_gpu_compare_noalloc(const ipuma_sw_config* sw, int32_t forward_only,
                                         const uint8_t* d_codes, size_t n_codes, const ipuma_pair* d_pairs,
                                         int32_t n, int32_t max_b_len, int32_t* d_score, int32_t* d_arange,
                                         int32_t* d_brange, void* stream) {
  if (!sw) return fail(IPUMA_ERR_INVALID_ARG, "null scoring configuration");
  if (n < 0) return fail(IPUMA_ERR_INVALID_ARG, "negative pair count");
  if (n == 0) return IPUMA_OK;
  if (!d_codes || !d_pairs || !d_score || !d_arange || !d_brange)
    return fail(IPUMA_ERR_INVALID_ARG, "null device buffer");
  if (max_b_len < 1 || max_b_len > kMaxLen)
    return fail(IPUMA_ERR_TOO_LONG, "max_b_len must be 1..65535 for the allocation-free entry point");
  const int gI = sw->gap_init, gE = sw->gap_extend;
  if (!(gI + gE < 0 && gE <= 0))
    return fail(IPUMA_ERR_INVALID_ARG,
                "the allocation-free entry point needs gap_init + gap_extend < 0 and gap_extend <= 0");
  int32_t m = 0, nn = 0;
  SimParam sim{};
  if (ipuma_select_matrix(sw->similarity, sw->match_value, sw->mismatch_value, sw->ambiguity_value, sim.v,
                          sizeof(sim.v), &m, &nn) != IPUMA_OK)
    return fail(IPUMA_ERR_INVALID_ARG, "invalid similarity");

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(IPUMA_ERR_NO_DEVICE, "no current CUDA device");
  DeviceSymbols* ds = &g_symbols[dev];
  {
    std::lock_guard<std::mutex> lk(g_symbols_mutex);
    if (!ds->ready) {
      // Once per device, with that device current: device addresses of the
      // file-scope arrays (their host-side names are not device addresses).
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess)
        return fail(IPUMA_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed");
      ds->scratch = static_cast<int2*>(p);
      if (cudaGetSymbolAddress(&p, g_noalloc_status) != cudaSuccess)
        return fail(IPUMA_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_status) failed");
      ds->status = static_cast<DevStatus*>(p);
      cudaDeviceProp prop;
      if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return fail(IPUMA_ERR_CUDA, "device query failed");
      ds->nsm = prop.multiProcessorCount;
      ds->ready = true;
    }
  }

  SwConst sc{};
  sc.gI = gI;
  sc.gE = gE;
  sc.gIgE = gI + gE;
  sc.M = m;
  sc.forwardOnly = forward_only ? 1 : 0;
  sc.s16Limit = 32767;  // (16-bit lanes are not used here)
  sc.u16Limit = 32767;
  sc.bits = 8;  // one byte per residue
  sc.P = m;     // a profile row per letter
  sc.pshift = 0;
  // Warps that fit the static scratch at this row count (2 rows per B row).
  const long rowsCap = max_b_len;
  const long warpsFit = kScratchInt2 / (2 * rowsCap);
  // rowsCap <= 65535 leaves room for at least 16 warps, so `blocks` whole
  // blocks of kWarps warps never index past the array.
  const long warps = std::max<long>(kWarps, std::min<long>({warpsFit, (long)ds->nsm * 16, (long)n}));
  const int blocks = (int)(warps / kWarps);
  const int smem = SmemLayout<LaneS32, 16, 32>::total(m, m, kWarps);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(ds->status, 0, sizeof(DevStatus), s) != cudaSuccess)
    return fail(IPUMA_ERR_CUDA, "clearing the status word failed");
  k_noalloc<16><<<blocks, 32 * kWarps, smem, s>>>(sc, sim, d_codes, (long long)n_codes,
                                                   reinterpret_cast<const PairDesc*>(d_pairs), n, ds->scratch,
                                                   rowsCap, ds->status, d_score, d_arange, d_brange);
  if (cudaGetLastError() != cudaSuccess) return fail(IPUMA_ERR_CUDA, "kernel launch failed");
  int status = 0;
  if (cudaMemcpyAsync(&status, ds->status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return fail(IPUMA_ERR_CUDA, "reading the status word failed");
  if (status == ERR_LENGTH)
    return fail(IPUMA_ERR_TOO_LONG, "a pair's b_len exceeds max_b_len or its a_len exceeds 65535");
  if (status == ERR_RANGE)
    return fail(IPUMA_ERR_INVALID_ARG, "a pair lies outside the code array (negative or past n_codes)");
  if (status) return fail(IPUMA_ERR_DEVICE, "kernel reported an error");
  return IPUMA_OK;
}
