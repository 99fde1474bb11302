// peak.cu -- measures the integer/DPX issue peak that bounds the alignment
// kernels: the instruction mix of one cell update of the wavefront classes
// (signed 16-bit halves, two cells per instruction)
//   1 x prmt (substitution bytes), 4 x viaddmax.s16x2 (F, Y with relu, E,
//   H), 1 x add.s16x2 (F term of Y), 1 x max.s16x2 (row maximum)
// (7 instructions = 14 lane-ops, two cells), run as independent chains by
// every thread of a full-occupancy grid.  Reported as lane-ops per second.
#include <cuda_runtime.h>

#include <cstdint>

#include "ipuma_b200.h"
#include "sw_device.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_int_peak(uint32_t seed, uint32_t* sink) {
  using T = ipuma_dev::Lane16;
  uint32_t e[kChains], f[kChains], h[kChains], w[kChains];
  const uint32_t g = T::splat(-1), go = T::splat(-2);
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    e[c] = seed ^ (threadIdx.x * 2654435761u) ^ c;
    f[c] = e[c] * 3u;
    h[c] = e[c] * 7u;
    w[c] = e[c] * 13u;
  }
  uint32_t rm = 0;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      const uint32_t sb = T::sub<1>(w[c], h[c]);          // prmt
      f[c] = T::addmax(f[c], g, h[c]);                    // F
      const uint32_t ft = T::add(f[c], go);                // F term of Y
      const uint32_t y = T::addmax_relu(h[c], sb, ft);     // Y
      e[c] = T::addmax(e[c], g, y);                       // E
      h[c] = T::addmax(e[c], go, y);                      // H
      rm = T::max2(rm, h[c]);                             // row maximum
    }
  }
  uint32_t acc = rm;
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc ^= e[c] ^ f[c] ^ h[c];
  if (acc == 0x12345678u) sink[threadIdx.x] = acc;  // keeps the work alive
}

}  // namespace

extern "C" int ipuma_measure_int_peak(int32_t device, double* lane_ops_per_s) {
  if (!lane_ops_per_s) return IPUMA_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return IPUMA_ERR_NO_DEVICE;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return IPUMA_ERR_CUDA;
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_int_peak, 256, 0);
  if (nb < 1) nb = 1;
  const int grid = nb * p.multiProcessorCount;
  uint32_t* sink = nullptr;
  if (cudaMalloc(&sink, 256 * sizeof(uint32_t)) != cudaSuccess) return IPUMA_ERR_NO_MEMORY;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_int_peak<<<grid, 256>>>(1u, sink);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(a);
    k_int_peak<<<grid, 256>>>(2u + r, sink);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (err != cudaSuccess) return IPUMA_ERR_CUDA;
  const double instr = (double)grid * 256 * kIters * kChains * 7.0;
  *lane_ops_per_s = instr * 2.0 / (best * 1e-3);
  return IPUMA_OK;
}
