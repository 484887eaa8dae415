// probe.cu — the random-access ceiling of the GPU this library runs on.
//
// The search and resolve kernels are chains of dependent random reads of 32-byte (narrow
// Occ record, sampled-SA record) or 96-byte (wide Occ record) pieces of a table far larger
// than L2.  A streaming copy's bandwidth is not reachable by that pattern; this probe
// measures what is: every thread issues independent loads of `span` bytes (32, 64 or 96)
// at uniformly random span-aligned offsets of a buffer of several GB, 256-288 bytes of
// them in flight per thread, over a grid of resident threads on every SM.  No counterpart
// in the reference.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "hfm_internal.h"

namespace hfm {

__device__ __forceinline__ uint64_t probe_mix(uint64_t x) {      // splitmix64 step
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

template <int SPAN, int DEPTH>
__global__ void __launch_bounds__(256) k_probe_gather(const uint4* __restrict__ buf, uint64_t nspans, uint32_t rounds,
                                                      uint64_t seed, uint32_t* __restrict__ sink) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t st = probe_mix(seed ^ (tid * 0x2545f4914f6cdd1dull));
  uint32_t acc = 0;
  for (uint32_t r = 0; r < rounds; r++) {
    uint4 v[DEPTH][SPAN / 16];
#pragma unroll
    for (int d = 0; d < DEPTH; d++) {
      st = probe_mix(st);
      const uint4* p = buf + (st % nspans) * (SPAN / 16);      // last uint4 read: nspans * SPAN / 16 - 1
#pragma unroll
      for (int k = 0; k < SPAN / 16; k++) v[d][k] = __ldg(p + k);
    }
#pragma unroll
    for (int d = 0; d < DEPTH; d++)
#pragma unroll
      for (int k = 0; k < SPAN / 16; k++) acc ^= v[d][k].x ^ v[d][k].y ^ v[d][k].z ^ v[d][k].w;
  }
  if (acc == 0x9e3779b9u) sink[0] = acc;      // keeps the loads; practically never stores
}

}  // namespace hfm

using namespace hfm;

extern "C" int hfm_probe_gather(int device, uint64_t buffer_bytes, uint32_t span, float* gbs_out, float* ms_out) {
  if (!gbs_out || (span != 32 && span != 64 && span != 96))
    return set_error(HFM_E_ARG, "span must be 32, 64 or 96 and gbs_out set");
  if (buffer_bytes < (64ull << 20)) return set_error(HFM_E_ARG, "buffer_bytes below 64 MiB");
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return set_error(HFM_E_ARG, "device ordinal out of range"); }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  void* buf = nullptr;
  uint32_t* sink = nullptr;
  if (cudaMalloc(&buf, buffer_bytes) != cudaSuccess) { cudaGetLastError(); return set_error(HFM_E_OOM, "probe buffer"); }
  if (cudaMalloc(&sink, 16) != cudaSuccess) { cudaGetLastError(); cudaFree(buf); return set_error(HFM_E_OOM, "probe sink"); }
  cudaStream_t s;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaMemsetAsync(buf, 0x5a, buffer_bytes, s);
  const uint64_t nspans = buffer_bytes / span;
  const unsigned grid = (unsigned)sms * 8, block = 256;
  const uint32_t rounds = 64, depth = span == 32 ? 8 : span == 64 ? 4 : 3;   // 256-288 bytes in flight per thread
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0); cudaEventCreate(&e1);
  auto launch = [&](uint64_t seed) {
    if (span == 32) k_probe_gather<32, 8><<<grid, block, 0, s>>>((const uint4*)buf, nspans, rounds, seed, sink);
    else if (span == 64) k_probe_gather<64, 4><<<grid, block, 0, s>>>((const uint4*)buf, nspans, rounds, seed, sink);
    else k_probe_gather<96, 3><<<grid, block, 0, s>>>((const uint4*)buf, nspans, rounds, seed, sink);
  };
  launch(1);                                   // warm-up
  cudaEventRecord(e0, s);
  const int reps = 5;
  for (int r = 0; r < reps; r++) launch(100 + r);
  cudaEventRecord(e1, s);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (err == cudaSuccess) err = cudaGetLastError();
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  cudaFree(buf); cudaFree(sink);
  if (err != cudaSuccess) return set_error(HFM_E_CUDA, std::string("probe: ") + cudaGetErrorString(err));
  const double bytes = (double)reps * grid * block * rounds * depth * span;
  *gbs_out = (float)(bytes / (ms / 1e3) / 1e9);
  if (ms_out) *ms_out = ms / reps;
  return HFM_OK;
}
