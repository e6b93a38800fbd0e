// Random-read ceiling probe: the rate at which this GPU serves random 32-byte
// sector reads from a table larger than L2, the access pattern of every walk
// step. Two forms: independent reads (8 in flight per thread, the bandwidth
// ceiling) and dependent chains (each read's address comes from the previous
// read, one chain per thread, the form a walk step has).
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "engine.cuh"

namespace bingo {
namespace {

__device__ __forceinline__ uint32_t probe_hash(uint32_t x) { return mix32(x * 0x9E3779B9u + 0x7F4A7C15u); }

// table holds n_words 32-bit words; reads touch random sector-aligned words.
__global__ void k_probe_independent(const uint32_t* __restrict__ table, uint32_t sector_mask, uint32_t rounds,
                                    uint32_t* sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t acc = 0;
  for (uint32_t r = 0; r < rounds; ++r) {
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = __ldg(table + ((size_t)(probe_hash(tid * 8191u + r * 131u + j) & sector_mask) << 3));
#pragma unroll
    for (int j = 0; j < 8; ++j) acc ^= v[j];
  }
  if (acc == 0x12345678u) sink[0] = acc;  // keeps the loads live
}

// Dependent chain: the table is filled with random sector indices; each read
// names the next sector.
__global__ void k_probe_fill(uint32_t* table, uint32_t sector_mask, uint64_t n_sectors) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sectors;
       s += (uint64_t)gridDim.x * blockDim.x)
    table[s << 3] = probe_hash((uint32_t)s ^ 0xA5A5A5A5u) & sector_mask;
}

__global__ void k_probe_chain(const uint32_t* __restrict__ table, uint32_t sector_mask, uint32_t steps,
                              uint32_t* sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s = probe_hash(tid) & sector_mask;
  for (uint32_t r = 0; r < steps; ++r) s = __ldg(table + ((size_t)s << 3));
  if (s == 0xFFFFFFFFu) sink[0] = s;
}

}  // namespace

// Returns sectors/s of the independent form and of the dependent form, and
// the mean dependent-read latency in ns at full occupancy.
void probe_gather(cudaStream_t st, uint64_t table_bytes, double out[3]) {
  uint64_t n_sectors = 1;
  while (n_sectors * 2 * 32 <= table_bytes) n_sectors <<= 1;
  const uint32_t mask = (uint32_t)(n_sectors - 1);
  DevBuf table, sink;
  table.ensure(n_sectors * 32, "probe table");
  sink.ensure(64, "probe sink");
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned blocks = sms * 8, threads = 256;
  k_probe_fill<<<blocks, threads, 0, st>>>(table.as<uint32_t>(), mask, n_sectors);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const uint32_t rounds = 64, steps = 256;
  float best_i = 1e30f, best_c = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    float ms = 0;
    cudaEventRecord(e0, st);
    k_probe_independent<<<blocks, threads, 0, st>>>(table.as<uint32_t>(), mask, rounds, sink.as<uint32_t>());
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    best_i = ms < best_i ? ms : best_i;
    cudaEventRecord(e0, st);
    k_probe_chain<<<blocks, threads, 0, st>>>(table.as<uint32_t>(), mask, steps, sink.as<uint32_t>());
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    best_c = ms < best_c ? ms : best_c;
  }
  cuda_check(cudaGetLastError(), "probe");
  const double threads_total = (double)blocks * threads;
  out[0] = threads_total * rounds * 8 / (best_i / 1e3);
  out[1] = threads_total * steps / (best_c / 1e3);
  out[2] = (best_c / 1e3) / steps * 1e9;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  table.release();
  sink.release();
}

}  // namespace bingo
