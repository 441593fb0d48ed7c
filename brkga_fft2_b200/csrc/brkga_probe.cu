// brkga_probe.cu — measurement kernels for the roofline denominators of the
// decode kernel (no reference counterpart).
//
// smem_stream_kernel: every thread streams 16-byte ld.shared.v4 loads over a
// 32 KB shared buffer, consecutive lanes on consecutive 16-byte words (no
// bank conflicts: one warp load = four 128-byte wavefronts), eight loads in
// flight per step, XOR-folded so nothing is dead code.  Launched with enough
// CTAs to fill every SM, its bytes per second are the shared-memory (L1 data
// pipe) bandwidth the decode kernel's plate and mask reads are served from.

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/brkga_b200.h"

namespace {

constexpr int kProbeWords = 2048;  // uint4 words: 32 KB of shared memory per CTA

__global__ void smem_stream_kernel(int iters, uint32_t* sink, long long* cycles) {
  __shared__ uint4 buf[kProbeWords];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < kProbeWords; i += nt) buf[i] = make_uint4(i, 3u * i + 1u, 5u * i + 2u, 7u * i + 3u);
  __syncthreads();
  uint32_t a = 0u, b = 0u, c = 0u, d = 0u;
  int idx = tid & (kProbeWords - 1);
  const long long t0 = clock64();
  for (int it = 0; it < iters; ++it) {
    uint4 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = buf[(idx + k * nt) & (kProbeWords - 1)];
#pragma unroll
    for (int k = 0; k < 8; k += 2) {
      a ^= v[k].x ^ v[k + 1].x;
      b ^= v[k].y ^ v[k + 1].y;
      c ^= v[k].z ^ v[k + 1].z;
      d ^= v[k].w ^ v[k + 1].w;
    }
    idx = (idx + 8 * nt + it) & (kProbeWords - 1);
  }
  const long long t1 = clock64();
  sink[(size_t)blockIdx.x * nt + tid] = a ^ b ^ c ^ d;
  if (tid == 0) cycles[blockIdx.x] = t1 - t0;
}

}  // namespace

extern "C" {

int brkga_probe_smem_stream(int32_t blocks, int32_t threads, int32_t iters, uint32_t* d_sink, int64_t* d_cycles,
                            void* stream) {
  if (blocks < 1 || threads < 32 || threads > 1024 || (threads & 31) || iters < 1 || !d_sink || !d_cycles)
    return BRKGA_ERR_INVALID_ARGUMENT;
  smem_stream_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, d_sink,
                                                                  reinterpret_cast<long long*>(d_cycles));
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

}  // extern "C"
