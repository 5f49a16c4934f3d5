// Integer-issue probe: the roofline denominator for Keccak-bound kernels.
//
// Keccak-f[1600] on 32-bit halves is LOP3 (three-input logic) and SHF (funnel
// shift) work, about two LOP3 per SHF.  This kernel issues only those two
// instructions, as independent dependency chains, so its op rate is the B200's
// sustained LOP3+SHF issue rate; perms/s roofline = rate / 4320.
#include "azk_internal.h"

namespace azk {

static constexpr int kProbeChains = 8;
static constexpr int kProbeIters = 2048;
// per iteration and chain: 2 LOP3 + 1 SHF
static constexpr int kProbeOpsPerIter = 3 * kProbeChains;

__global__ void __launch_bounds__(256) int_issue_probe_kernel(uint32_t seed, uint32_t shift, uint32_t* out) {
  uint32_t a[kProbeChains], b[kProbeChains];
#pragma unroll
  for (int c = 0; c < kProbeChains; c++) {
    a[c] = seed ^ (threadIdx.x * 0x9E3779B9u) ^ (c * 0x85EBCA6Bu);
    b[c] = (seed + c) * 0xC2B2AE35u ^ blockIdx.x;
  }
#pragma unroll 4
  for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) {
      asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(a[c]) : "r"(a[c]), "r"(b[c]), "r"(a[(c + 1) % kProbeChains]));
      asm volatile("lop3.b32 %0, %1, %2, %3, 0xD2;" : "=r"(b[c]) : "r"(b[c]), "r"(a[c]), "r"(b[(c + 3) % kProbeChains]));
      asm volatile("shf.l.wrap.b32 %0, %1, %2, %3;" : "=r"(a[c]) : "r"(a[c]), "r"(b[c]), "r"(shift));
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int c = 0; c < kProbeChains; c++) acc ^= a[c] ^ b[c];
  if (acc == 0x12345678u) out[0] = acc;  // keeps the chains live
}

cudaError_t launch_int_issue_probe(int sm_count, cudaStream_t s, uint32_t* d_sink, double* ops_per_launch, uint32_t* blocks_out) {
  uint32_t blocks = (uint32_t)sm_count * 8;
  int_issue_probe_kernel<<<blocks, 256, 0, s>>>(0x1234567u, 13u, d_sink);
  if (ops_per_launch) *ops_per_launch = (double)blocks * 256.0 * kProbeIters * kProbeOpsPerIter;
  if (blocks_out) *blocks_out = blocks;
  return cudaGetLastError();
}

}  // namespace azk
