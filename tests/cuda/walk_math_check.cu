// Device check of two exact shortcuts of the walker (csrc/walk.cuh), compiled
// and run by tests/test_gpu_walk_math.py:
//   * div_int(x, n, RN(1/n)) is the correctly rounded x / n (Markstein's
//     correction) for integer-valued n, compared bit for bit with __ddiv_rn;
//   * trace_test(sd, cn, mx, mn, p) decides as tanh(p_accept) <= p does in FP64.
// Prints "<division cases> <division mismatches> <trace cases> <trace mismatches>".
#include <cstdio>
#include <cstdint>

#include "walk.cuh"

using namespace felog;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_check(uint64_t n_div, uint64_t n_trace, unsigned long long *out) {
  const uint64_t t0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, st = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long dbad = 0, tbad = 0;
  for (uint64_t i = t0; i < n_div; i += st) {
    const uint64_t h = mix64(i), h2 = mix64(h);
    const double n = (double)(2 + (h & 1023));  // S + 1 for walks up to 1024 tokens
    const double u = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
    double x;
    switch ((h >> 20) & 3) {
      case 0: x = (u - 0.5) * 64.0; break;                                 // entropy-sized values
      case 1: x = (u - 0.5) * 1e-9; break;                                 // small differences
      case 2: x = ldexp(u + 1.0, (int)(h2 & 127) - 64) * ((h2 >> 8) & 1 ? -1.0 : 1.0); break;
      default: x = ldexp(u, -1000); break;                                  // near the underflow range
    }
    const double q = div_int(x, n, __drcp_rn(n));
    dbad += __double_as_longlong(q) != __double_as_longlong(__ddiv_rn(x, n));
  }
  for (uint64_t i = t0; i < n_trace; i += st) {
    const uint64_t h = mix64(i ^ 0xABCDEFull), h2 = mix64(h);
    const int sd = 1 + (int)(h % 4096), dd = 1 + (int)((h >> 12) % 100000);
    const int cn = (int)((h >> 40) % 8) - 2;
    const int mx = sd > dd ? sd : dd, mn = sd < dd ? sd : dd;
    double p = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
    if ((h2 & 3) == 0) {  // p next to tanh(p_accept): the FP64 fallback decides
      const double pa = __ddiv_rn(__dmul_rn(__ddiv_rn(1.0, (double)(sd - cn)), (double)mx), (double)mn);
      p = tanh(pa) + ((h2 >> 2) & 1 ? 1e-12 : -1e-12);
      if (p < 0.0) p = 0.0;
    }
    const double pa = __ddiv_rn(__dmul_rn(__ddiv_rn(1.0, (double)(sd - cn)), (double)mx), (double)mn);
    tbad += trace_test(sd, cn, mx, mn, p) != (tanh(pa) <= p);
  }
  atomicAdd(&out[0], dbad);
  atomicAdd(&out[1], tbad);
}

int main(int argc, char **argv) {
  const uint64_t n_div = argc > 1 ? strtoull(argv[1], nullptr, 10) : (1ull << 28);
  const uint64_t n_trace = argc > 2 ? strtoull(argv[2], nullptr, 10) : (1ull << 26);
  unsigned long long *d = nullptr, h[2] = {0, 0};
  if (cudaMalloc(&d, sizeof h) != cudaSuccess) return 2;
  cudaMemset(d, 0, sizeof h);
  k_check<<<148 * 8, 256>>>(n_div, n_trace, d);
  const cudaError_t e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    fprintf(stderr, "%s\n", cudaGetErrorString(e));
    return 2;
  }
  printf("%llu %llu %llu %llu\n", (unsigned long long)n_div, h[0], (unsigned long long)n_trace, h[1]);
  return 0;
}
