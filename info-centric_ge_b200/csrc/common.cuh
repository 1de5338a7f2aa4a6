// Shared device helpers: counter-based RNG, the trainer's LCG with
// jump-ahead, error reporting from kernels, warp utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace felog {

constexpr int kWarp = 32;

// ---------------------------------------------------------------- errors
// A kernel that detects a problem writes the first error code it sees and
// returns; the host turns the code into a felog_status.
enum DevErr : int {
  kErrNone = 0,
  kErrDrawsExhausted = 1,   // injected draw stream too short
  kErrArenaFull = 2,        // spill arena for long walks exhausted
  kErrBadVertex = 3,        // edge endpoint >= v_num
  kErrWaitTimeout = 4,      // bounded device wait gave up
  kErrBadWeight = 5,        // alias table over a negative / non-finite weight
  kErrPlanOverflow = 6,     // batch plan larger than its buffers
  kErrWalkLimit = 7,        // a walker exceeded the iteration limit
};

// Upper bound on candidate draws of one walker.  The reference redraws a
// step-0 self-loop forever when every neighbour of the start vertex is the
// vertex itself (walk.hpp:981-983); the device walker stops there instead.
constexpr uint32_t kWalkIterLimit = 1u << 24;

__device__ __forceinline__ void set_error(int *err, int code) { atomicCAS(err, 0, code); }

// ------------------------------------------------------- Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11: 10 rounds of the 4x32 bijection with multipliers 0xD2511F53 and
// 0xCD9E8D57 and Weyl key increments 0x9E3779B9, 0xBB67AE85.
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

__host__ __device__ __forceinline__ uint32_t mulhi64_u32(uint64_t r, uint32_t n) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__umul64hi(r, (uint64_t)n);
#else
  return (uint32_t)(((unsigned __int128)r * n) >> 64);
#endif
}

// Walk draw for iteration `iter` of the walker (start, replica) in `round`:
// a candidate index in [0, deg) and a trace threshold p in [0, 1).
__device__ __forceinline__ void walk_draw(uint64_t seed, uint32_t start, uint32_t round, uint32_t iter,
                                          uint32_t replica, uint32_t deg, uint32_t &index, double &p) {
  uint4 o = philox4x32_10(make_uint4(start, round, iter, replica),
                          make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  index = mulhi64_u32(((uint64_t)o.w << 32) | o.x, deg);
  p = (double)((((uint64_t)o.y << 32) | o.z) >> 11) * (1.0 / 9007199254740992.0);
}

// ----------------------------------------------------------------- LCG
// The trainer's generator, state' = state * 25214903917 + 11 mod 2^64
// (word2vec.cu:134-143).  Jump-ahead by n composes the affine map:
// tables hold (A^(2^i), C_(2^i)) for i < 64.
struct LcgJump {
  unsigned long long a[64];
  unsigned long long c[64];
};

inline void lcg_jump_table(LcgJump &t) {
  unsigned long long a = 25214903917ULL, c = 11ULL;
  for (int i = 0; i < 64; i++) {
    t.a[i] = a;
    t.c[i] = c;
    c = a * c + c;  // (x -> a x + c) composed with itself
    a = a * a;
  }
}

__host__ __device__ __forceinline__ unsigned long long lcg_jump(const LcgJump &t, unsigned long long s,
                                                                unsigned long long n) {
  int i = 0;
  while (n) {
    if (n & 1ULL) s = t.a[i] * s + t.c[i];
    n >>= 1;
    i++;
  }
  return s;
}

__host__ __device__ __forceinline__ unsigned long long lcg_next(unsigned long long s) {
  return s * 25214903917ULL + 11ULL;
}

// ---------------------------------------------------------- warp helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

}  // namespace felog
