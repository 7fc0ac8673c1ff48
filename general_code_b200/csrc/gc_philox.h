// Philox-4x32-10 counter-based random numbers (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), plus uniform doubles
// with 53 random bits and Box-Muller normals. Host and device.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define GC_RNG_HD __host__ __device__ __forceinline__
#else
#define GC_RNG_HD inline
#endif

namespace gc {

struct u32x4 {
  uint32_t v[4];
};

GC_RNG_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

GC_RNG_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c.v[0], hi0, lo0);
    mulhilo32(M1, c.v[2], hi1, lo1);
    u32x4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Uniform in (0,1) from two 32-bit words (53 bits).
GC_RNG_HD double u01(uint32_t hi, uint32_t lo) {
  uint64_t x = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
}

// Two independent N(0,1) draws from one Philox block (Box-Muller).
GC_RNG_HD void normal_pair(u32x4 r, double &z0, double &z1) {
  double u1 = u01(r.v[0], r.v[1]);
  double u2 = u01(r.v[2], r.v[3]);
  double rad = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  z0 = rad * cos(th);
  z1 = rad * sin(th);
}

// A stream of normals addressed by (key, item index, stream id): draw k of an
// item uses counter (idx_lo, idx_hi, k/2, stream).
struct NormalStream {
  uint32_t k0, k1, stream;
  uint64_t item;
  uint32_t next_block = 0;
  double cache = 0;
  bool have = false;
  GC_RNG_HD NormalStream(uint32_t key0, uint32_t key1, uint32_t stream_id,
                         uint64_t item_index)
      : k0(key0), k1(key1), stream(stream_id), item(item_index) {}
  GC_RNG_HD double next() {
    if (have) {
      have = false;
      return cache;
    }
    u32x4 c = {{(uint32_t)item, (uint32_t)(item >> 32), next_block++, stream}};
    double z0, z1;
    normal_pair(philox4x32_10(c, k0, k1), z0, z1);
    cache = z1;
    have = true;
    return z0;
  }
};

} // namespace gc
