// philox.h -- TEST INFRASTRUCTURE ONLY.  The oracle's counter-based random
// numbers, shared by the oracle (oracle/fcm_oracle.cpp) and the SPRNG stand-in of
// the reference build (oracle/ref_shim), so both draw the same uniforms.
#pragma once

#include <cmath>
#include <cstdint>

namespace orcrng {

// ============================================================ Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of the 4x32 Philox S-box with
// multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 /
// 0xBB67AE85.
struct Philox {
  static inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
  }
  static void gen(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for (int r = 0; r < 10; ++r) {
      uint32_t hi0, lo0, hi1, lo1;
      mulhilo(0xD2511F53u, c0, hi0, lo0);
      mulhilo(0xCD9E8D57u, c2, hi1, lo1);
      uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
      c0 = n0; c1 = n1; c2 = n2; c3 = n3;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
  }
};

// Sequential uniform stream on (0,1) built from Philox blocks, standing in for
// SPRNG's sprng() (parallel_random_numbers.hpp:13-17).
struct UniformStream {
  uint32_t key0, key1;
  uint64_t block;
  uint32_t buf[4];
  int pos;
  UniformStream(uint64_t seed, uint64_t stream) : key0((uint32_t)seed), key1((uint32_t)(seed >> 32)), block(0), pos(4) {
    stream_lo = (uint32_t)stream;
    stream_hi = (uint32_t)(stream >> 32);
  }
  uint32_t stream_lo, stream_hi;
  double next() {
    if (pos == 4) {
      uint32_t c[4] = {(uint32_t)block, (uint32_t)(block >> 32), stream_lo, stream_hi};
      Philox::gen(c, key0, key1, buf);
      ++block;
      pos = 0;
    }
    uint32_t a = buf[pos++];
    return ((double)a + 0.5) * (1.0 / 4294967296.0);
  }
  // parallel_random_numbers.cpp:8-19 (Marsaglia polar method, one normal).
  double gaussian_random() {
    double x1, x2, w = 10.0;
    while (w > 1.0 || w == 1) {
      x1 = 2.0 * next() - 1.0;
      x2 = 2.0 * next() - 1.0;
      w = x1 * x1 + x2 * x2;
    }
    w = std::sqrt((-2.0 * std::log(w)) / w);
    return w * x1;
  }
};

}  // namespace orcrng
