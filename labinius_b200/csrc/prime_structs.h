// Per-prime constant tables as the device reads them (filled on the host from ring_tables.h).
#pragma once
#include <cstdint>

#include "ring_tables.h"

namespace lbg {

// Hot per-prime constants, in constant memory: the butterfly twiddles of the six level-2 blocks
// and the cube root of unity.
struct HotPrime {
  Twiddle tw[6][13];
  uint32_t omega, omega_s;
};

// Cold per-prime tables, in global memory.
struct DevPrime {
  uint32_t lut[6][64];
  uint16_t pow3_to_leaf[N162];
  uint16_t leaf_to_pow3[N162];
  uint32_t theta_leaf[N162];
  uint16_t key_rows[N162][4];
  uint32_t key_D[N162][4][4];
  uint32_t zinv3[5][54];  // 3^-1 z_{L,k}^-1 (inverse transform)
  uint32_t zinv3sq[5][54];  // 3^-1 z_{L,k}^-2
  uint32_t omega, inv3, zeta6, det0;
  uint32_t chal[N162 * N162];  // (-1)^p theta^{E[j] p}
};

}  // namespace lbg
