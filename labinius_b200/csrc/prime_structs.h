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
  uint32_t zfwd[5][54];     // z_{L,k} (forward transform of general coefficients)
  uint32_t omega, inv3, zeta6, det0;
  uint32_t chal[N162 * N162];  // (-1)^p theta^{E[j] p}
};

// The reference's 648-point transform of a splitting prime (crates/pcs/src/scalar.rs:35-84 and
// its inverse :123-177): twiddles of levels 1..6 of its tree (crates/pcs/src/params.rs:64-76)
// with Shoup companions; the inverse twiddles carry the 1/2 or 1/3 of their butterfly.
struct Ntt648Tables {
  uint32_t z6, z6s;                 // level 0: zeta6 = psi^324
  uint32_t omega, omega_s;          // psi^648
  uint32_t f1[2][2], f2[4][2];      // radix-2 levels: (z, zs)
  Twiddle f3[8], f4[24], f5[72], f6[216];
  uint32_t i1[2][2], i2[4][2];      // z^-1 / 2
  uint32_t inv2, inv2s, inv3, inv3s;
  Twiddle i3[8], i4[24], i5[72], i6[216];  // (z^-1 / 3, z^-2 / 3)
  uint32_t det, dets;               // 1 / (2 zeta6 - 1)
};

}  // namespace lbg
