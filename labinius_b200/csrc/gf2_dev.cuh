// Binary-field arithmetic on the device: F162 = GF(2)[x]/(x^162 + x^81 + 1) and
// B128 = GF(2)[x]/(x^128 + x^7 + x^2 + x + 1) (crates/pcs/src/fields/scalar.rs:4-116), bit i of a
// value the coefficient of x^i, little-endian 64-bit limbs.
#pragma once
#include <cstdint>

namespace lbg {

struct F162d {
  uint64_t w[3];
};
__device__ __forceinline__ F162d f_add(F162d a, F162d b) {
  return F162d{{a.w[0] ^ b.w[0], a.w[1] ^ b.w[1], a.w[2] ^ b.w[2]}};
}
// r * x with the reduction folded in (x^162 = x^81 + 1)
__device__ __forceinline__ F162d f_times_x(F162d r) {
  const uint64_t M34 = (1ull << 34) - 1;
  uint64_t top = (r.w[2] >> 33) & 1;
  r.w[2] = ((r.w[2] << 1) | (r.w[1] >> 63)) & M34;
  r.w[1] = (r.w[1] << 1) | (r.w[0] >> 63);
  r.w[0] <<= 1;
  uint64_t tm = 0 - top;
  r.w[0] ^= tm & 1;
  r.w[1] ^= tm & (1ull << 17);
  return r;
}
// Shift-and-add product with the reduction folded into the shift.
__device__ inline F162d f_mul(F162d a, F162d b) {
  F162d r{{0, 0, 0}};
  for (int i = 161; i >= 0; i--) {
    r = f_times_x(r);
    uint64_t bm = 0 - ((b.w[i >> 6] >> (i & 63)) & 1);
    r.w[0] ^= a.w[0] & bm;
    r.w[1] ^= a.w[1] & bm;
    r.w[2] ^= a.w[2] & bm;
  }
  return r;
}

struct B128d {
  uint64_t lo, hi;
};
__device__ __forceinline__ B128d b_add(B128d a, B128d b) { return B128d{a.lo ^ b.lo, a.hi ^ b.hi}; }
// Shift-and-add product modulo x^128 + x^7 + x^2 + x + 1.
__device__ inline B128d b_mul(B128d a, B128d b) {
  B128d r{0, 0};
  for (int i = 127; i >= 0; i--) {
    uint64_t top = r.hi >> 63;
    r.hi = (r.hi << 1) | (r.lo >> 63);
    r.lo = (r.lo << 1) ^ ((0 - top) & 0x87ull);
    uint64_t bm = 0 - (((i < 64 ? b.lo >> i : b.hi >> (i - 64))) & 1);
    r.lo ^= a.lo & bm;
    r.hi ^= a.hi & bm;
  }
  return r;
}

}  // namespace lbg
