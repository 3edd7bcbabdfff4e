// Binary-field arithmetic on the device: F162 = GF(2)[x]/(x^162 + x^81 + 1) and
// B128 = GF(2)[x]/(x^128 + x^7 + x^2 + x + 1) (crates/pcs/src/fields/scalar.rs:4-116), bit i of a
// value the coefficient of x^i, little-endian 64-bit limbs.
//
// Products are carry-less multiplications by the comb method with 4-bit windows (Lopez and
// Dahab, "High-speed software multiplication in F_2^m", INDOCRYPT 2000) on 32-bit limbs: the
// multiples a x^s (s < 4) stay in registers, each nibble of b selects them by sign-extended bit
// masks and adds them word-aligned (one LOP3 per limb), and the accumulator shifts by 4 bits once
// per nibble position (7 shifts in all), followed by the reduction of the double-length result.
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
// r * x^4: the four bits shifted past x^161 come back at x^0 and x^81.
__device__ __forceinline__ F162d f_times_x4(F162d r) {
  const uint64_t M34 = (1ull << 34) - 1;
  uint64_t t = (r.w[2] >> 30) & 15;
  r.w[2] = ((r.w[2] << 4) | (r.w[1] >> 60)) & M34;
  r.w[1] = (r.w[1] << 4) | (r.w[0] >> 60);
  r.w[0] = (r.w[0] << 4) ^ t;
  r.w[1] ^= t << 17;
  return r;
}

// All ones when bit `pos` of x is set, else zero: the bit moved to the sign position, then an
// arithmetic shift. With `pos` known at compile time the first shift is a multiply by a power of
// two, which the compiler may issue to the multiply-add pipe, leaving one integer-pipe instruction
// per mask.
__device__ __forceinline__ uint32_t bit_mask(uint32_t x, uint32_t pos) {
  return (uint32_t)((int32_t)(x << (31 - pos)) >> 31);
}

// c = a * b as polynomials. a's multiples by x^s (s < 4) fit NAX limbs; b has NB limbs, of which
// the top one holds TOPNIB nibbles; c has NC limbs (NC >= NB - 1 + NAX, and wide enough for the
// whole product).
template <int NAX, int NB, int TOPNIB, int NC>
__device__ __forceinline__ void clmul_comb(const uint32_t (&a)[NAX], const uint32_t (&b)[NB], uint32_t (&c)[NC]) {
  uint32_t A[4][NAX];
#pragma unroll
  for (int q = 0; q < NAX; q++) A[0][q] = a[q];
#pragma unroll
  for (int s = 1; s < 4; s++) {
    A[s][0] = A[s - 1][0] << 1;
#pragma unroll
    for (int q = 1; q < NAX; q++) A[s][q] = __funnelshift_l(A[s - 1][q - 1], A[s - 1][q], 1);
  }
#pragma unroll
  for (int q = 0; q < NC; q++) c[q] = 0;
#pragma unroll
  for (int k = 7; k >= 0; k--) {
#pragma unroll
    for (int i = 0; i < NB; i++) {
      if (i == NB - 1 && k >= TOPNIB) continue;
#pragma unroll
      for (int s = 0; s < 4; s++) {
        uint32_t m = bit_mask(b[i], 4 * k + s);
#pragma unroll
        for (int q = 0; q < NAX; q++) c[i + q] ^= A[s][q] & m;
      }
    }
    if (k > 0) {
#pragma unroll
      for (int q = NC - 1; q > 0; q--) c[q] = __funnelshift_l(c[q - 1], c[q], 4);
      c[0] <<= 4;
    }
  }
}

__device__ __forceinline__ F162d f_mul(F162d a, F162d b) {
  uint32_t A[6], B[6], c[11];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    A[2 * k] = (uint32_t)a.w[k];
    A[2 * k + 1] = (uint32_t)(a.w[k] >> 32);
    B[2 * k] = (uint32_t)b.w[k];
    B[2 * k + 1] = (uint32_t)(b.w[k] >> 32);
  }
  // a has at most 162 bits, so a x^3 fits 6 limbs; b's limb 5 holds bits 160-161 (one nibble);
  // the product has at most 323 bits (11 limbs).
  clmul_comb<6, 6, 1, 11>(A, B, c);
  uint64_t P[6];
#pragma unroll
  for (int k = 0; k < 5; k++) P[k] = (uint64_t)c[2 * k] | ((uint64_t)c[2 * k + 1] << 32);
  P[5] = c[10];
  // P = L + H x^162 with deg H <= 160; x^162 = x^81 + 1, so P = L + H + H x^81, and
  // H x^81 = Hlo x^81 + Hhi (x^81 + 1) with Hlo = H mod x^81, Hhi = H >> 81 (deg <= 79).
  const uint64_t M34 = (1ull << 34) - 1, M17 = (1ull << 17) - 1;
  uint64_t h0 = (P[2] >> 34) | (P[3] << 30);
  uint64_t h1 = (P[3] >> 34) | (P[4] << 30);
  uint64_t h2 = (P[4] >> 34) | (P[5] << 30);
  uint64_t lo0 = h0, lo1 = h1 & M17;                        // Hlo
  uint64_t hi0 = (h1 >> 17) | (h2 << 47), hi1 = h2 >> 17;   // Hhi
  F162d r;
  r.w[0] = P[0] ^ h0 ^ hi0;
  r.w[1] = P[1] ^ h1 ^ hi1;
  r.w[2] = (P[2] & M34) ^ h2;
  // + (Hlo + Hhi) x^81: bit 81 is word 1, bit 17
  uint64_t s0 = lo0 ^ hi0, s1 = lo1 ^ hi1;
  r.w[1] ^= s0 << 17;
  r.w[2] ^= (s0 >> 47) | (s1 << 17);
  r.w[2] &= M34;
  return r;
}

struct B128d {
  uint64_t lo, hi;
};
__device__ __forceinline__ B128d b_add(B128d a, B128d b) { return B128d{a.lo ^ b.lo, a.hi ^ b.hi}; }
// a * x modulo x^128 + x^7 + x^2 + x + 1
__device__ __forceinline__ B128d b_times_x(B128d a) {
  uint64_t top = a.hi >> 63;
  return B128d{(a.lo << 1) ^ ((0 - top) & 0x87ull), (a.hi << 1) | (a.lo >> 63)};
}
// a * x^4: the four bits shifted past x^127 come back times x^7 + x^2 + x + 1.
__device__ __forceinline__ B128d b_times_x4(B128d a) {
  const uint64_t t = a.hi >> 60;
  return B128d{(a.lo << 4) ^ (t << 7) ^ (t << 2) ^ (t << 1) ^ t, (a.hi << 4) | (a.lo >> 60)};
}
__device__ __forceinline__ B128d b_mul(B128d a, B128d b) {
  uint32_t A[5], B[4], c[8];
  A[0] = (uint32_t)a.lo;
  A[1] = (uint32_t)(a.lo >> 32);
  A[2] = (uint32_t)a.hi;
  A[3] = (uint32_t)(a.hi >> 32);
  A[4] = 0;
  B[0] = (uint32_t)b.lo;
  B[1] = (uint32_t)(b.lo >> 32);
  B[2] = (uint32_t)b.hi;
  B[3] = (uint32_t)(b.hi >> 32);
  clmul_comb<5, 4, 8, 8>(A, B, c);
  uint64_t P0 = (uint64_t)c[0] | ((uint64_t)c[1] << 32), P1 = (uint64_t)c[2] | ((uint64_t)c[3] << 32);
  uint64_t H0 = (uint64_t)c[4] | ((uint64_t)c[5] << 32), H1 = (uint64_t)c[6] | ((uint64_t)c[7] << 32);
  // H x^128 = H (x^7 + x^2 + x + 1); the bits of H x^7, H x^2, H x past x^127 fold once more.
  uint64_t t0 = H0 ^ (H0 << 1) ^ (H0 << 2) ^ (H0 << 7);
  uint64_t t1 = H1 ^ ((H1 << 1) | (H0 >> 63)) ^ ((H1 << 2) | (H0 >> 62)) ^ ((H1 << 7) | (H0 >> 57));
  uint64_t ov = (H1 >> 63) ^ (H1 >> 62) ^ (H1 >> 57);
  t0 ^= ov ^ (ov << 1) ^ (ov << 2) ^ (ov << 7);
  return B128d{P0 ^ t0, P1 ^ t1};
}

}  // namespace lbg
