// Device kernels of the labinius prover path for B200 (sm_100a).
//
// Arithmetic: exact modular integer arithmetic mod q < 2^15 on 32-bit lanes (Shoup products with
// precomputed companions, lazily reduced between levels) and GF(2) XOR arithmetic for F162.
// Nothing here is floating point; every output is canonical, so results are bit-identical to the
// reference's whatever the internal representatives.
#pragma once
#include <cstdint>

#include "gf2_dev.cuh"
#include "prime_structs.h"
#include "ring_tables.h"

namespace lbg {

// Compile-time primes, indexed like PRIMES.
template <int PI>
struct Pr;
#define LBG_PRIME(I, QV)                                     \
  template <>                                                \
  struct Pr<I> {                                             \
    static constexpr uint32_t q = QV;                        \
    static constexpr uint32_t qs = (uint32_t)((1ull << 32) / QV); \
  };
LBG_PRIME(0, 2917)
LBG_PRIME(1, 3889)
LBG_PRIME(2, 4861)
LBG_PRIME(3, 9721)
LBG_PRIME(4, 12637)
LBG_PRIME(5, 17497)
LBG_PRIME(6, 19441)
#undef LBG_PRIME

// Hot per-prime constants in constant memory. This header is included by kernels.cu only (the
// one translation unit that launches kernels), so the definition lives here.
__constant__ HotPrime c_hot[7];

// ---------------------------------------------------------------------------------------------
// modular helpers
// ---------------------------------------------------------------------------------------------
// a * w mod q in [0, 2q) for any a < 2^32 (ws = floor(w 2^32 / q)).
__device__ __forceinline__ uint32_t mul_shoup(uint32_t a, uint32_t w, uint32_t ws, uint32_t q) {
  uint32_t t = __umulhi(a, ws);
  return a * w - t * q;
}
// x mod q, fully reduced, for x < 2^32.
template <int PI>
__device__ __forceinline__ uint32_t red_full(uint32_t x) {
  constexpr uint32_t q = Pr<PI>::q;
  uint32_t r = x - __umulhi(x, Pr<PI>::qs) * q;
  return r >= q ? r - q : r;
}
template <int PI>
__device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b) {
  static_assert((uint64_t)(Pr<PI>::q - 1) * (Pr<PI>::q - 1) < (1ull << 32), "the product fits 32 bits");
  return red_full<PI>(a * b);
}
// x mod q up to one extra q: [0, 2q), for x < 2^32.
template <int PI>
__device__ __forceinline__ uint32_t red_half(uint32_t x) {
  return x - __umulhi(x, Pr<PI>::qs) * Pr<PI>::q;
}
// a * b mod q for a, b < q (the product is below 2^32 for every prime here).
template <int PI>
__device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b);
// a signed accumulator brought back to |r| < 2q (exact modulo q).
template <int PI>
__device__ __forceinline__ int32_t red_signed(int32_t x) {
  return x - __mulhi(x, (int32_t)Pr<PI>::qs) * (int32_t)Pr<PI>::q;
}
template <int PI>
__device__ __forceinline__ uint32_t red_signed_full(int32_t x) {
  constexpr int32_t q = Pr<PI>::q;
  int32_t r = x % q;
  return (uint32_t)(r < 0 ? r + q : r);
}
template <int PI>
__device__ __forceinline__ int16_t center(uint32_t x) {
  constexpr uint32_t q = Pr<PI>::q;
  return (int16_t)(x > (q - 1) / 2 ? (int32_t)x - (int32_t)q : (int32_t)x);
}

// Lazy radix-3 butterfly of the 162-point tree: sub-ring Y^n - z^3 -> children Y^{n/3} - z w^s,
// y_s = a0 + (z w^s) a1 + (z w^s)^2 a2, with w^2 = -1 - w:
//   t1 = z a1, t2 = z^2 a2, m = w (t1 - t2);  y0 = a0 + t1 + t2,  y1 = a0 - t2 + m,  y2 = a0 - t1 - m.
// Products are Shoup's, in [0, 2q); the constant 4q keeps every difference non-negative, so an
// output exceeds its inputs' bound by at most 6q.
template <int PI>
__device__ __forceinline__ void bfly3(uint32_t& a0, uint32_t& a1, uint32_t& a2, const Twiddle& t,
                                      uint32_t om, uint32_t oms) {
  constexpr uint32_t q = Pr<PI>::q;
  uint32_t t1 = mul_shoup(a1, t.z, t.zs, q);
  uint32_t t2 = mul_shoup(a2, t.z2, t.z2s, q);
  uint32_t m = mul_shoup(t1 - t2 + 2 * q, om, oms, q);
  uint32_t b = a0 + 4 * q;
  a0 = a0 + t1 + t2;
  a1 = b - t2 + m;
  a2 = b - t1 - m;
}

// The same butterfly when a1 and a2 arrive already multiplied by z and z^2 (t1 = z a1, t2 = z^2 a2,
// both in [0, q)): only the omega product is left, and every output stays within bfly3's bound.
template <int PI>
__device__ __forceinline__ void bfly3_scaled(uint32_t& a0, uint32_t& t1, uint32_t& t2, uint32_t om, uint32_t oms) {
  constexpr uint32_t q = Pr<PI>::q;
  uint32_t m = mul_shoup(t1 - t2 + 2 * q, om, oms, q);
  uint32_t b = a0 + 4 * q;
  uint32_t y0 = a0 + t1 + t2, y1 = b - t2 + m, y2 = b - t1 - m;
  a0 = y0;
  t1 = y1;
  t2 = y2;
}

// The 27 six-bit LUT indices of one F162, as byte offsets into a u16 table (2 x index, one per
// byte, four per word): index m collects bits m + 27 t, t = 0..5, of the element, the
// coefficients that levels 0 and 1 of the tree combine.
__device__ __forceinline__ void f162_windows(uint64_t w0, uint64_t w1, uint64_t w2, uint32_t idx[7]) {
  const uint32_t M27 = 0x7FFFFFFu;
  uint32_t c[6];
  c[0] = (uint32_t)w0 & M27;
  c[1] = (uint32_t)(w0 >> 27) & M27;
  c[2] = (uint32_t)((w0 >> 54) | (w1 << 10)) & M27;
  c[3] = (uint32_t)(w1 >> 17) & M27;
  c[4] = (uint32_t)((w1 >> 44) | (w2 << 20)) & M27;
  c[5] = (uint32_t)(w2 >> 7) & M27;
#pragma unroll
  for (int g = 0; g < 7; g++) {
    uint32_t acc = 0;
#pragma unroll
    for (int t = 0; t < 6; t++) {
      uint32_t nib = (c[t] >> (4 * g)) & 15u;
      acc += ((nib * 0x00204081u) & 0x01010101u) << (t + 1);
    }
    idx[g] = acc;
  }
}

// The shared-memory window tables of the transform: per block tau three 64-entry u16 tables of
// 128 bytes each (one row of the 32 banks, so the 32 lanes' lookups never conflict): the window
// values (levels 0 and 1 at once), and the same times the block's level-2 twiddle z and z^2, so
// that level 2 reads its products instead of computing them.
constexpr int NTT_LUT_U16 = 6 * 3 * 64;
template <int PI>
__device__ __forceinline__ void load_ntt_lut(uint16_t* __restrict__ lut, const DevPrime* __restrict__ D) {
  for (int x = threadIdx.x; x < NTT_LUT_U16; x += blockDim.x) {
    const int tau = x / 192, g = (x / 64) % 3;
    uint32_t v = D->lut[tau][x % 64];
    if (g) v = red_full<PI>(v * (g == 1 ? c_hot[PI].tw[tau][0].z : c_hot[PI].tw[tau][0].z2));
    lut[x] = (uint16_t)v;
  }
}

// Forward transform of one level-2 block (27 leaves) of one F162: v[x] = w(theta^{E[27 tau + x]}),
// reduced to [0, 2q), from the tables load_ntt_lut wrote.
template <int PI, int TAU>
__device__ __forceinline__ void ntt_block(const uint32_t idx[7], const uint8_t* __restrict__ lut,
                                          uint32_t v[27]) {
  const HotPrime& H = c_hot[PI];
  const uint32_t om = H.omega, oms = H.omega_s;
#pragma unroll
  for (int m = 0; m < 27; m++)
    v[m] = *(const uint16_t*)(lut + TAU * 384 + (m / 9) * 128 + __byte_perm(idx[m >> 2], 0, 0x4440 | (m & 3)));
#pragma unroll
  for (int i = 0; i < 9; i++) bfly3_scaled<PI>(v[i], v[9 + i], v[18 + i], om, oms);
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int i = 0; i < 3; i++) bfly3<PI>(v[9 * s + i], v[9 * s + 3 + i], v[9 * s + 6 + i], H.tw[TAU][1 + s], om, oms);
#pragma unroll
  for (int s = 0; s < 9; s++) bfly3<PI>(v[3 * s], v[3 * s + 1], v[3 * s + 2], H.tw[TAU][4 + s], om, oms);
#pragma unroll
  for (int m = 0; m < 27; m++) v[m] = red_half<PI>(v[m]);
}

// Exact inverse of the 162-point transform, in place on x[0..161] (values in [0, q)), one
// thread. Used for the folded witness and the bit-dropped residues, a few thousand per round.
template <int PI>
__device__ void intt162_serial(uint32_t* x, const DevPrime& D) {
  constexpr uint32_t q = Pr<PI>::q;
  const uint32_t w = D.omega, w2 = mulmod<PI>(D.omega, D.omega);
  // inverse radix-3 levels 4, 3, 2, 1: sub-ring k of level L spans n = 81 / 3^{L-1}
  for (int L = 4; L >= 1; L--) {
    int n = 81;
    for (int l = 1; l < L; l++) n /= 3;
    int m = n / 3;
    int subrings = 162 / n;
    for (int k = 0; k < subrings; k++) {
      uint32_t zi = D.zinv3[L][k], zi2 = D.zinv3sq[L][k];
      int base = k * n;
      for (int i = 0; i < m; i++) {
        uint32_t y0 = x[base + i], y1 = x[base + m + i], y2 = x[base + 2 * m + i];
        uint32_t s0 = (y0 + y1 + y2) % q;
        uint32_t s1 = (y0 + mulmod<PI>(w2, y1) + mulmod<PI>(w, y2)) % q;
        uint32_t s2 = (y0 + mulmod<PI>(w, y1) + mulmod<PI>(w2, y2)) % q;
        x[base + i] = mulmod<PI>(s0, D.inv3);
        x[base + m + i] = mulmod<PI>(s1, zi);
        x[base + 2 * m + i] = mulmod<PI>(s2, zi2);
      }
    }
  }
  // level 0: y0 = a + zeta6 b, y1 = a + zeta6^-1 b  =>  b = (y0 - y1) / (2 zeta6 - 1), a = y0 - zeta6 b
  for (int i = 0; i < 81; i++) {
    uint32_t y0 = x[i], y1 = x[i + 81];
    uint32_t b = mulmod<PI>((y0 + q - y1) % q, D.det0);
    uint32_t a = (y0 + q - mulmod<PI>(D.zeta6, b)) % q;
    x[i] = a;
    x[i + 81] = b;
  }
}

// intt162_serial by a group of threads: x[0..161] in shared memory, thread j < 54 of the group
// makes one radix-3 butterfly per level (the 54 of a level touch disjoint entries) and the
// radix-2 pairs j and j + 54 of level 0, with the same arithmetic. Every thread of the block calls
// it: it synchronises the block after each level.
template <int PI>
__device__ __forceinline__ void intt162_group(uint32_t* x, int j, const DevPrime& D) {
  const uint32_t w = D.omega, w2 = mulmod<PI>(D.omega, D.omega);
  for (int L = 4; L >= 1; L--) {
    const int n = L == 4 ? 3 : L == 3 ? 9 : L == 2 ? 27 : 81, m = n / 3;
    if (j < 54) {
      const int k = j / m, i = j - k * m, base = k * n;
      const uint32_t y0 = x[base + i], y1 = x[base + m + i], y2 = x[base + 2 * m + i];
      const uint32_t s0 = red_full<PI>(y0 + y1 + y2);
      const uint32_t s1 = red_full<PI>(y0 + mulmod<PI>(w2, y1) + mulmod<PI>(w, y2));
      const uint32_t s2 = red_full<PI>(y0 + mulmod<PI>(w, y1) + mulmod<PI>(w2, y2));
      x[base + i] = mulmod<PI>(s0, D.inv3);
      x[base + m + i] = mulmod<PI>(s1, D.zinv3[L][k]);
      x[base + 2 * m + i] = mulmod<PI>(s2, D.zinv3sq[L][k]);
    }
    __syncthreads();
  }
  constexpr uint32_t q = Pr<PI>::q;
  for (int i = j; i < 81 && j < 54; i += 54) {
    const uint32_t y0 = x[i], y1 = x[i + 81];
    const uint32_t b = mulmod<PI>(red_full<PI>(y0 + q - y1), D.det0);
    x[i] = red_full<PI>(y0 + q - mulmod<PI>(D.zeta6, b));
    x[i + 81] = b;
  }
  __syncthreads();
}

// ntt162_serial by a group of threads (as intt162_group): level 0's pairs j and j + 54, then one
// radix-3 butterfly per thread j < 54 and level. Every thread of the block calls it.
template <int PI>
__device__ __forceinline__ void ntt162_group(uint32_t* x, int j, const DevPrime& D) {
  constexpr uint32_t q = Pr<PI>::q;
  const uint32_t w = D.omega, w2 = mulmod<PI>(D.omega, D.omega);
  for (int i = j; i < 81 && j < 54; i += 54) {
    const uint32_t a = x[i], b = x[i + 81];
    const uint32_t t = mulmod<PI>(D.zeta6, b);
    x[i] = red_full<PI>(a + t);
    x[i + 81] = red_full<PI>(a + b + q - t);
  }
  __syncthreads();
  for (int L = 1; L <= 4; L++) {
    const int n = L == 1 ? 81 : L == 2 ? 27 : L == 3 ? 9 : 3, m = n / 3;
    if (j < 54) {
      const int k = j / m, i = j - k * m, base = k * n;
      const uint32_t z = D.zfwd[L][k], z2 = mulmod<PI>(z, z);
      const uint32_t a0 = x[base + i];
      const uint32_t t1 = mulmod<PI>(x[base + m + i], z), t2 = mulmod<PI>(x[base + 2 * m + i], z2);
      x[base + i] = red_full<PI>(a0 + t1 + t2);
      x[base + m + i] = red_full<PI>(a0 + mulmod<PI>(w, t1) + mulmod<PI>(w2, t2));
      x[base + 2 * m + i] = red_full<PI>(a0 + mulmod<PI>(w2, t1) + mulmod<PI>(w, t2));
    }
    __syncthreads();
  }
}

// The forward 162-point transform of general coefficients in [0, q), in place on x[0..161], one
// thread; leaves come out in the tree order the commit uses (the exact inverse of
// intt162_serial). Used by the verifier, a few thousand per call.
template <int PI>
__device__ void ntt162_serial(uint32_t* x, const DevPrime& D) {
  constexpr uint32_t q = Pr<PI>::q;
  const uint32_t w = D.omega, w2 = mulmod<PI>(D.omega, D.omega);
  // level 0: y0 = a + zeta6 b, y1 = a + (1 - zeta6) b
  for (int i = 0; i < 81; i++) {
    uint32_t a = x[i], b = x[i + 81];
    uint32_t t = mulmod<PI>(D.zeta6, b);
    x[i] = (a + t) % q;
    x[i + 81] = (a + b + q - t) % q;
  }
  // radix-3 levels 1..4: sub-ring k of level L spans n = 81 / 3^{L-1}
  for (int L = 1; L <= 4; L++) {
    int n = 81;
    for (int l = 1; l < L; l++) n /= 3;
    int m = n / 3;
    int subrings = 162 / n;
    for (int k = 0; k < subrings; k++) {
      uint32_t z = D.zfwd[L][k], z2 = mulmod<PI>(z, z);
      int base = k * n;
      for (int i = 0; i < m; i++) {
        uint32_t a0 = x[base + i];
        uint32_t t1 = mulmod<PI>(x[base + m + i], z), t2 = mulmod<PI>(x[base + 2 * m + i], z2);
        x[base + i] = (a0 + t1 + t2) % q;
        x[base + m + i] = (a0 + mulmod<PI>(w, t1) + mulmod<PI>(w2, t2)) % q;
        x[base + 2 * m + i] = (a0 + mulmod<PI>(w2, t1) + mulmod<PI>(w, t2)) % q;
      }
    }
  }
}

}  // namespace lbg
