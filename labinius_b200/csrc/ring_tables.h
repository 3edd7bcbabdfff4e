// Host-side constant tables for the B200 prover path.
//
// The GPU transforms every F162 element separately: read as the 0/1 polynomial
// w_k(Y) = sum_m bit_m Y^m, it is evaluated at the 162 primitive 486-th roots of unity theta^v of
// R_162' = Z_q[Y]/(Y^162 - Y^81 + 1), where Y = X^4 and theta = psi^4 (splitting primes) or
// psi'^2 (quadratic-leaf primes). These are exactly the R_162 slots of the reference's commitment
// components (crates/pcs/src/ring/mod.rs:22-55), so the 648-slot commitment of a ring element
// w = sum_k X^k w_k(X^4) is the 4x4 "module" product of the key's components with these
// transforms: Y_k'(v) = sum_i [sum_{d+k=k'} a_d w_k + theta^v sum_{d+k=k'+4} a_d w_k] at leaf v.
//
// The 162-point tree (this project's own; the reference has only the 648-point trees of
// crates/pcs/src/params.rs): level 0 splits Y^162 - Y^81 + 1 into Y^81 - theta^81 and
// Y^81 - theta^405 (the Phi_6 split), levels 1..4 are radix 3, Y^n - theta^e ->
// Y^{n/3} - theta^{(e + 486 s)/3}, child s at block offset s n/3. Leaf j is Y - theta^{E[j]}.
#pragma once
#include <cstdint>
#include <vector>

namespace lbg {

constexpr int N648 = 648;
constexpr int N162 = 162;
constexpr int MAX_LIMBS = 7;

// The seven supported primes (crates/pcs/src/ring/mod.rs:87-135).
constexpr uint32_t PRIMES[7] = {2917, 3889, 4861, 9721, 12637, 17497, 19441};
int prime_index(uint32_t q);  // -1 if unsupported
bool quadratic_slots(uint32_t q);

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t q);
uint64_t inv_mod(uint64_t a, uint64_t q);

// Twiddle z with its square and their Shoup companions floor(w 2^32 / q).
struct Twiddle {
  uint32_t z, zs, z2, z2s;
};

struct PrimeTables {
  uint32_t q = 0;
  bool quad = false;
  uint64_t psi = 0;    // primitive 1944-th root (split) or 972-nd root (quad), as the reference picks it
  uint64_t theta = 0;  // primitive 486-th root naming the R_162 slots
  uint32_t omega = 0, omega_s = 0;  // theta^162 (cube root of unity) and its Shoup companion
  uint32_t zeta6 = 0;               // theta^81
  uint16_t leaf_exp[N162];          // E[j]
  uint16_t pow3_to_leaf[N162];      // reference R_162 slot s -> leaf j of this tree
  uint16_t leaf_to_pow3[N162];
  uint32_t lut[6][64];              // level-2 values of a 6-bit window (levels 0 and 1 at once)
  Twiddle tw[6][13];                // per level-2 block tau: 1 (level 2) + 3 (level 3) + 9 (level 4)
  uint32_t z_level[5][54];          // z_{L,k} = theta^{e_{L,k}/3} for L = 1..4 (forward twiddles)
  uint32_t theta_leaf[N162];        // theta^{E[j]}
  // Reference key rows -> components (crates/pcs/src/ring/mod.rs:217-340, 363-417): for slot s,
  // Y_k(v_s) = sum_t D[s][k][t] * row(rows[s][t]) mod q.
  uint16_t key_rows[N162][4];
  uint32_t key_D[N162][4][4];
  // Challenge slot table: T[p][j] = (-1)^p theta^{E[j] p}, the leaf-j value of Z^p embedded as
  // c(-X^4) (crates/pcs/src/fold.rs:287-300, 809-833).
  std::vector<uint32_t> chal_table;  // [162][162]
  uint32_t inv3 = 0, det0 = 0;        // 1/3 and 1/(2 zeta6 - 1), for the inverse transform
};

const PrimeTables& prime_tables(uint32_t q);

// Reference tree tables restated from crates/pcs/src/params.rs:63-89, 305-401 and
// crates/pcs/src/ring/mod.rs:149-179: needed to read the reference's key layout and to emit the
// commitment in the reference's R_162 slot order.
struct RefTables {
  uint32_t slot_exp[N648];
  uint32_t quad_slot_exp[324];
  uint32_t pow3_slot_exp[N162];
  uint32_t slot_648[4][N162];
  uint32_t quad_class_slot[2][N162];
};
const RefTables& ref_tables();

// Tables of the reference's 648-point transform for a splitting prime (nullptr for a
// quadratic-leaf prime); the struct is defined with the device structs.
struct Ntt648Tables;
const Ntt648Tables* ntt648_tables(uint32_t q);

// The 162-point binary transform as a tensor-core operand: the matrix T[m][v] = theta^{E[v] m}
// (bit m of an F162 times the value of Y^m at leaf v), split into T = lo + 128 hi with lo < 128 and
// hi < 256 and laid out as the B operand of a kind::i8 multiply (N = 176 leaf rows, the last 14
// zero; K = 384 bytes: lo for m < 162 at K-byte m, hi at K-byte 192 + m, zeros elsewhere), K-major
// with the 128-byte swizzle: 8-row x 128-byte atoms of 1024 bytes, the 16-byte chunk c of a row
// stored at chunk c ^ (row % 8) (tc_swizzled_offset). With the A operand of an F162 row holding
// bit m at K-byte m and 128 * bit m at K-byte 192 + m, the s32 product is sum_m bit_m T[m][v]
// exactly (at most 162 (q - 1) < 2^22).
constexpr int TC_LEAVES = 176;          // N of the transform multiply
constexpr int TC_KBYTES = 384;          // K of the transform multiply, in bytes
constexpr int TC_ATOM = 1024;           // one swizzle atom: 8 rows x 128 bytes
constexpr int TC_B_BYTES = TC_LEAVES * TC_KBYTES;  // 67584
constexpr int TC_T16_BYTES = TC_LEAVES * TC_LEAVES * 2;  // T[m][v] as u16 rows of 176 (v) x 176 (m)
// Byte offset of (row, K-byte kb) in a K-major, 128-byte-swizzled operand of `rows` rows (a
// multiple of 8): the K-atoms (128 bytes of K) one after another, each holding all row groups.
#ifdef __CUDACC__
#define LBG_HOST_DEVICE __host__ __device__
#else
#define LBG_HOST_DEVICE
#endif
LBG_HOST_DEVICE constexpr int tc_swizzled_offset(int row, int kb, int rows) {
  return (kb >> 7) * (rows * 128) + (row >> 3) * TC_ATOM + (row & 7) * 128 + ((((kb >> 4) & 7) ^ (row & 7)) << 4) +
         (kb & 15);
}
void tc_transform_operand(const PrimeTables& T, uint8_t* out /* TC_B_BYTES */);

// xorshift64* state transition as GF(2) columns: jump[k][c] = T^(2^k) applied to e_c.
const std::vector<uint64_t>& xorshift_jumps();  // 64 * 64 words

}  // namespace lbg
