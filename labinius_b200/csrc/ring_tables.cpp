#include "ring_tables.h"

#include "prime_structs.h"

#include <mutex>
#include <stdexcept>

namespace lbg {

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1;
  b %= q;
  while (e) {
    if (e & 1) r = r * b % q;
    b = b * b % q;
    e >>= 1;
  }
  return r;
}
uint64_t inv_mod(uint64_t a, uint64_t q) { return pow_mod(a % q, q - 2, q); }

int prime_index(uint32_t q) {
  for (int i = 0; i < 7; i++)
    if (PRIMES[i] == q) return i;
  return -1;
}

// crates/pcs/src/params.rs:266-268
bool quadratic_slots(uint32_t q) { return (q - 1) % 972 == 0 && (q - 1) % 1944 != 0; }

// ---------------------------------------------------------------------------------------------
// The reference's 648-point tree orders (crates/pcs/src/params.rs:63-89, 300-401 and
// crates/pcs/src/ring/mod.rs:149-179), restated to read its key layout and emit its slot order.
// ---------------------------------------------------------------------------------------------
static const int RADIX648[7] = {2, 2, 2, 3, 3, 3, 3};
static const int RADIXQ[6] = {2, 2, 3, 3, 3, 3};

static uint32_t subring_exp648(int level, int k) {
  if (level == 1) return k == 0 ? 324 : 1620;
  uint32_t p = RADIX648[level - 1];
  return (subring_exp648(level - 1, k / p) + 1944u * (k % p)) / p;
}
static uint32_t subring_exp_quad648(int level, int k) {
  if (level == 1) return k == 0 ? 162 : 810;
  uint32_t p = RADIXQ[level - 1];
  return (subring_exp_quad648(level - 1, k / p) + 972u * (k % p)) / p;
}

static uint32_t shoup32(uint32_t w, uint32_t q) { return (uint32_t)(((uint64_t)w << 32) / q); }

// Twiddles of the 648-point tree: zeta_{L,k} = psi^{subring_exp(L,k) / RADIX[L]}
// (crates/pcs/src/params.rs:64-76, 115-166), psi the reference's primitive 1944-th root.
static Ntt648Tables* build_ntt648(uint32_t q) {
  Ntt648Tables* T = new Ntt648Tables();
  uint64_t psi = 0;
  for (uint64_t x = 2;; x++)
    if (pow_mod(x, 1944, q) == 1 && pow_mod(x, 972, q) != 1 && pow_mod(x, 648, q) != 1) {
      psi = x;
      break;
    }
  auto zeta = [&](int level, int k) { return (uint32_t)pow_mod(psi, subring_exp648(level, k) / RADIX648[level], q); };
  auto tw = [&](uint32_t z) {
    Twiddle w;
    w.z = z;
    w.zs = shoup32(z, q);
    w.z2 = (uint32_t)((uint64_t)z * z % q);
    w.z2s = shoup32(w.z2, q);
    return w;
  };
  uint64_t inv2 = inv_mod(2, q), inv3 = inv_mod(3, q);
  auto itw = [&](uint32_t z) {  // (z^-1 / 3, z^-2 / 3)
    uint64_t zi = inv_mod(z, q);
    Twiddle w;
    w.z = (uint32_t)(zi * inv3 % q);
    w.zs = shoup32(w.z, q);
    w.z2 = (uint32_t)(zi * zi % q * inv3 % q);
    w.z2s = shoup32(w.z2, q);
    return w;
  };
  T->z6 = (uint32_t)pow_mod(psi, 324, q);
  T->z6s = shoup32(T->z6, q);
  T->omega = (uint32_t)pow_mod(psi, 648, q);
  T->omega_s = shoup32(T->omega, q);
  for (int k = 0; k < 2; k++) {
    uint32_t z = zeta(1, k);
    T->f1[k][0] = z;
    T->f1[k][1] = shoup32(z, q);
    uint32_t zi = (uint32_t)(inv_mod(z, q) * inv2 % q);
    T->i1[k][0] = zi;
    T->i1[k][1] = shoup32(zi, q);
  }
  for (int k = 0; k < 4; k++) {
    uint32_t z = zeta(2, k);
    T->f2[k][0] = z;
    T->f2[k][1] = shoup32(z, q);
    uint32_t zi = (uint32_t)(inv_mod(z, q) * inv2 % q);
    T->i2[k][0] = zi;
    T->i2[k][1] = shoup32(zi, q);
  }
  for (int k = 0; k < 8; k++) T->f3[k] = tw(zeta(3, k)), T->i3[k] = itw(zeta(3, k));
  for (int k = 0; k < 24; k++) T->f4[k] = tw(zeta(4, k)), T->i4[k] = itw(zeta(4, k));
  for (int k = 0; k < 72; k++) T->f5[k] = tw(zeta(5, k)), T->i5[k] = itw(zeta(5, k));
  for (int k = 0; k < 216; k++) T->f6[k] = tw(zeta(6, k)), T->i6[k] = itw(zeta(6, k));
  T->inv2 = (uint32_t)inv2;
  T->inv2s = shoup32(T->inv2, q);
  T->inv3 = (uint32_t)inv3;
  T->inv3s = shoup32(T->inv3, q);
  T->det = (uint32_t)inv_mod((2ull * T->z6 + q - 1) % q, q);
  T->dets = shoup32(T->det, q);
  return T;
}

const Ntt648Tables* ntt648_tables(uint32_t q) {
  static std::mutex mu;
  static Ntt648Tables* cache[7] = {nullptr};
  int pi = prime_index(q);
  if (pi < 0 || quadratic_slots(q)) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (!cache[pi]) cache[pi] = build_ntt648(q);
  return cache[pi];
}

static RefTables build_ref() {
  RefTables t;
  for (int j = 0; j < N648; j++) t.slot_exp[j] = subring_exp648(7, j);
  for (int j = 0; j < 324; j++) t.quad_slot_exp[j] = subring_exp_quad648(6, j);
  int pos[486];
  for (int i = 0; i < 486; i++) pos[i] = -1;
  int n = 0;
  for (int j = 0; j < N648; j++) {
    uint32_t u = t.slot_exp[j], v = u % 486, tt = (u - v) / 486;
    if (pos[v] < 0) {
      pos[v] = n;
      t.pow3_slot_exp[n++] = v;
    }
    t.slot_648[tt][pos[v]] = j;
  }
  if (n != N162) throw std::runtime_error("R_162 slot order has the wrong size");
  for (int s = 0; s < N162; s++) {
    uint32_t v = t.pow3_slot_exp[s];
    for (int j = 0; j < 324; j++) {
      if (t.quad_slot_exp[j] == v) t.quad_class_slot[0][s] = j;
      if (t.quad_slot_exp[j] == v + 486) t.quad_class_slot[1][s] = j;
    }
  }
  return t;
}

const RefTables& ref_tables() {
  static RefTables t = build_ref();
  return t;
}

// crates/pcs/src/params.rs:53-61, 291-299
static uint64_t find_root(uint64_t q, uint64_t order, uint64_t d1, uint64_t d2) {
  for (uint64_t x = 2;; x++)
    if (pow_mod(x, order, q) == 1 && pow_mod(x, d1, q) != 1 && pow_mod(x, d2, q) != 1) return x;
}

static uint32_t shoup(uint32_t w, uint32_t q) { return (uint32_t)(((uint64_t)w << 32) / q); }

static PrimeTables* build_prime(uint32_t q) {
  PrimeTables* P = new PrimeTables();
  P->q = q;
  P->quad = quadratic_slots(q);
  if (!P->quad) {
    P->psi = find_root(q, 1944, 972, 648);
    P->theta = pow_mod(P->psi, 4, q);
  } else {
    P->psi = find_root(q, 972, 486, 324);
    P->theta = pow_mod(P->psi, 2, q);
  }
  uint64_t th = P->theta;
  P->omega = (uint32_t)pow_mod(th, 162, q);
  P->omega_s = shoup(P->omega, q);
  P->zeta6 = (uint32_t)pow_mod(th, 81, q);
  P->inv3 = (uint32_t)inv_mod(3, q);
  P->det0 = (uint32_t)inv_mod((2ull * P->zeta6 + q - 1) % q, q);

  // exponents of the 162-point tree: e[L][k], L = 1..5 (level 5 = leaves)
  std::vector<std::vector<uint32_t>> e(6);
  e[1] = {81, 405};
  for (int L = 1; L <= 4; L++)
    for (size_t k = 0; k < e[L].size(); k++)
      for (uint32_t s = 0; s < 3; s++) e[L + 1].push_back((e[L][k] + 486u * s) / 3);
  for (int j = 0; j < N162; j++) P->leaf_exp[j] = (uint16_t)e[5][j];
  for (int L = 1; L <= 4; L++)
    for (size_t k = 0; k < e[L].size(); k++) P->z_level[L][k] = (uint32_t)pow_mod(th, e[L][k] / 3, q);
  for (int j = 0; j < N162; j++) P->theta_leaf[j] = (uint32_t)pow_mod(th, e[5][j], q);

  // level-2 LUT: block tau is Z_q[Y]/(Y^27 - c), c = theta^{e[2][tau]}; coefficient m of a binary
  // polynomial reduced there is sum_{t<6} b_{m+27t} c^t.
  for (int tau = 0; tau < 6; tau++) {
    uint64_t c = pow_mod(th, e[2][tau], q);
    for (int idx = 0; idx < 64; idx++) {
      uint64_t acc = 0, ct = 1;
      for (int t = 0; t < 6; t++) {
        if ((idx >> t) & 1) acc = (acc + ct) % q;
        ct = ct * c % q;
      }
      P->lut[tau][idx] = (uint32_t)acc;
    }
  }
  auto mk = [&](uint32_t z) {
    Twiddle w;
    w.z = z;
    w.zs = shoup(z, q);
    w.z2 = (uint32_t)((uint64_t)z * z % q);
    w.z2s = shoup(w.z2, q);
    return w;
  };
  for (int tau = 0; tau < 6; tau++) {
    P->tw[tau][0] = mk(P->z_level[2][tau]);
    for (int s = 0; s < 3; s++) P->tw[tau][1 + s] = mk(P->z_level[3][3 * tau + s]);
    for (int s = 0; s < 9; s++) P->tw[tau][4 + s] = mk(P->z_level[4][9 * tau + s]);
  }

  const RefTables& R = ref_tables();
  for (int s = 0; s < N162; s++) {
    int found = -1;
    for (int j = 0; j < N162; j++)
      if (P->leaf_exp[j] == R.pow3_slot_exp[s]) found = j;
    if (found < 0) throw std::runtime_error("R_162 slot without a leaf");
    P->pow3_to_leaf[s] = (uint16_t)found;
    P->leaf_to_pow3[found] = (uint16_t)s;
  }

  // key rows -> components
  for (int s = 0; s < N162; s++) {
    uint64_t v = R.pow3_slot_exp[s];
    if (!P->quad) {
      uint64_t inv4 = inv_mod(4, q), i4 = pow_mod(P->psi, 486, q);
      for (int t = 0; t < 4; t++) P->key_rows[s][t] = (uint16_t)R.slot_648[t][s];
      for (int k = 0; k < 4; k++) {
        uint64_t tw = inv4 * pow_mod(P->psi, (1944 - (v * k) % 1944) % 1944, q) % q;
        for (int t = 0; t < 4; t++)
          P->key_D[s][k][t] = (uint32_t)(tw * pow_mod(i4, (4 - (t * k) % 4) % 4, q) % q);
      }
    } else {
      uint64_t inv2 = inv_mod(2, q);
      uint64_t tw = inv2 * pow_mod(P->psi, (972 - v) % 972, q) % q;
      uint32_t jp = R.quad_class_slot[0][s], jm = R.quad_class_slot[1][s];
      P->key_rows[s][0] = (uint16_t)(2 * jp);
      P->key_rows[s][1] = (uint16_t)(2 * jp + 1);
      P->key_rows[s][2] = (uint16_t)(2 * jm);
      P->key_rows[s][3] = (uint16_t)(2 * jm + 1);
      uint32_t D[4][4] = {{(uint32_t)inv2, 0, (uint32_t)inv2, 0},
                          {0, (uint32_t)inv2, 0, (uint32_t)inv2},
                          {(uint32_t)tw, 0, (uint32_t)((q - tw) % q), 0},
                          {0, (uint32_t)tw, 0, (uint32_t)((q - tw) % q)}};
      for (int k = 0; k < 4; k++)
        for (int t = 0; t < 4; t++) P->key_D[s][k][t] = D[k][t];
    }
  }

  P->chal_table.resize(N162 * N162);
  for (int p = 0; p < N162; p++)
    for (int j = 0; j < N162; j++) {
      uint64_t x = pow_mod(P->theta_leaf[j], p, q);
      if (p % 2) x = (q - x) % q;
      P->chal_table[p * N162 + j] = (uint32_t)x;
    }
  return P;
}

const PrimeTables& prime_tables(uint32_t q) {
  static std::mutex mu;
  static PrimeTables* cache[7] = {nullptr};
  int i = prime_index(q);
  if (i < 0) throw std::runtime_error("unsupported prime");
  std::lock_guard<std::mutex> g(mu);
  if (!cache[i]) cache[i] = build_prime(q);
  return *cache[i];
}

// crates/pcs/src/rng.rs:11-17: x ^= x >> 12; x ^= x << 25; x ^= x >> 27 is GF(2)-linear.
static uint64_t xs_step(uint64_t x) {
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  return x;
}
static uint64_t apply_cols(const uint64_t* M, uint64_t s) {
  uint64_t r = 0;
  for (int c = 0; c < 64; c++)
    if ((s >> c) & 1) r ^= M[c];
  return r;
}

const std::vector<uint64_t>& xorshift_jumps() {
  static std::vector<uint64_t> J = [] {
    std::vector<uint64_t> j(64 * 64);
    for (int c = 0; c < 64; c++) j[c] = xs_step(1ull << c);
    for (int k = 1; k < 64; k++)
      for (int c = 0; c < 64; c++) j[k * 64 + c] = apply_cols(&j[(k - 1) * 64], j[(k - 1) * 64 + c]);
    return j;
  }();
  return J;
}

void tc_transform_operand(const PrimeTables& T, uint8_t* out) {
  for (int i = 0; i < TC_B_BYTES; i++) out[i] = 0;
  for (int v = 0; v < N162; v++) {
    uint64_t x = 1;
    for (int m = 0; m < N162; m++) {
      const uint32_t t = (uint32_t)x;
      const int lo_kb = m, hi_kb = 192 + m;
      out[tc_swizzled_offset(v, lo_kb, TC_LEAVES)] = (uint8_t)(t & 127u);
      out[tc_swizzled_offset(v, hi_kb, TC_LEAVES)] = (uint8_t)(t >> 7);
      x = x * T.theta_leaf[v] % T.q;
    }
  }
}

}  // namespace lbg
