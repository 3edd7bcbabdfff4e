#include "transcript.h"

#include <cmath>
#include <cstring>
#include <mutex>

namespace lbg {

static void le64(uint64_t x, uint8_t b[8]) {
  for (int i = 0; i < 8; i++) b[i] = (uint8_t)(x >> (8 * i));
}

Transcript::Transcript(const uint8_t* domain, size_t len) {
  uint8_t b[8];
  le64(len, b);
  state_.update(b, 8);
  state_.update(domain, len);
}

void Transcript::absorb_bytes(const uint8_t* data, size_t len) {
  uint8_t b[8];
  le64(len, b);
  state_.update(b, 8);
  state_.update(data, len);
}

void Transcript::absorb_u64(uint64_t x) {
  uint8_t b[8];
  le64(x, b);
  state_.update(b, 8);
}

// A derivation: the absorbing state, then the sample counter, the label length and the label.
Blake3 Transcript::derive(const char* label) {
  Blake3 h = state_;
  uint8_t b[8];
  le64(counter_, b);
  h.update(b, 8);
  size_t n = std::strlen(label);
  le64(n, b);
  h.update(b, 8);
  h.update(label, n);
  counter_++;
  return h;
}

void Transcript::fill(const char* label, uint8_t* out, size_t n) {
  Blake3 h = derive(label);
  h.finalize(0, out, n);
}

void Transcript::absorb_b128(const uint64_t* words, size_t n) {
  uint8_t b[8];
  le64(n, b);
  state_.update(b, 8);
  for (size_t i = 0; i < 2 * n; i++) {
    le64(words[i], b);
    state_.update(b, 8);
  }
}

void Transcript::absorb_f162(const uint64_t* words, size_t n) {
  uint8_t b[8];
  le64(n, b);
  state_.update(b, 8);
  for (size_t i = 0; i < 3 * n; i++) {
    le64(words[i], b);
    state_.update(b, 8);
  }
}

void Transcript::sample_f162(const char* label, uint64_t* out, size_t n) {
  std::vector<uint8_t> bytes(24 * n);
  fill(label, bytes.data(), bytes.size());
  for (size_t i = 0; i < n; i++) {
    std::memcpy(out + 3 * i, bytes.data() + 24 * i, 24);
    out[3 * i + 2] &= (1ull << 34) - 1;
  }
}

// ---------------------------------------------------------------------------------------------
// the sampler
// ---------------------------------------------------------------------------------------------
namespace {

struct Phase {
  double re[162][81];
  double im[162][81];
};

// exp(2 pi i p u_k / 243) for the first 81 units u_k (crates/pcs/src/challenge.rs:329-360).
const Phase& phase() {
  static Phase* ph = [] {
    Phase* p = new Phase();
    int units[81], n = 0;
    for (int x = 1; n < 81; x++)
      if (x % 3) units[n++] = x;
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < 162; k++)
      for (int j = 0; j < 81; j++) {
        int m = (k * units[j]) % 243;
        volatile double two_pi = 2.0 * pi;
        double angle = two_pi * (double)m;
        angle = angle / 243.0;
        p->re[k][j] = std::cos(angle);
        p->im[k][j] = std::sin(angle);
      }
    return p;
  }();
  return *ph;
}

// max_u |c(zeta^u)|^2 <= bound_sq, term by term in position order with the reference's f64
// operation order (crates/pcs/src/challenge.rs:362-419).
bool within(const Challenge& c, double bound_sq) {
  const Phase& P = phase();
  for (int j = 0; j < 81; j++) {
    double vr = 0.0, vi = 0.0;
    for (uint32_t i = 0; i < c.weight; i++) {
      int p = c.positions[i];
      bool neg = (c.signs >> i) & 1;
      vr = vr + (neg ? -P.re[p][j] : P.re[p][j]);
      vi = vi + (neg ? -P.im[p][j] : P.im[p][j]);
    }
    volatile double a = vr * vr;
    volatile double b = vi * vi;
    double x = a + b;
    if (x > bound_sq) return false;
  }
  return true;
}

const Blake3& signs_hasher() {
  static const Blake3 key = Blake3::derive_key("labinius 2026 challenge signs v1");
  return key;
}

// keyed-by-context hash of the position set (crates/pcs/src/challenge.rs:237-269)
uint32_t signs_of(const Challenge& c) {
  Blake3 h = signs_hasher();
  uint8_t b[8];
  le64(c.weight, b);
  h.update(b, 8);
  h.update(c.positions, c.weight);
  uint8_t d[4];
  h.finalize(0, d, 4);
  uint32_t bits = (uint32_t)d[0] | ((uint32_t)d[1] << 8) | ((uint32_t)d[2] << 16) | ((uint32_t)d[3] << 24);
  return bits & (uint32_t)((1ull << c.weight) - 1);
}

// rejection sampling below n from little-endian u16s (crates/pcs/src/challenge.rs:197-221)
uint16_t below(Blake3Reader& x, uint16_t n) {
  uint32_t limit = (65536u / n) * n;
  uint64_t magic = (1ull << 32) / n + 1;
  for (;;) {
    uint32_t lo = x.byte();
    uint32_t hi = x.byte();
    uint32_t r = lo | (hi << 8);
    if (r < limit) return (uint16_t)(r - (uint32_t)(((uint64_t)r * magic) >> 32) * n);
  }
}

}  // namespace

const double* sampler_phase_re() { return &phase().re[0][0]; }
const double* sampler_phase_im() { return &phase().im[0][0]; }
const uint32_t* sampler_signs_key() { return signs_hasher().key_words(); }

Challenge sample_short_challenge(Transcript& t, uint32_t weight, double bound, uint64_t* attempts) {
  volatile double b2 = bound * bound;
  double bound_sq = b2 + 1e-12;
  Blake3Reader x(t.derive("short-challenge"));
  uint64_t n_att = 0;
  for (;;) {
    n_att++;
    uint8_t perm[162];
    for (int i = 0; i < 162; i++) perm[i] = (uint8_t)i;
    for (uint32_t i = 0; i < weight; i++) {
      uint32_t j = i + below(x, (uint16_t)(162 - i));
      uint8_t tmp = perm[i];
      perm[i] = perm[j];
      perm[j] = tmp;
    }
    uint64_t seen[3] = {0, 0, 0};
    for (uint32_t i = 0; i < weight; i++) seen[perm[i] >> 6] |= 1ull << (perm[i] & 63);
    Challenge c;
    std::memset(&c, 0, sizeof(c));
    c.weight = weight;
    int n = 0;
    for (int w = 0; w < 3; w++)
      for (uint64_t b = seen[w]; b; b &= b - 1) c.positions[n++] = (uint8_t)(64 * w + __builtin_ctzll(b));
    c.signs = signs_of(c);
    if (within(c, bound_sq)) {
      if (attempts) *attempts = n_att;
      return c;
    }
  }
}

uint32_t residue_bits(uint32_t q) { return 32 - __builtin_clz(q - 1); }
uint32_t top_bits(uint32_t q, uint32_t d) {
  uint32_t bound = ((q - 1) + (1u << (d - 1))) >> d;
  return 32 - __builtin_clz(bound);
}

std::vector<uint8_t> pack_dropped(const RoundShape& s, const uint16_t* top, const uint16_t* digits) {
  std::vector<uint8_t> out;
  size_t count = s.columns() * 648;
  uint32_t tb = top_bits(s.primes[0], s.dropped_bits);
  uint32_t bits_per = tb;
  for (uint32_t k = 1; k < s.limbs; k++) bits_per += residue_bits(s.primes[k]);
  out.reserve((count * bits_per + 7) / 8);
  uint64_t acc = 0;
  uint32_t n = 0;
  auto put = [&](uint64_t v, uint32_t bits) {
    acc |= (v & ((1ull << bits) - 1)) << n;
    n += bits;
    while (n >= 8) {
      out.push_back((uint8_t)acc);
      acc >>= 8;
      n -= 8;
    }
  };
  for (size_t i = 0; i < count; i++) {
    put(top[i], tb);
    for (uint32_t k = 1; k < s.limbs; k++) put(digits[(k - 1) * count + i], residue_bits(s.primes[k]));
  }
  if (n > 0) out.push_back((uint8_t)acc);
  return out;
}

void absorb_commitment_header(const RoundShape& s, Transcript& t) {
  t.absorb_bytes((const uint8_t*)"labinius/parameters", 19);
  t.absorb_u64(s.witness_log_len);
  t.absorb_u64(s.column_log_len);
  for (uint32_t k = 0; k < s.limbs; k++) t.absorb_u64(s.primes[k]);
  t.absorb_u64(0);  // no recursion on this path
  if (s.dropped_bits > 0) {
    t.absorb_bytes((const uint8_t*)"labinius/dropped-bits", 21);
    t.absorb_u64(s.dropped_bits);
  }
  t.absorb_bytes(s.matrix_seed, 32);
  t.absorb_bytes((const uint8_t*)"labinius/commitment", 19);
  t.absorb_u64(s.columns());
  if (s.dropped_bits > 0) t.absorb_bytes((const uint8_t*)"labinius/dropped-commitment", 27);
}

void evaluation_point_from(const RoundShape& s, Transcript& t, uint64_t* p0, uint64_t* p1) {
  size_t rows = s.row_log_len(), cols = s.column_log_len;
  std::vector<uint8_t> bytes(24 * (rows + cols));
  t.fill("labinius/evaluation-point", bytes.data(), bytes.size());
  for (size_t i = 0; i < rows + cols; i++) {
    uint64_t limb[3];
    std::memcpy(limb, bytes.data() + 24 * i, 24);
    limb[2] &= (1ull << 34) - 1;
    uint64_t* dst = i < rows ? p0 + 3 * i : p1 + 3 * (i - rows);
    std::memcpy(dst, limb, 24);
  }
}

void derive_evaluation_point(const RoundShape& s, Transcript& t, const int16_t* matrix,
                             const uint16_t* top, const uint16_t* digits, uint64_t* p0, uint64_t* p1) {
  absorb_commitment_header(s, t);
  if (s.dropped_bits == 0) {
    // absorb_elements per column: the element count (4), then each element's limbs as LE i16
    size_t per_col = 4 * (size_t)s.limbs * 162;
    for (size_t j = 0; j < s.columns(); j++) {
      t.absorb_u64(4);
      t.absorb_raw((const uint8_t*)(matrix + j * per_col), per_col * 2);  // little-endian host
    }
  } else {
    std::vector<uint8_t> b = pack_dropped(s, top, digits);
    t.absorb_bytes(b.data(), b.size());
  }
  evaluation_point_from(s, t, p0, p1);
}

void derive_folding_challenges(const RoundShape& s, Transcript& t, const uint64_t* u, Challenge* out) {
  t.absorb_bytes((const uint8_t*)"labinius/row-evaluation", 23);
  t.absorb_bytes((const uint8_t*)u, 24 * s.columns());
  for (size_t j = 0; j < s.columns(); j++) out[j] = sample_short_challenge(t, 28, 12.0, nullptr);
}

}  // namespace lbg
