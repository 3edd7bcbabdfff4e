// Host side of the round: the Fiat-Shamir transcript, the short-challenge sampler and the
// absorb/derive steps of the verifier. These stay on the host (they are sequential BLAKE3 work
// and must reproduce the reference's transcript bytes); the GPU path consumes their outputs.
#pragma once
#include <cstdint>
#include <vector>

#include "blake3_host.h"

namespace lbg {

// crates/pcs/src/challenge.rs:227-235 (positions sorted, signs bit i = -1 at positions[i]).
struct Challenge {
  uint8_t positions[32];
  uint32_t signs;
  uint32_t weight;
};
static_assert(sizeof(Challenge) == 40, "lbg_challenge layout");

// crates/pcs/src/challenge.rs:66-161
class Transcript {
 public:
  explicit Transcript(const uint8_t* domain, size_t len);
  void absorb_bytes(const uint8_t* b, size_t len);
  void absorb_u64(uint64_t x);
  void absorb_raw(const uint8_t* b, size_t len) { state_.update(b, len); }
  void fill(const char* label, uint8_t* out, size_t n);
  // absorb_b128 / absorb_f162 (crates/pcs/src/challenge.rs:113-127): the count, then each value's
  // little-endian words (2 per B128, 3 per F162).
  void absorb_b128(const uint64_t* words, size_t n);
  void absorb_f162(const uint64_t* words, size_t n);
  // sample_f162 (crates/pcs/src/challenge.rs:129-140): n F162, three LE words each, the top one
  // cut to 34 bits.
  void sample_f162(const char* label, uint64_t* out, size_t n);
  Blake3 derive(const char* label);
  // The absorbing state and the derivation counter, for moving the transcript to the device.
  const Blake3& state() const { return state_; }
  Blake3& state() { return state_; }
  uint64_t counter() const { return counter_; }
  void set_counter(uint64_t c) { counter_ = c; }

 private:
  Blake3 state_;
  uint64_t counter_ = 0;
};

// The sampler's tables for the device copy of it: exp(2 pi i p u_k / 243) as re/im [162][81]
// doubles, and the context key (8 words) of the sign hash.
const double* sampler_phase_re();
const double* sampler_phase_im();
const uint32_t* sampler_signs_key();

// crates/pcs/src/challenge.rs:517-533
Challenge sample_short_challenge(Transcript& t, uint32_t weight, double bound, uint64_t* attempts);

// The round shape the host steps need (crates/pcs/src/scheme/params.rs:62-68).
struct RoundShape {
  uint32_t witness_log_len, column_log_len, limbs, dropped_bits;
  uint32_t primes[8];
  uint8_t matrix_seed[32];
  size_t columns() const { return (size_t)1 << column_log_len; }
  uint32_t row_log_len() const { return witness_log_len - column_log_len; }
};

// The steps of derive_evaluation_point (crates/pcs/src/scheme/verifier.rs:41-100):
// the parameters and the commitment's framing (everything up to the commitment's own bytes) ...
void absorb_commitment_header(const RoundShape& s, Transcript& t);
// ... and, once the commitment's bytes are absorbed, the point itself.
void evaluation_point_from(const RoundShape& s, Transcript& t, uint64_t* p0, uint64_t* p1);
// crates/pcs/src/scheme/verifier.rs:41-100
void derive_evaluation_point(const RoundShape& s, Transcript& t, const int16_t* matrix,
                             const uint16_t* top, const uint16_t* digits, uint64_t* p0, uint64_t* p1);
// crates/pcs/src/scheme/commitment.rs:217-229, 320-331
void derive_folding_challenges(const RoundShape& s, Transcript& t, const uint64_t* u, Challenge* out);
// crates/pcs/src/wire/mod.rs:386-397
std::vector<uint8_t> pack_dropped(const RoundShape& s, const uint16_t* top, const uint16_t* digits);
uint32_t top_bits(uint32_t q, uint32_t dropped_bits);
uint32_t residue_bits(uint32_t q);

}  // namespace lbg
