// Incremental BLAKE3 for the host side of the prover: the Fiat-Shamir transcript, the key seed
// of PublicParameters::from_seed and the sign hash of the short challenges all go through it.
// Written from the public BLAKE3 specification (the reference uses the `blake3` crate 1.8.7,
// Cargo.lock:665-668): a chunk state, a stack of chaining values merged by the chunk counter,
// keyed and derive-key modes, and an extendable-output reader that can seek.
#pragma once
#include <cstddef>
#include <cstdint>

#include "hasher_state.h"

namespace lbg {

class Blake3 {
 public:
  Blake3();                                        // plain hash
  static Blake3 keyed(const uint8_t key[32]);      // keyed hash
  static Blake3 derive_key(const char* context);   // derive-key (context string, material follows)
  void update(const void* data, size_t len);
  // Extendable output of everything absorbed so far, bytes [seek, seek + len).
  void finalize(uint64_t seek, uint8_t* out, size_t len) const;
  // The state as plain data (canonical form, hasher_state.h) and back.
  void save(HasherState& s) const;
  void load(const HasherState& s);
  // The key words and mode flags (the context key of a derive-key hasher).
  const uint32_t* key_words() const { return key_; }
  uint32_t mode_flags() const { return flags_; }

 private:
  uint32_t key_[8];
  uint32_t flags_;
  // current chunk
  uint32_t cv_[8];
  uint8_t buf_[64];
  uint32_t buf_len_;
  uint32_t blocks_;
  uint64_t chunk_counter_;
  // completed subtree chaining values
  uint32_t stack_[54][8];
  uint32_t stack_len_;
  void push_cv(const uint32_t cv[8], uint64_t total_chunks);
  void init(const uint32_t key[8], uint32_t flags);
};

// A streaming reader over one finalised state (the XOF).
class Blake3Reader {
 public:
  explicit Blake3Reader(const Blake3& h) : h_(h), pos_(0), have_(0), off_(0) {}
  uint8_t byte();
  void read(uint8_t* out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = byte();
  }

 private:
  Blake3 h_;
  uint64_t pos_;
  uint8_t buf_[1024];
  size_t have_, off_;
};

}  // namespace lbg
