// The state of an incremental BLAKE3 hasher as plain data, shared by the host hasher and the
// device transcript kernels so a transcript can move between them.
//
// Both sides keep it in one canonical form after every update: with `total` bytes absorbed
// (total >= 1), chunk_counter = (total - 1) / 1024 chunks are complete and their subtrees are
// merged by the chunk count (one stack entry per set bit of chunk_counter, largest subtree first);
// the current chunk holds the remaining 1..1024 bytes, of which the last 1..64 are buffered
// uncompressed (buf_len) and the `blocks` 64-byte blocks before them are folded into cv.
#pragma once
#include <cstdint>

namespace lbg {

struct HasherState {
  uint32_t key[8];
  uint32_t flags;
  uint32_t cv[8];
  uint8_t buf[64];
  uint32_t buf_len;
  uint32_t blocks;
  uint64_t chunk_counter;
  uint32_t stack[54][8];
  uint32_t stack_len;
  uint32_t pad_;
};

namespace b3 {
constexpr uint32_t CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8, KEYED_HASH = 16,
                   DERIVE_KEY_CONTEXT = 32, DERIVE_KEY_MATERIAL = 64;
}  // namespace b3

// Bytes absorbed so far by a hasher in the canonical form.
inline uint64_t absorbed_len(const HasherState& s) {
  return s.chunk_counter * 1024 + (uint64_t)s.blocks * 64 + s.buf_len;
}

}  // namespace lbg
