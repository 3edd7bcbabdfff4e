// TEST INFRASTRUCTURE (oracle): an all-in-memory BLAKE3 written from the public BLAKE3
// specification (compression function, chunk chaining, binary tree of parents, keyed and
// derive-key modes, extendable output with seek). It exists only to check the product's own
// incremental BLAKE3 and transcript, and it is itself checked against the Python `blake3`
// package in tests/test_oracle_blake3.py.
//
// The reference (osdnk/labinius) uses the `blake3` crate 1.8.7 (Cargo.lock) for
// `PublicParameters::from_seed` (crates/pcs/src/scheme/params.rs:320-322), `Witness::random`
// (crates/pcs/src/scheme/witness.rs:66-87) and the Fiat-Shamir transcript
// (crates/pcs/src/challenge.rs:66-161). That crate is not vendored in the reference tree; this
// file restates the published algorithm.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

enum : uint32_t {
  B3_CHUNK_START = 1,
  B3_CHUNK_END = 2,
  B3_PARENT = 4,
  B3_ROOT = 8,
  B3_KEYED_HASH = 16,
  B3_DERIVE_KEY_CONTEXT = 32,
  B3_DERIVE_KEY_MATERIAL = 64,
};

static const uint32_t B3_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const int B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

inline uint32_t b3_rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

inline void b3_g(uint32_t* s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
  s[a] = s[a] + s[b] + mx;
  s[d] = b3_rotr(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];
  s[b] = b3_rotr(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + my;
  s[d] = b3_rotr(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];
  s[b] = b3_rotr(s[b] ^ s[c], 7);
}

// The full 16-word output of one compression.
inline void b3_compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter,
                        uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t s[16];
  for (int i = 0; i < 8; i++) s[i] = cv[i];
  for (int i = 0; i < 4; i++) s[8 + i] = B3_IV[i];
  s[12] = (uint32_t)counter;
  s[13] = (uint32_t)(counter >> 32);
  s[14] = block_len;
  s[15] = flags;
  uint32_t m[16];
  for (int i = 0; i < 16; i++) m[i] = block[i];
  for (int r = 0; r < 7; r++) {
    b3_g(s, 0, 4, 8, 12, m[0], m[1]);
    b3_g(s, 1, 5, 9, 13, m[2], m[3]);
    b3_g(s, 2, 6, 10, 14, m[4], m[5]);
    b3_g(s, 3, 7, 11, 15, m[6], m[7]);
    b3_g(s, 0, 5, 10, 15, m[8], m[9]);
    b3_g(s, 1, 6, 11, 12, m[10], m[11]);
    b3_g(s, 2, 7, 8, 13, m[12], m[13]);
    b3_g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; i++) t[i] = m[B3_PERM[i]];
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
  }
  for (int i = 0; i < 8; i++) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}

inline void b3_load_block(const uint8_t* p, size_t len, uint32_t w[16]) {
  uint8_t buf[64];
  std::memset(buf, 0, 64);
  if (len) std::memcpy(buf, p, len);
  for (int i = 0; i < 16; i++)
    w[i] = (uint32_t)buf[4 * i] | ((uint32_t)buf[4 * i + 1] << 8) |
           ((uint32_t)buf[4 * i + 2] << 16) | ((uint32_t)buf[4 * i + 3] << 24);
}

// The last compression of a node, not yet performed: what the root output (or a chaining value)
// is computed from.
struct B3Node {
  uint32_t cv[8];
  uint32_t block[16];
  uint64_t counter;
  uint32_t block_len;
  uint32_t flags;
  void chaining_value(uint32_t out8[8]) const {
    uint32_t o[16];
    b3_compress(cv, block, counter, block_len, flags, o);
    for (int i = 0; i < 8; i++) out8[i] = o[i];
  }
};

inline B3Node b3_chunk(const uint32_t key[8], const uint8_t* data, size_t len,
                       uint64_t chunk_counter, uint32_t flags) {
  size_t nblocks = len == 0 ? 1 : (len + 63) / 64;
  uint32_t cv[8];
  for (int i = 0; i < 8; i++) cv[i] = key[i];
  for (size_t b = 0; b + 1 < nblocks; b++) {
    uint32_t w[16], o[16];
    b3_load_block(data + 64 * b, 64, w);
    b3_compress(cv, w, chunk_counter, 64, flags | (b == 0 ? B3_CHUNK_START : 0), o);
    for (int i = 0; i < 8; i++) cv[i] = o[i];
  }
  B3Node n;
  for (int i = 0; i < 8; i++) n.cv[i] = cv[i];
  size_t last = len - 64 * (nblocks - 1);
  b3_load_block(data + 64 * (nblocks - 1), last, n.block);
  n.counter = chunk_counter;
  n.block_len = (uint32_t)last;
  n.flags = flags | (nblocks == 1 ? B3_CHUNK_START : 0) | B3_CHUNK_END;
  return n;
}

// The subtree over `len` bytes starting at chunk `chunk0`: a chunk when it fits in 1024 bytes,
// otherwise a parent whose left child holds the largest power of two number of chunks that
// leaves the right child non-empty.
inline B3Node b3_subtree(const uint32_t key[8], const uint8_t* data, size_t len, uint64_t chunk0,
                         uint32_t flags) {
  if (len <= 1024) return b3_chunk(key, data, len, chunk0, flags);
  size_t nchunks = (len + 1023) / 1024;
  size_t left_chunks = 1;
  while (left_chunks * 2 < nchunks) left_chunks *= 2;
  size_t left_len = left_chunks * 1024;
  uint32_t l[8], r[8];
  b3_subtree(key, data, left_len, chunk0, flags).chaining_value(l);
  b3_subtree(key, data + left_len, len - left_len, chunk0 + left_chunks, flags).chaining_value(r);
  B3Node n;
  for (int i = 0; i < 8; i++) {
    n.cv[i] = key[i];
    n.block[i] = l[i];
    n.block[8 + i] = r[i];
  }
  n.counter = 0;
  n.block_len = 64;
  n.flags = flags | B3_PARENT;
  return n;
}

// Extendable output of the root node, bytes [seek, seek + out_len).
inline void b3_root_output(const B3Node& root, uint64_t seek, uint8_t* out, size_t out_len) {
  uint64_t block = seek / 64;
  size_t skip = (size_t)(seek % 64);
  size_t done = 0;
  while (done < out_len) {
    uint32_t o[16];
    b3_compress(root.cv, root.block, block, root.block_len, root.flags | B3_ROOT, o);
    uint8_t bytes[64];
    for (int i = 0; i < 16; i++) {
      bytes[4 * i] = (uint8_t)o[i];
      bytes[4 * i + 1] = (uint8_t)(o[i] >> 8);
      bytes[4 * i + 2] = (uint8_t)(o[i] >> 16);
      bytes[4 * i + 3] = (uint8_t)(o[i] >> 24);
    }
    for (size_t i = skip; i < 64 && done < out_len; i++) out[done++] = bytes[i];
    skip = 0;
    block++;
  }
}

inline void b3_key_words(const uint8_t key[32], uint32_t w[8]) {
  for (int i = 0; i < 8; i++)
    w[i] = (uint32_t)key[4 * i] | ((uint32_t)key[4 * i + 1] << 8) |
           ((uint32_t)key[4 * i + 2] << 16) | ((uint32_t)key[4 * i + 3] << 24);
}

// mode 0: plain hash; 1: keyed (key = 32 bytes); 2: derive_key (key = context bytes, ctx_len).
inline void b3_xof(int mode, const uint8_t* key, size_t ctx_len, const uint8_t* data, size_t len,
                   uint64_t seek, uint8_t* out, size_t out_len) {
  uint32_t kw[8];
  uint32_t flags = 0;
  if (mode == 0) {
    for (int i = 0; i < 8; i++) kw[i] = B3_IV[i];
  } else if (mode == 1) {
    b3_key_words(key, kw);
    flags = B3_KEYED_HASH;
  } else {
    B3Node ctx = b3_subtree(B3_IV, key, ctx_len, 0, B3_DERIVE_KEY_CONTEXT);
    uint8_t ck[32];
    b3_root_output(ctx, 0, ck, 32);
    b3_key_words(ck, kw);
    flags = B3_DERIVE_KEY_MATERIAL;
  }
  B3Node root = b3_subtree(kw, data, len, 0, flags);
  b3_root_output(root, seek, out, out_len);
}

}  // namespace orc
