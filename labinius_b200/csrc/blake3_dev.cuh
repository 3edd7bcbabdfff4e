// Device BLAKE3 (written from the public BLAKE3 specification, the algorithm of the `blake3` crate
// 1.8.7 the reference uses, Cargo.lock:665-668): the compression function with the message
// permutation applied in registers, and a derivation on top of a read-only hasher state (the
// transcript's derive(): clone, append a few bytes, finalize as an extendable output).
#pragma once
#include <cstdint>

#include "hasher_state.h"
#include "launch.h"

namespace lbg {
namespace dev {

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

__device__ __forceinline__ void mix(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t x, uint32_t y) {
  a = a + b + x;
  d = rotr(d ^ a, 16);
  c = c + d;
  b = rotr(b ^ c, 12);
  a = a + b + y;
  d = rotr(d ^ a, 8);
  c = c + d;
  b = rotr(b ^ c, 7);
}

// One compression of a 64-byte block (16 little-endian words): 16 output words; the first 8 are
// the chaining value.
__device__ __forceinline__ void compress(const uint32_t cv[8], const uint32_t msg[16], uint64_t counter,
                                         uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t s0 = cv[0], s1 = cv[1], s2 = cv[2], s3 = cv[3], s4 = cv[4], s5 = cv[5], s6 = cv[6], s7 = cv[7];
  uint32_t s8 = 0x6A09E667u, s9 = 0xBB67AE85u, s10 = 0x3C6EF372u, s11 = 0xA54FF53Au;
  uint32_t s12 = (uint32_t)counter, s13 = (uint32_t)(counter >> 32), s14 = block_len, s15 = flags;
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = msg[i];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    mix(s0, s4, s8, s12, m[0], m[1]);
    mix(s1, s5, s9, s13, m[2], m[3]);
    mix(s2, s6, s10, s14, m[4], m[5]);
    mix(s3, s7, s11, s15, m[6], m[7]);
    mix(s0, s5, s10, s15, m[8], m[9]);
    mix(s1, s6, s11, s12, m[10], m[11]);
    mix(s2, s7, s8, s13, m[12], m[13]);
    mix(s3, s4, s9, s14, m[14], m[15]);
    if (r < 6) {  // the spec's message permutation
      uint32_t t[16] = {m[2], m[6], m[3], m[10], m[7], m[0], m[4], m[13],
                        m[1], m[11], m[12], m[5], m[9], m[14], m[15], m[8]};
#pragma unroll
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
  }
  out[0] = s0 ^ s8;
  out[1] = s1 ^ s9;
  out[2] = s2 ^ s10;
  out[3] = s3 ^ s11;
  out[4] = s4 ^ s12;
  out[5] = s5 ^ s13;
  out[6] = s6 ^ s14;
  out[7] = s7 ^ s15;
  out[8] = s8 ^ cv[0];
  out[9] = s9 ^ cv[1];
  out[10] = s10 ^ cv[2];
  out[11] = s11 ^ cv[3];
  out[12] = s12 ^ cv[4];
  out[13] = s13 ^ cv[5];
  out[14] = s14 ^ cv[6];
  out[15] = s15 ^ cv[7];
}

// parent node of two chaining values (no ROOT flag): the merged chaining value
__device__ __forceinline__ void parent_cv(const uint32_t key[8], uint32_t flags, const uint32_t l[8], const uint32_t r[8],
                                          uint32_t out[8]) {
  uint32_t m[16], o[16];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    m[i] = l[i];
    m[8 + i] = r[i];
  }
  compress(key, m, 0, 64, flags | b3::PARENT, o);
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = o[i];
}

__device__ __forceinline__ void bytes_to_words(const uint8_t* b, uint32_t* w, int n) {
  for (int i = 0; i < n; i++)
    w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
           ((uint32_t)b[4 * i + 3] << 24);
}

// One out-of-line copy of the compression for the single-thread transcript steps below: their
// kernels run it a handful of times per launch, and one shared copy of its code stays in the
// instruction cache where a copy inlined at every call site would be fetched cold each time.
static __device__ __noinline__ void compress_ool(const uint32_t cv[8], const uint32_t msg[16], uint64_t counter,
                                                 uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  compress(cv, msg, counter, block_len, flags, out);
}
static __device__ __forceinline__ void parent_cv_ool(const uint32_t key[8], uint32_t flags, const uint32_t l[8],
                                                     const uint32_t r[8], uint32_t out[8]) {
  uint32_t m[16], o[16];
  for (int i = 0; i < 8; i++) {
    m[i] = l[i];
    m[8 + i] = r[i];
  }
  compress_ool(key, m, 0, 64, flags | b3::PARENT, o);
  for (int i = 0; i < 8; i++) out[i] = o[i];
}
static __device__ __forceinline__ void root_block_ool(const XofRoot& r, uint64_t t, uint32_t out[16]) {
  compress_ool(r.cv, r.m, t, r.block_len, r.flags | b3::ROOT, out);
}

// Output block t of a finalized hasher (its root node): 64 bytes as 16 words.
__device__ __forceinline__ void root_block(const XofRoot& r, uint64_t t, uint32_t out[16]) {
  compress(r.cv, r.m, t, r.block_len, r.flags | b3::ROOT, out);
}

// A derivation on top of a read-only base state: the base's stack stays where it is, merges
// consume its entries from the top, and new subtrees go to a small local stack.
struct Tail {
  const HasherState* base;
  uint32_t base_len;
  uint32_t extra[4][8];
  uint32_t n_extra;
  uint32_t key[8];
  uint32_t flags;
  uint32_t cv[8];
  uint8_t buf[64];
  uint32_t buf_len;
  uint32_t blocks;
  uint64_t chunk_counter;

  __device__ void init(const HasherState* s) {
    base = s;
    base_len = s->stack_len < 54 ? s->stack_len : 54;
    n_extra = 0;
    for (int i = 0; i < 8; i++) {
      key[i] = s->key[i];
      cv[i] = s->cv[i];
    }
    flags = s->flags;
    for (int i = 0; i < 64; i++) buf[i] = s->buf[i];
    buf_len = s->buf_len;
    blocks = s->blocks;
    chunk_counter = s->chunk_counter;
  }

  __device__ void compress_buf(uint32_t fl, uint32_t out[16]) {
    uint32_t m[16];
    bytes_to_words(buf, m, 16);
    compress(cv, m, chunk_counter, 64, fl, out);
  }

  // merge while the chunk count has trailing zero bits, then push (the host hasher's rule)
  __device__ void push_cv(const uint32_t in[8], uint64_t total_chunks) {
    uint32_t cur[8];
    for (int i = 0; i < 8; i++) cur[i] = in[i];
    while ((total_chunks & 1) == 0) {
      if (n_extra > 0) {
        n_extra--;
        parent_cv(key, flags, extra[n_extra], cur, cur);
      } else if (base_len > 0) {
        base_len--;
        parent_cv(key, flags, base->stack[base_len], cur, cur);
      } else {
        break;  // not a canonical state: nothing left to merge with
      }
      total_chunks >>= 1;
    }
    if (n_extra == 4) return;  // more than this derivation appends
    for (int i = 0; i < 8; i++) extra[n_extra][i] = cur[i];
    n_extra++;
  }

  __device__ void update(const uint8_t* p, uint32_t len) {
    while (len > 0) {
      if (blocks == 15 && buf_len == 64) {
        uint32_t o[16];
        compress_buf(flags | b3::CHUNK_END, o);
        chunk_counter++;
        push_cv(o, chunk_counter);
        for (int i = 0; i < 8; i++) cv[i] = key[i];
        buf_len = 0;
        blocks = 0;
      }
      if (buf_len == 64) {
        uint32_t o[16];
        compress_buf(flags | (blocks == 0 ? b3::CHUNK_START : 0), o);
        for (int i = 0; i < 8; i++) cv[i] = o[i];
        blocks++;
        buf_len = 0;
      }
      uint32_t take = 64 - buf_len;
      if (take > len) take = len;
      for (uint32_t i = 0; i < take; i++) buf[buf_len + i] = p[i];
      buf_len += take;
      p += take;
      len -= take;
    }
  }

  __device__ void update_u64(uint64_t x) {
    uint8_t b[8];
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(x >> (8 * i));
    update(b, 8);
  }

  // the root node: the current chunk's last block, then parents up the stack
  __device__ void root(XofRoot& r) {
    uint8_t blk[64];
    for (int i = 0; i < 64; i++) blk[i] = i < (int)buf_len ? buf[i] : 0;
    uint32_t m[16];
    bytes_to_words(blk, m, 16);
    uint32_t c[8];
    for (int i = 0; i < 8; i++) c[i] = cv[i];
    uint32_t block_len = buf_len;
    uint64_t counter = chunk_counter;
    uint32_t fl = flags | b3::CHUNK_END | (blocks == 0 ? b3::CHUNK_START : 0);
    int total = (int)(base_len + n_extra);
    for (int e = total - 1; e >= 0; e--) {
      uint32_t o[16];
      compress(c, m, counter, block_len, fl, o);
      const uint32_t* left = e >= (int)base_len ? extra[e - base_len] : base->stack[e];
      for (int i = 0; i < 8; i++) {
        m[i] = left[i];
        m[8 + i] = o[i];
        c[i] = key[i];
      }
      block_len = 64;
      counter = 0;
      fl = flags | b3::PARENT;
    }
    for (int i = 0; i < 8; i++) r.cv[i] = c[i];
    for (int i = 0; i < 16; i++) r.m[i] = m[i];
    r.block_len = block_len;
    r.flags = fl;
  }
};

// hs_copy moves a hasher state between device and shared memory with the whole block (the
// transcript steps of the switch work on a shared copy).
__device__ inline void hs_copy(HasherState* dst, const HasherState* src) {
  static_assert(sizeof(HasherState) % 4 == 0, "HasherState is copied as words");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(HasherState) / 4); i += blockDim.x) d[i] = s[i];
}

// Staged absorbs and derivations: the bytes to hash are first laid out by the whole block in a
// word-aligned shared buffer, `stage` = the state's open block (buf_len bytes) followed by the new
// bytes (`total` in all, zero-filled to the next 64-byte boundary); one thread then compresses
// whole 64-byte blocks read as words, so its sequential work is the compressions alone. The
// state keeps the canonical form of hasher_state.h, so the host and the parallel absorb kernels
// can continue from it.
//
// hs_absorb_staged: every block of the stage but the last (it stays open, 1..64 bytes) is
// compressed into s (in place, shared memory), completed chunks merged into its stack. Returns
// the offset of the last block; the caller copies it into s->buf and sets s->buf_len.
__device__ inline uint32_t hs_absorb_staged(HasherState* s, const uint32_t* stage, uint32_t total) {
  uint32_t off = 0;
  while (total - off > 64) {
    uint32_t m[16], o[16];
    for (int q = 0; q < 16; q++) m[q] = stage[off / 4 + q];
    if (s->blocks == 15) {
      compress_ool(s->cv, m, s->chunk_counter, 64, s->flags | b3::CHUNK_END, o);
      s->chunk_counter++;
      uint64_t chunks = s->chunk_counter;
      uint32_t cur[8];
      for (int i = 0; i < 8; i++) cur[i] = o[i];
      while ((chunks & 1) == 0 && s->stack_len > 0) {
        s->stack_len--;
        parent_cv_ool(s->key, s->flags, s->stack[s->stack_len], cur, cur);
        chunks >>= 1;
      }
      if (s->stack_len < 54) {
        for (int i = 0; i < 8; i++) s->stack[s->stack_len][i] = cur[i];
        s->stack_len++;
      }
      for (int i = 0; i < 8; i++) s->cv[i] = s->key[i];
      s->blocks = 0;
    } else {
      compress_ool(s->cv, m, s->chunk_counter, 64, s->flags | (s->blocks == 0 ? b3::CHUNK_START : 0), o);
      for (int i = 0; i < 8; i++) s->cv[i] = o[i];
      s->blocks++;
    }
    off += 64;
  }
  return off;
}
// hs_absorb_staged by a whole block: the chunks the stage's compressed blocks fall in are
// compressed by one thread each (a chunk's blocks depend on one another, different chunks do
// not), then thread 0 folds the completed chunks into the stack in order, as hs_absorb_staged
// does one block at a time. cvs: shared scratch of 8 chaining values (a stage of at most
// 8 * 1024 - 64 bytes). Every thread calls it; it returns the offset of the last block to all.
__device__ inline uint32_t hs_absorb_staged_par(HasherState* s, const uint32_t* stage, uint32_t total,
                                                uint32_t (*cvs)[8]) {
  const uint32_t nb = (total + 63) / 64 - 1;  // every block but the last is compressed
  const uint32_t B = s->blocks;
  const uint32_t nch = nb == 0 ? 0 : (B + nb - 1) / 16 + 1;
  // chunk r of the absorb: stage blocks [q0, q1), chunk positions from p0
  auto span = [&](uint32_t r, uint32_t& q0, uint32_t& q1, uint32_t& p0) {
    p0 = r == 0 ? B : 0;
    q0 = r == 0 ? 0 : 16 * r - B;
    q1 = 16 * (r + 1) - B < nb ? 16 * (r + 1) - B : nb;
  };
  if (threadIdx.x < nch) {
    const uint32_t r = threadIdx.x;
    uint32_t q0, q1, p0, cv[8], m[16], o[16];
    span(r, q0, q1, p0);
    for (int i = 0; i < 8; i++) cv[i] = r == 0 ? s->cv[i] : s->key[i];
    for (uint32_t q = q0; q < q1; q++) {
      const uint32_t pos = p0 + (q - q0);
      for (int w = 0; w < 16; w++) m[w] = stage[q * 16 + w];
      const uint32_t fl = s->flags | (pos == 0 ? b3::CHUNK_START : 0) | (pos == 15 ? b3::CHUNK_END : 0);
      compress_ool(cv, m, s->chunk_counter + r, 64, fl, o);
      for (int i = 0; i < 8; i++) cv[i] = o[i];
    }
    for (int i = 0; i < 8; i++) cvs[r][i] = cv[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t r = 0; r < nch; r++) {
      uint32_t q0, q1, p0;
      span(r, q0, q1, p0);
      const uint32_t done = p0 + (q1 - q0);  // the chunk's compressed blocks
      if (done == 16) {
        s->chunk_counter++;
        uint64_t chunks = s->chunk_counter;
        uint32_t cur[8];
        for (int i = 0; i < 8; i++) cur[i] = cvs[r][i];
        while ((chunks & 1) == 0 && s->stack_len > 0) {
          s->stack_len--;
          parent_cv_ool(s->key, s->flags, s->stack[s->stack_len], cur, cur);
          chunks >>= 1;
        }
        if (s->stack_len < 54) {
          for (int i = 0; i < 8; i++) s->stack[s->stack_len][i] = cur[i];
          s->stack_len++;
        }
        for (int i = 0; i < 8; i++) s->cv[i] = s->key[i];
        s->blocks = 0;
      } else {
        for (int i = 0; i < 8; i++) s->cv[i] = cvs[r][i];
        s->blocks = done;
      }
    }
  }
  __syncthreads();
  return nb * 64;
}


// The root node of a derivation from s: stage = s's open block followed by the derivation's
// bytes (at most 128 bytes in all, so at most one chunk completes on the way). s is not changed.
__device__ inline void hs_derive_staged(const HasherState* s, const uint32_t* stage, uint32_t total, XofRoot& r) {
  uint32_t cv[8], extra[8];
  for (int i = 0; i < 8; i++) cv[i] = s->cv[i];
  uint32_t blocks = s->blocks, base_len = s->stack_len < 54 ? s->stack_len : 54;
  uint64_t chunks = s->chunk_counter;
  bool has_extra = false;
  uint32_t off = 0;
  while (total - off > 64) {
    uint32_t m[16], o[16];
    for (int q = 0; q < 16; q++) m[q] = stage[off / 4 + q];
    if (blocks == 15) {
      compress_ool(cv, m, chunks, 64, s->flags | b3::CHUNK_END, o);
      chunks++;
      uint64_t t = chunks;
      for (int i = 0; i < 8; i++) extra[i] = o[i];
      while ((t & 1) == 0 && base_len > 0) {
        base_len--;
        parent_cv_ool(s->key, s->flags, s->stack[base_len], extra, extra);
        t >>= 1;
      }
      has_extra = true;
      for (int i = 0; i < 8; i++) cv[i] = s->key[i];
      blocks = 0;
    } else {
      compress_ool(cv, m, chunks, 64, s->flags | (blocks == 0 ? b3::CHUNK_START : 0), o);
      for (int i = 0; i < 8; i++) cv[i] = o[i];
      blocks++;
    }
    off += 64;
  }
  uint32_t m[16];
  for (int q = 0; q < 16; q++) m[q] = stage[off / 4 + q];
  uint32_t block_len = total - off;
  uint64_t counter = chunks;
  uint32_t fl = s->flags | b3::CHUNK_END | (blocks == 0 ? b3::CHUNK_START : 0);
  int entries = (int)base_len + (has_extra ? 1 : 0);
  for (int e = entries - 1; e >= 0; e--) {
    uint32_t o[16];
    compress_ool(cv, m, counter, block_len, fl, o);
    const uint32_t* left = e >= (int)base_len ? extra : s->stack[e];
    for (int i = 0; i < 8; i++) {
      m[i] = left[i];
      m[8 + i] = o[i];
      cv[i] = s->key[i];
    }
    block_len = 64;
    counter = 0;
    fl = s->flags | b3::PARENT;
  }
  for (int i = 0; i < 8; i++) r.cv[i] = cv[i];
  for (int i = 0; i < 16; i++) r.m[i] = m[i];
  r.block_len = block_len;
  r.flags = fl;
}

// The transcript's derive(label) on a base state with derivation counter `counter`.
__device__ __forceinline__ void derive_root(const HasherState* st, uint64_t counter, const char* label, uint32_t len,
                                            XofRoot& r) {
  Tail t;
  t.init(st);
  t.update_u64(counter);
  t.update_u64(len);
  t.update((const uint8_t*)label, len);
  t.root(r);
}

// Sequential reader over a root node's output (the transcript's XOF stream).
struct Reader {
  XofRoot r;
  uint64_t block;
  uint32_t w[16];
  uint32_t off;
  __device__ void init(const XofRoot& root) {
    r = root;
    block = 0;
    off = 64;
  }
  __device__ uint32_t byte() {
    if (off == 64) {
      root_block(r, block++, w);
      off = 0;
    }
    uint32_t b = (w[off >> 2] >> (8 * (off & 3))) & 0xFF;
    off++;
    return b;
  }
};

}  // namespace dev
}  // namespace lbg
