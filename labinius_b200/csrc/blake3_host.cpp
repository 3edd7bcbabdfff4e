#include "blake3_host.h"

#include <cstring>

namespace lbg {

namespace {
using namespace b3;
constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                            0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
// message word schedule of the seven rounds (the spec's permutation applied r times)
constexpr uint8_t SCHED[7][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8},
    {3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1},
    {10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6},
    {12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4},
    {9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7},
    {11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13},
};

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
inline void g(uint32_t* s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
  s[a] += s[b] + x;
  s[d] = rotr(s[d] ^ s[a], 16);
  s[c] += s[d];
  s[b] = rotr(s[b] ^ s[c], 12);
  s[a] += s[b] + y;
  s[d] = rotr(s[d] ^ s[a], 8);
  s[c] += s[d];
  s[b] = rotr(s[b] ^ s[c], 7);
}
void compress(const uint32_t cv[8], const uint8_t block[64], uint32_t block_len, uint64_t counter,
              uint32_t flags, uint32_t out[16]) {
  uint32_t m[16];
  for (int i = 0; i < 16; i++)
    m[i] = (uint32_t)block[4 * i] | ((uint32_t)block[4 * i + 1] << 8) |
           ((uint32_t)block[4 * i + 2] << 16) | ((uint32_t)block[4 * i + 3] << 24);
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    IV[0], IV[1], IV[2], IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                    block_len, flags};
  for (int r = 0; r < 7; r++) {
    const uint8_t* w = SCHED[r];
    g(s, 0, 4, 8, 12, m[w[0]], m[w[1]]);
    g(s, 1, 5, 9, 13, m[w[2]], m[w[3]]);
    g(s, 2, 6, 10, 14, m[w[4]], m[w[5]]);
    g(s, 3, 7, 11, 15, m[w[6]], m[w[7]]);
    g(s, 0, 5, 10, 15, m[w[8]], m[w[9]]);
    g(s, 1, 6, 11, 12, m[w[10]], m[w[11]]);
    g(s, 2, 7, 8, 13, m[w[12]], m[w[13]]);
    g(s, 3, 4, 9, 14, m[w[14]], m[w[15]]);
  }
  for (int i = 0; i < 8; i++) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}
void words_to_bytes(const uint32_t* w, int n, uint8_t* b) {
  for (int i = 0; i < n; i++) {
    b[4 * i] = (uint8_t)w[i];
    b[4 * i + 1] = (uint8_t)(w[i] >> 8);
    b[4 * i + 2] = (uint8_t)(w[i] >> 16);
    b[4 * i + 3] = (uint8_t)(w[i] >> 24);
  }
}
void bytes_to_words(const uint8_t* b, uint32_t* w) {
  for (int i = 0; i < 8; i++)
    w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
           ((uint32_t)b[4 * i + 3] << 24);
}
}  // namespace

void Blake3::init(const uint32_t key[8], uint32_t flags) {
  std::memcpy(key_, key, sizeof(key_));
  flags_ = flags;
  std::memcpy(cv_, key, sizeof(cv_));
  buf_len_ = 0;
  blocks_ = 0;
  chunk_counter_ = 0;
  stack_len_ = 0;
  std::memset(buf_, 0, sizeof(buf_));
}

Blake3::Blake3() { init(IV, 0); }

Blake3 Blake3::keyed(const uint8_t key[32]) {
  Blake3 h;
  uint32_t k[8];
  bytes_to_words(key, k);
  h.init(k, KEYED_HASH);
  return h;
}

Blake3 Blake3::derive_key(const char* context) {
  Blake3 c;
  c.init(IV, DERIVE_KEY_CONTEXT);
  c.update(context, std::strlen(context));
  uint8_t ck[32];
  c.finalize(0, ck, 32);
  Blake3 h;
  uint32_t k[8];
  bytes_to_words(ck, k);
  h.init(k, DERIVE_KEY_MATERIAL);
  return h;
}

// Merge completed subtrees while the chunk count has trailing zero bits, then push.
void Blake3::push_cv(const uint32_t cv[8], uint64_t total_chunks) {
  uint32_t cur[8];
  std::memcpy(cur, cv, sizeof(cur));
  while ((total_chunks & 1) == 0) {
    uint8_t block[64];
    words_to_bytes(stack_[stack_len_ - 1], 8, block);
    words_to_bytes(cur, 8, block + 32);
    uint32_t out[16];
    compress(key_, block, 64, 0, flags_ | PARENT, out);
    std::memcpy(cur, out, sizeof(cur));
    stack_len_--;
    total_chunks >>= 1;
  }
  std::memcpy(stack_[stack_len_++], cur, sizeof(cur));
}

void Blake3::update(const void* data, size_t len) {
  const uint8_t* p = (const uint8_t*)data;
  while (len > 0) {
    // a full chunk that more input follows: finish it and move on
    if (blocks_ == 15 && buf_len_ == 64) {
      uint32_t out[16];
      compress(cv_, buf_, 64, chunk_counter_, flags_ | CHUNK_END, out);
      chunk_counter_++;
      push_cv(out, chunk_counter_);
      std::memcpy(cv_, key_, sizeof(cv_));
      buf_len_ = 0;
      blocks_ = 0;
    }
    if (buf_len_ == 64) {
      uint32_t out[16];
      compress(cv_, buf_, 64, chunk_counter_, flags_ | (blocks_ == 0 ? CHUNK_START : 0), out);
      std::memcpy(cv_, out, sizeof(cv_));
      blocks_++;
      buf_len_ = 0;
    }
    size_t take = 64 - buf_len_;
    if (take > len) take = len;
    std::memcpy(buf_ + buf_len_, p, take);
    buf_len_ += (uint32_t)take;
    p += take;
    len -= take;
  }
}

void Blake3::finalize(uint64_t seek, uint8_t* out, size_t len) const {
  // the last node: the current chunk's final block, then parents up the stack
  uint32_t cv[8];
  uint8_t block[64];
  std::memset(block, 0, 64);
  std::memcpy(block, buf_, buf_len_);
  std::memcpy(cv, cv_, sizeof(cv));
  uint32_t block_len = buf_len_;
  uint64_t counter = chunk_counter_;
  uint32_t flags = flags_ | CHUNK_END | (blocks_ == 0 ? CHUNK_START : 0);
  for (int i = (int)stack_len_ - 1; i >= 0; i--) {
    uint32_t o[16];
    compress(cv, block, block_len, counter, flags, o);
    uint8_t pb[64];
    words_to_bytes(stack_[i], 8, pb);
    words_to_bytes(o, 8, pb + 32);
    std::memcpy(block, pb, 64);
    std::memcpy(cv, key_, sizeof(cv));
    block_len = 64;
    counter = 0;
    flags = flags_ | PARENT;
  }
  uint64_t b = seek / 64;
  size_t skip = (size_t)(seek % 64), done = 0;
  while (done < len) {
    uint32_t o[16];
    compress(cv, block, block_len, b, flags | ROOT, o);
    uint8_t bytes[64];
    words_to_bytes(o, 16, bytes);
    for (size_t i = skip; i < 64 && done < len; i++) out[done++] = bytes[i];
    skip = 0;
    b++;
  }
}

void Blake3::save(HasherState& s) const {
  std::memset(&s, 0, sizeof(s));
  std::memcpy(s.key, key_, sizeof(key_));
  s.flags = flags_;
  std::memcpy(s.cv, cv_, sizeof(cv_));
  std::memcpy(s.buf, buf_, sizeof(buf_));
  s.buf_len = buf_len_;
  s.blocks = blocks_;
  s.chunk_counter = chunk_counter_;
  std::memcpy(s.stack, stack_, sizeof(uint32_t) * 8 * stack_len_);
  s.stack_len = stack_len_;
}

void Blake3::load(const HasherState& s) {
  std::memcpy(key_, s.key, sizeof(key_));
  flags_ = s.flags;
  std::memcpy(cv_, s.cv, sizeof(cv_));
  std::memcpy(buf_, s.buf, sizeof(buf_));
  buf_len_ = s.buf_len;
  blocks_ = s.blocks;
  chunk_counter_ = s.chunk_counter;
  stack_len_ = s.stack_len;
  std::memcpy(stack_, s.stack, sizeof(uint32_t) * 8 * stack_len_);
}

uint8_t Blake3Reader::byte() {
  if (off_ == have_) {
    h_.finalize(pos_, buf_, sizeof(buf_));
    pos_ += sizeof(buf_);
    have_ = sizeof(buf_);
    off_ = 0;
  }
  return buf_[off_++];
}

}  // namespace lbg
