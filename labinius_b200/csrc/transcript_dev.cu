// The round's Fiat-Shamir transcript on the device (transcript_dev.h).
//
// An absorb of a long byte string into a BLAKE3 hasher is data parallel once its length is
// known: every chunk that completes is compressed on its own (chunk index = counter), the
// completed chunks' chaining values are merged level by level into the aligned subtrees of
// the new chunk count, and only the subtrees that straddle the old chunk count need the old
// stack. The result is the hasher's canonical state (hasher_state.h), the same one the host
// hasher reaches by absorbing the same bytes one after another.
#include <cstring>
#include <mutex>

#include "blake3_dev.cuh"
#include "transcript.h"
#include "transcript_dev.h"
#include "upload.h"

namespace lbg {

namespace {

__device__ __forceinline__ uint32_t src_byte(const AbsorbSource& s, uint64_t o) {
  if (o < s.prefix_len) return s.prefix[o];
  o -= s.prefix_len;
  uint64_t per = s.hdr_len + s.row_bytes;
  uint64_t row = o / per, c = o - row * per;
  if (c < s.hdr_len) return s.hdr[c];
  return s.data[row * s.row_stride + (c - s.hdr_len)];
}

// Staging: chunk t0 .. t1 of every job laid out contiguously (positions relative to chunk t0's
// first byte): chunk t0's buffered bytes, then the new bytes, zeros after. One thread per 16
// bytes; the thread that covers a job's first word also saves the old chaining value.
__global__ void k_absorb_stage(const AbsorbJob* __restrict__ jobs, int njobs, const uint64_t* __restrict__ word_off,
                               uint8_t* __restrict__ stage, uint32_t* __restrict__ oldcv) {
  uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= word_off[njobs]) return;
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (word_off[mid] <= w) lo = mid;
    else hi = mid - 1;
  }
  const AbsorbJob& J = jobs[lo];
  uint64_t x0 = (w - word_off[lo]) * 16;
  if (x0 == 0)
    for (int i = 0; i < 8; i++) oldcv[8 * lo + i] = J.st->cv[i];
  uint32_t head = J.ob * 64, obl = J.obl;
  uint32_t v[4] = {0, 0, 0, 0};
  for (int k = 0; k < 16; k++) {
    uint64_t x = x0 + k;
    uint32_t b = 0;
    if (x >= head && x < J.stage_len) {
      uint64_t r = x - head;
      b = r < obl ? J.st->buf[r] : src_byte(J.src, r - obl);
    }
    v[k >> 2] |= b << (8 * (k & 3));
  }
  *reinterpret_cast<uint4*>(stage + J.stage_off + x0) = make_uint4(v[0], v[1], v[2], v[3]);
}

// One thread per chunk t0 .. t1 of every job: complete chunks give their chaining values (level
// 0 of the job's subtrees); the open chunk t1 becomes the hasher's current chunk.
__global__ void k_absorb_chunks(const AbsorbJob* __restrict__ jobs, const int* __restrict__ entry_job, int nentries,
                                const uint8_t* __restrict__ stage, const uint32_t* __restrict__ oldcv,
                                uint32_t* __restrict__ cvs) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nentries) return;
  int j = entry_job[e];
  const AbsorbJob& J = jobs[j];
  HasherState* st = J.st;
  uint64_t i = (uint64_t)(e - (int)J.entry_off);
  uint64_t c = J.t0 + i;
  uint32_t cv[8], key[8];
  for (int k = 0; k < 8; k++) key[k] = st->key[k];
  uint32_t flags = st->flags;
  uint32_t start = 0;
  if (i == 0) {
    for (int k = 0; k < 8; k++) cv[k] = oldcv[8 * j + k];
    start = J.ob;
  } else {
    for (int k = 0; k < 8; k++) cv[k] = key[k];
  }
  const uint8_t* base = stage + J.stage_off + i * 1024;
  bool open = c == J.t1;
  uint32_t nbytes = open ? J.c1 : 1024;
  uint32_t last = (nbytes - 1) / 64;  // the block that stays buffered in an open chunk
  uint32_t end = open ? last : 16;
  for (uint32_t b = start; b < end; b++) {
    uint32_t m[16];
    const uint4* q = reinterpret_cast<const uint4*>(base + 64 * b);
    for (int k = 0; k < 4; k++) {
      uint4 v = q[k];
      m[4 * k] = v.x;
      m[4 * k + 1] = v.y;
      m[4 * k + 2] = v.z;
      m[4 * k + 3] = v.w;
    }
    uint32_t fl = flags | (b == 0 ? b3::CHUNK_START : 0) | (!open && b == 15 ? b3::CHUNK_END : 0);
    uint32_t o[16];
    dev::compress(cv, m, c, 64, fl, o);
    for (int k = 0; k < 8; k++) cv[k] = o[k];
  }
  if (!open) {
    uint32_t* dst = cvs + 8 * (J.level_off + i);
    for (int k = 0; k < 8; k++) dst[k] = cv[k];
    return;
  }
  for (int k = 0; k < 8; k++) st->cv[k] = cv[k];
  uint32_t bl = nbytes - 64 * last;
  for (int k = 0; k < 64; k++) st->buf[k] = k < (int)bl ? base[64 * last + k] : 0;
  st->buf_len = bl;
  st->blocks = last;
  st->chunk_counter = c;
}

struct Levels {
  uint64_t t0, t1;
  uint64_t off[64];
  __device__ uint64_t lo(int k) const { return (t0 + ((1ull << k) - 1)) >> k; }
  __device__ uint64_t hi(int k) const { return t1 >> k; }
  __device__ bool inner(int k, uint64_t a) const { return a >= lo(k) && a < hi(k); }
  __device__ bool straddles(int k, uint64_t a) const { return (a << k) < t0 && t0 < ((a + 1) << k); }
};

// One CTA per job: the subtrees of chunks t0 .. t1-1 level by level, then the stack of chunk
// count t1 (one subtree per set bit, largest first) from those and the old stack.
__global__ void k_absorb_tree(const AbsorbJob* __restrict__ jobs, uint32_t* __restrict__ cvs) {
  const AbsorbJob& J = jobs[blockIdx.x];
  if (J.t1 == J.t0) return;
  HasherState* st = J.st;
  __shared__ Levels L;
  __shared__ uint32_t key[8];
  __shared__ uint32_t nst[54][8];
  __shared__ int top;
  if (threadIdx.x == 0) {
    L.t0 = J.t0;
    L.t1 = J.t1;
    L.off[0] = J.level_off;
    top = 0;
    for (int k = 1; k < 64; k++) {
      uint64_t lo = (J.t0 + ((1ull << (k - 1)) - 1)) >> (k - 1), hi = J.t1 >> (k - 1);
      L.off[k] = L.off[k - 1] + (hi > lo ? hi - lo : 0);
    }
  }
  if (threadIdx.x < 8) key[threadIdx.x] = st->key[threadIdx.x];
  __syncthreads();
  uint32_t flags = st->flags;
  for (int k = 1; k < 64 && (1ull << k) <= J.t1; k++) {
    uint64_t lo = L.lo(k), hi = L.hi(k);
    uint64_t plo = L.lo(k - 1);
    for (uint64_t a = lo + threadIdx.x; a < hi; a += blockDim.x) {
      const uint32_t* l = cvs + 8 * (L.off[k - 1] + 2 * a - plo);
      const uint32_t* r = l + 8;
      uint32_t out[8];
      dev::parent_cv(key, flags, l, r, out);
      uint32_t* dst = cvs + 8 * (L.off[k] + a - lo);
      for (int q = 0; q < 8; q++) dst[q] = out[q];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  uint64_t t0 = J.t0, t1 = J.t1;
  // a node that does not straddle t0: a level entry or an entry of the old stack
  auto get = [&](int k, uint64_t a, uint32_t out[8]) {
    const uint32_t* s;
    if (L.inner(k, a)) s = cvs + 8 * (L.off[k] + a - L.lo(k));
    else s = st->stack[min(__popcll(t0 >> (k + 1)), 53)];
    for (int q = 0; q < 8; q++) out[q] = s[q];
  };
  for (int k = 63; k >= 0; k--) {
    if (!((t1 >> k) & 1)) continue;
    uint64_t a = (t1 >> (k + 1)) << 1;
    uint32_t cur[8];
    if (!L.straddles(k, a)) {
      get(k, a, cur);
    } else {
      uint32_t sib[64][8];
      bool sib_right[64];
      int depth = 0, kk = k;
      uint64_t aa = a;
      while (L.straddles(kk, aa)) {
        kk--;
        uint64_t l = 2 * aa, r = l + 1;
        if (L.straddles(kk, l)) {
          get(kk, r, sib[depth]);
          sib_right[depth] = true;
          aa = l;
        } else {
          get(kk, l, sib[depth]);
          sib_right[depth] = false;
          aa = r;
        }
        depth++;
      }
      get(kk, aa, cur);
      for (int d = depth - 1; d >= 0; d--) {
        if (sib_right[d]) dev::parent_cv(key, flags, cur, sib[d], cur);
        else dev::parent_cv(key, flags, sib[d], cur, cur);
      }
    }
    for (int q = 0; q < 8; q++) nst[top][q] = cur[q];
    top++;
  }
  for (int e = 0; e < top; e++)
    for (int q = 0; q < 8; q++) st->stack[e][q] = nst[e][q];
  st->stack_len = (uint32_t)top;
}

// ----------------------------------------------------------------------------------------------
// evaluation point, folding challenges, claims, bit-dropped packing
// ----------------------------------------------------------------------------------------------
__constant__ char c_point_label[] = "labinius/evaluation-point";
__constant__ char c_chal_label[] = "short-challenge";

// One CTA per instance: derive("labinius/evaluation-point"), 24 bytes per coordinate, the top
// limb masked to 34 bits (crates/pcs/src/scheme/verifier.rs:86-100).
__global__ void k_point(const RoundInst* __restrict__ inst, uint32_t row_log, uint64_t* __restrict__ p0,
                        uint64_t* __restrict__ p1) {
  const RoundInst& I = inst[blockIdx.x];
  __shared__ XofRoot root;
  __shared__ uint32_t words[6 * 64];  // up to 64 coordinates
  if (threadIdx.x == 0) dev::derive_root(I.st, I.point_counter, c_point_label, 25, root);
  __syncthreads();
  uint32_t n = row_log + I.col_log;
  uint32_t nblocks = (24 * n + 63) / 64;
  for (uint32_t t = threadIdx.x; t < nblocks; t += blockDim.x) {
    uint32_t o[16];
    dev::root_block(root, t, o);
    for (int k = 0; k < 16; k++) words[16 * t + k] = o[k];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint64_t limb[3];
    for (int k = 0; k < 3; k++) limb[k] = (uint64_t)words[6 * i + 2 * k] | ((uint64_t)words[6 * i + 2 * k + 1] << 32);
    limb[2] &= (1ull << 34) - 1;
    uint64_t* dst = i < row_log ? p0 + 3 * ((uint64_t)row_log * blockIdx.x + i) : p1 + 3 * (32ull * blockIdx.x + i - row_log);
    for (int k = 0; k < 3; k++) dst[k] = limb[k];
  }
}

// rejection sampling below n from little-endian u16s (crates/pcs/src/challenge.rs:197-221)
__device__ __forceinline__ uint32_t below(dev::Reader& x, uint32_t n) {
  uint32_t limit = (65536u / n) * n;
  uint64_t magic = (1ull << 32) / n + 1;
  for (int tries = 0; tries < (1 << 16); tries++) {  // each try passes with probability > 0.99
    uint32_t lo = x.byte();
    uint32_t hi = x.byte();
    uint32_t r = lo | (hi << 8);
    if (r < limit) return r - (uint32_t)(((uint64_t)r * magic) >> 32) * n;
  }
  return 0;
}

// One warp per column: lane 0 derives "short-challenge" with the column's counter and runs the
// sampler's sequential part of each attempt (crates/pcs/src/challenge.rs:517-533: a partial
// Fisher-Yates shuffle of 0..161, the sorted positions, the sign hash); the 32 lanes then test
// the spectral bound for 81 evaluation points between them, each point's sum in f64 in the host's
// operation order (no contraction). The first attempt every point passes is the challenge.
constexpr int CHAL_WARPS = 4;

__global__ void __launch_bounds__(32 * CHAL_WARPS)
    k_challenges(const RoundInst* __restrict__ inst, const int* __restrict__ col_inst, int total_cols,
                 SamplerTables tab, lbg_challenge_d* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * CHAL_WARPS + (threadIdx.x >> 5);
  if (j >= total_cols) return;  // the whole warp
  const RoundInst& I = inst[col_inst[j]];
  const uint32_t weight = tab.weight < 32 ? tab.weight : 32;
  dev::Reader x;
  if (lane == 0) {
    XofRoot root;
    dev::derive_root(I.st, I.chal_counter + (uint64_t)(j - (int)I.col_off), c_chal_label, 15, root);
    x.init(root);
  }
  for (int attempt = 0; attempt < 4096; attempt++) {  // an attempt passes with probability ~2/3
    uint32_t pw[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // the sorted positions, four per word
    uint32_t signs = 0;
    if (lane == 0) {
      uint8_t perm[162];
      for (int i = 0; i < 162; i++) perm[i] = (uint8_t)i;
      for (uint32_t i = 0; i < weight; i++) {
        uint32_t k = i + below(x, 162 - i);
        uint8_t t = perm[i];
        perm[i] = perm[k];
        perm[k] = t;
      }
      uint64_t seen[3] = {0, 0, 0};
      for (uint32_t i = 0; i < weight; i++) seen[perm[i] >> 6] |= 1ull << (perm[i] & 63);
      uint8_t pos[32];
      for (int i = 0; i < 32; i++) pos[i] = 0;
      int n = 0;
      for (int w = 0; w < 3; w++)
        for (uint64_t b = seen[w]; b; b &= b - 1) pos[n++] = (uint8_t)(64 * w + __ffsll((long long)b) - 1);
      // signs: derive-key hash of le64(weight) || positions (one block, one chunk, root)
      uint8_t blk[64];
      for (int i = 0; i < 64; i++) blk[i] = 0;
      for (int i = 0; i < 8; i++) blk[i] = (uint8_t)((uint64_t)weight >> (8 * i));
      for (uint32_t i = 0; i < weight; i++) blk[8 + i] = pos[i];
      uint32_t m[16], o[16];
      dev::bytes_to_words(blk, m, 16);
      dev::compress(tab.signs_key, m, 0, 8 + weight,
                    b3::DERIVE_KEY_MATERIAL | b3::CHUNK_START | b3::CHUNK_END | b3::ROOT, o);
      signs = o[0] & (uint32_t)((1ull << weight) - 1);
      dev::bytes_to_words(pos, pw, 8);
    }
#pragma unroll
    for (int w = 0; w < 8; w++) pw[w] = __shfl_sync(0xffffffffu, pw[w], 0);
    signs = __shfl_sync(0xffffffffu, signs, 0);
    bool bad = false;
    for (int u = lane; u < 81; u += 32) {
      double vr = 0.0, vi = 0.0;
#pragma unroll
      for (int i = 0; i < 32; i++) {
        if (i < (int)weight) {
          int p = (pw[i >> 2] >> (8 * (i & 3))) & 0xFF;
          double re = __ldg(tab.re + 81 * p + u), im = __ldg(tab.im + 81 * p + u);
          bool neg = (signs >> i) & 1;
          vr = __dadd_rn(vr, neg ? -re : re);
          vi = __dadd_rn(vi, neg ? -im : im);
        }
      }
      double xx = __dadd_rn(__dmul_rn(vr, vr), __dmul_rn(vi, vi));
      if (xx > tab.bound_sq) bad = true;
    }
    if (!__any_sync(0xffffffffu, bad)) {
      if (lane == 0) {
        lbg_challenge_d c;
        for (int i = 0; i < 32; i++) c.positions[i] = (uint8_t)(pw[i >> 2] >> (8 * (i & 3)));
        c.signs = signs;
        c.weight = weight;
        out[j] = c;
      }
      return;
    }
  }
  if (lane == 0) {
    lbg_challenge_d none;  // weight 0: no challenge found (the host reports it)
    for (int i = 0; i < 32; i++) none.positions[i] = 0;
    none.signs = 0;
    none.weight = 0;
    out[j] = none;
  }
}

// One thread per output byte: bit g of the stream is bit r of field f of element g / bits_per.
__global__ void k_pack_dropped(const uint16_t* __restrict__ top, const uint16_t* __restrict__ digits, uint64_t count,
                               uint64_t digit_stride, PackDropped pk, uint8_t* __restrict__ out, uint64_t nbytes) {
  uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nbytes) return;
  uint32_t v = 0;
  for (int b = 0; b < 8; b++) {
    uint64_t g = 8 * k + b;
    uint64_t e = g / pk.bits_per;
    if (e >= count) break;
    uint32_t r = (uint32_t)(g - e * pk.bits_per);
    uint32_t bit;
    if (r < pk.top_bits) {
      bit = (top[e] >> r) & 1;
    } else {
      r -= pk.top_bits;
      uint32_t f = 1;
      while (r >= pk.residue_bits[f]) {
        r -= pk.residue_bits[f];
        f++;
      }
      bit = (digits[(f - 1) * digit_stride + e] >> r) & 1;
    }
    v |= bit << b;
  }
  out[k] = (uint8_t)v;
}

}  // namespace

void AbsorbPlan::clear() {
  jobs.clear();
  entry_job.clear();
  stage_word_off.assign(1, 0);
  stage_bytes = cv_slots = 0;
}

void AbsorbPlan::release() {
  cudaFree(d_jobs);
  cudaFree(d_entry_job);
  cudaFree(d_stage_word_off);
  d_jobs = nullptr;
  d_entry_job = nullptr;
  d_stage_word_off = nullptr;
}

void plan_absorb(AbsorbPlan& p, HasherState* d_state, uint64_t old_len, const AbsorbSource& src) {
  if (p.stage_word_off.empty()) p.stage_word_off.push_back(0);
  AbsorbJob J;
  J.st = d_state;
  J.src = src;
  uint64_t t0 = (old_len - 1) / 1024, c0 = old_len - 1024 * t0;
  J.obl = (uint32_t)((c0 - 1) % 64 + 1);
  J.ob = (uint32_t)((c0 - J.obl) / 64);
  uint64_t new_len = old_len + src.length();
  uint64_t t1 = (new_len - 1) / 1024;
  J.t0 = t0;
  J.t1 = t1;
  J.c1 = (uint32_t)(new_len - 1024 * t1);
  J.stage_len = (t1 - t0) * 1024 + J.c1;
  J.stage_off = p.stage_bytes;
  p.stage_bytes += (J.stage_len + 1023) / 1024 * 1024;
  p.stage_word_off.push_back(p.stage_word_off.back() + (J.stage_len + 15) / 16);
  J.entry_off = (uint32_t)p.entry_job.size();
  for (uint64_t i = 0; i <= t1 - t0; i++) p.entry_job.push_back((int)p.jobs.size());
  J.level_off = p.cv_slots;
  p.cv_slots += 2 * (t1 - t0) + 2;
  p.jobs.push_back(J);
}

cudaError_t upload_absorb(AbsorbPlan& p) {
  p.release();
  cudaError_t e = cudaMalloc((void**)&p.d_jobs, p.jobs.size() * sizeof(AbsorbJob));
  if (e == cudaSuccess) e = cudaMalloc((void**)&p.d_entry_job, p.entry_job.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&p.d_stage_word_off, p.stage_word_off.size() * sizeof(uint64_t));
  if (e == cudaSuccess)
    e = upload_sync(p.d_jobs, p.jobs.data(), p.jobs.size() * sizeof(AbsorbJob));
  if (e == cudaSuccess)
    e = upload_sync(p.d_entry_job, p.entry_job.data(), p.entry_job.size() * sizeof(int));
  if (e == cudaSuccess)
    e = upload_sync(p.d_stage_word_off, p.stage_word_off.data(), p.stage_word_off.size() * sizeof(uint64_t));
  return e;
}

cudaError_t launch_absorb(const AbsorbPlan& p, uint8_t* d_stage, uint32_t* d_cvs, uint32_t* d_oldcv, cudaStream_t st) {
  int njobs = (int)p.jobs.size();
  if (njobs == 0) return cudaSuccess;
  uint64_t words = p.stage_word_off.back();
  k_absorb_stage<<<(unsigned)((words + 255) / 256), 256, 0, st>>>(p.d_jobs, njobs, p.d_stage_word_off, d_stage,
                                                                  d_oldcv);
  int ne = (int)p.entry_job.size();
  k_absorb_chunks<<<(ne + 127) / 128, 128, 0, st>>>(p.d_jobs, p.d_entry_job, ne, d_stage, d_oldcv, d_cvs);
  k_absorb_tree<<<njobs, 256, 0, st>>>(p.d_jobs, d_cvs);
  return cudaGetLastError();
}

cudaError_t launch_point(const RoundInst* d_inst, int count, uint32_t row_log, uint64_t* p0, uint64_t* p1,
                         cudaStream_t st) {
  k_point<<<count, 64, 0, st>>>(d_inst, row_log, p0, p1);
  return cudaGetLastError();
}

cudaError_t sampler_tables(int device, SamplerTables& out) {
  static std::mutex mu;
  static double* re[64] = {nullptr};
  static double* im[64] = {nullptr};
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(mu);
  if (!re[device]) {
    size_t bytes = 162 * 81 * sizeof(double);
    double *r = nullptr, *i = nullptr;
    cudaError_t e = cudaMalloc((void**)&r, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&i, bytes);
    if (e == cudaSuccess) e = upload_sync(r, sampler_phase_re(), bytes);
    if (e == cudaSuccess) e = upload_sync(i, sampler_phase_im(), bytes);
    if (e != cudaSuccess) {
      cudaFree(r);
      cudaFree(i);
      return e;
    }
    re[device] = r;
    im[device] = i;
  }
  out.re = re[device];
  out.im = im[device];
  std::memcpy(out.signs_key, sampler_signs_key(), sizeof(out.signs_key));
  out.weight = 28;
  volatile double b2 = 12.0 * 12.0;
  out.bound_sq = b2 + 1e-12;
  return cudaSuccess;
}

cudaError_t launch_challenges(const RoundInst* d_inst, const int* col_inst, int total_cols, SamplerTables tab,
                              lbg_challenge_d* out, cudaStream_t st) {
  k_challenges<<<(total_cols + CHAL_WARPS - 1) / CHAL_WARPS, 32 * CHAL_WARPS, 0, st>>>(d_inst, col_inst, total_cols,
                                                                                     tab, out);
  return cudaGetLastError();
}

cudaError_t launch_pack_dropped(const uint16_t* top, const uint16_t* digits, uint64_t count, uint64_t digit_stride,
                                PackDropped pk, uint8_t* out, uint64_t nbytes, cudaStream_t st) {
  k_pack_dropped<<<(unsigned)((nbytes + 255) / 256), 256, 0, st>>>(top, digits, count, digit_stride, pk, out, nbytes);
  return cudaGetLastError();
}

}  // namespace lbg
