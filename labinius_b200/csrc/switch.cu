// The cross-field switch prover on the device (crates/pcs/src/switch.rs:133-168,
// crates/pcs/src/fields/crossfield.rs, crates/pcs/src/fields/sumcheck.rs).
//
// A B128 trace of 2^l words, committed as Witness::lifted, carries a claim in B128 at r_hi; the
// switch turns it into the F162 claim the commitment opens, at the point its sumcheck ends on.
// The prover's work is two passes over the trace and a sumcheck of l rounds:
//  * eq_hi = the expansion of r_hi (one B128 product per entry, from two half-size tables);
//  * a_j = psi(eq_hi[j]) = sum_k bit_k(eq_hi[j]) batch[k], p_j = the trace word t_j as an F162;
//  * round k sends (sum a0 p0, sum (a0 + a1)(p0 + p1)) over the index pairs (j, j + half) and
//    folds both tables with its challenge r: x0 + r (x0 + x1).
// The first pass needs no field product per element. The 128 partial evaluations
// v[k] = sum_j bit_k(t_j) eq_j and round 0's message (sum_k batch[k] P_k, sum_k batch[k] Q_k with
// P_k = sum_{j < n/2} bit_k(eq_j) t_j and Q_k the same over the pairs' sums) are all read off
// three 128 x 128 GF(2) matrices sum_j t_j (x) eq_j (bit k of one times bit m of the other), over
// j >= n/2, over j < n/2, and over the pairs (v is the sum of the first two, P and Q are columns
// of the last two). One pass accumulates all three, a warp lane owning four selector bits and
// masking the value words by them (k_sw_sums).
// The second pass is round 0's fold with round 1's message; later rounds fold in place. Every
// fold and the next message are one kernel; products by r go through 4-bit tables of (t x^4i) r in
// shared memory, a through nibble tables of the batch (psi is linear, so a_j + a_j' =
// psi(eq_j + eq_j')); round 0's tables are read through eq and the trace and never stored, so the
// folded tables take n/2 entries. The last rounds run in one CTA per instance (k_sw_tail).
// The transcript runs on the device too: each instance's hasher state absorbs the statement,
// the partials and every message, and the batch and round challenges are derived from it (one
// CTA per instance), so a whole switch is one pass on a stream with no host round trip. The
// single-instance entry point moves the caller's transcript to the device and back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "blake3_dev.cuh"
#include "error.h"
#include "gf2_dev.cuh"
#include "handles.h"
#include "switch.h"
#include "transcript.h"

namespace lbg {
namespace {

constexpr int SW_THREADS = 256;
constexpr uint32_t SW_CAP = 148 * 8;  // blocks per instance and launch, at most

__constant__ char c_sw_label[16] = "labinius/switch";
__constant__ char c_sw_batch[22] = "labinius/switch-batch";
__constant__ char c_sw_round[22] = "labinius/switch-round";

// Rounds from sw_tail_start(l) on run in k_sw_tail: their messages sum at most 2^(SW_TAIL_LOG - 2)
// pairs, little enough for one block, so the rounds that are left cost no launches.
constexpr uint32_t SW_TAIL_LOG = 10;
__host__ __device__ inline uint32_t sw_tail_start(uint32_t l) {
  return l > SW_TAIL_LOG ? l - SW_TAIL_LOG : (l > 0 ? 1u : 0u);
}

// Work units of an instance with l variables in a launch: stage 0 counts elements, stage 1 the
// pairs of round 0's message, stage 2 the work of round k's fold (the pairs of round k + 1's
// message, or the one pair of the last fold; none from the instance's tail on); stages 3
// and 4 split the eq expansion: elements of instances whose low half-table is short (stage 3),
// segments of 2^ll entries that share their high factor otherwise (stage 4).
constexpr uint32_t SW_SEG_LL = 10;
__host__ __device__ inline uint64_t sw_units(uint32_t l, int stage, int k) {
  uint64_t n = 1ull << l;
  const uint32_t ll = l - l / 2;
  if (stage == 0) return n;
  if (stage == 1) return n / 2;
  if (stage == 3) return ll < SW_SEG_LL ? n : 0;
  if (stage == 4) return ll < SW_SEG_LL ? 0 : 1ull << (l / 2);
  if ((uint32_t)k >= sw_tail_start(l)) return 0;
  if ((uint32_t)k + 1 == l) return 1;
  return n >> (k + 2);
}
__host__ __device__ inline uint32_t sw_blocks(uint64_t units, int per_block) {
  uint64_t b = (units + per_block - 1) / per_block;
  return (uint32_t)(b < SW_CAP ? b : SW_CAP);
}

// Blocks are dealt to the instances in order, each getting sw_blocks(its units); this block's
// instance (or -1), its rank among the instance's blocks and their number.
__device__ __forceinline__ int sw_find(const SwInst* __restrict__ I, int count, int stage, int k, int per_block,
                                       uint32_t& local, uint32_t& nblk) {
  uint32_t b = blockIdx.x;
  for (int i = 0; i < count; i++) {
    uint32_t nb = sw_blocks(sw_units(I[i].l, stage, k), per_block);
    if (b < nb) {
      local = b;
      nblk = nb;
      return i;
    }
    b -= nb;
  }
  return -1;
}

__device__ __forceinline__ B128d ld_b(const uint64_t* p, size_t j) {
  ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p + 2 * j);
  return B128d{v.x, v.y};
}
__device__ __forceinline__ void st_b(uint64_t* p, size_t j, B128d x) {
  *reinterpret_cast<ulonglong2*>(p + 2 * j) = make_ulonglong2(x.lo, x.hi);
}
__device__ __forceinline__ F162d ld_f(const uint64_t* p, size_t j) {
  return F162d{{p[3 * j], p[3 * j + 1], p[3 * j + 2]}};
}
__device__ __forceinline__ void st_f(uint64_t* p, size_t j, F162d x) {
  p[3 * j] = x.w[0];
  p[3 * j + 1] = x.w[1];
  p[3 * j + 2] = x.w[2];
}
// trace word j as an F162 (the low 128 bits of the lifted element)
__device__ __forceinline__ F162d ld_word(const uint64_t* __restrict__ w, size_t j) {
  return F162d{{__ldg(w + 3 * j), __ldg(w + 3 * j + 1), 0}};
}

// Entry idx of the expansion of r[0..m): the product over rounds of r_round or 1 + r_round, by
// bit m-1-round of idx (crates/pcs/src/fields/crossfield.rs:78-98: the last coordinate is bit 0).
// Block (0, i) also clears instance i's matrix and message accumulators and its status.
__global__ void k_sw_tables(const SwInst* __restrict__ I) {
  const SwInst& s = I[blockIdx.y];
  if (blockIdx.x == 0) {
    uint32_t* m = &s.s->mat[0][0][0];
    for (int t = threadIdx.x; t < 3 * 128 * 4; t += blockDim.x) m[t] = 0;
    if (threadIdx.x < 8) s.s->msg[threadIdx.x] = 0;
    if (threadIdx.x == 0) s.s->status = 0;
  }
  uint32_t nh = 1u << s.lh, nl = 1u << s.ll;
  uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nh + nl) return;
  bool high = g < nh;
  uint32_t idx = high ? g : g - nh;
  uint32_t m = high ? s.lh : s.ll;
  const uint64_t* rr = s.r_hi + 2 * (high ? 0 : s.lh);
  B128d acc{1, 0};
  for (uint32_t round = 0; round < m; round++) {
    B128d f = ld_b(rr, round);
    if (!((idx >> (m - 1 - round)) & 1)) f.lo ^= 1;
    acc = b_mul(acc, f);
  }
  st_b(high ? s.e_hi : s.e_lo, idx, acc);
}

__global__ void __launch_bounds__(SW_THREADS) k_sw_eq(const SwInst* __restrict__ I, int count) {
  uint32_t local, nblk;
  int i = sw_find(I, count, 3, 0, SW_THREADS, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  size_t n = 1ull << s.l;
  uint64_t lm = (1ull << s.ll) - 1;
  for (size_t j = (size_t)local * SW_THREADS + threadIdx.x; j < n; j += (size_t)nblk * SW_THREADS)
    st_b(s.eq, j, b_mul(ld_b(s.e_hi, j >> s.ll), ld_b(s.e_lo, j & lm)));
}

// eq over segments: the 2^ll entries j = (a << ll) | b share e_hi[a], so a block builds the tables
// of (t x^{4c}) e_hi[a] (32 nibble positions, 16 values) once and multiplies every e_lo[b] by 32
// lookups.
__global__ void __launch_bounds__(SW_THREADS) k_sw_eq_seg(const SwInst* __restrict__ I, int count) {
  __shared__ B128d T[32 * 16];
  __shared__ B128d R4[32];
  uint32_t local, nblk;
  int i = sw_find(I, count, 4, 0, 1, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  const uint32_t nseg = 1u << s.lh, seglen = 1u << s.ll;
  for (uint32_t a = local; a < nseg; a += nblk) {
    __syncthreads();
    if (threadIdx.x == 0) {
      B128d r = ld_b(s.e_hi, a);
      for (int c = 0; c < 32; c++) {
        R4[c] = r;
        r = b_times_x4(r);
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
      const int c = e >> 4, t = e & 15;
      B128d x = R4[c], acc{0, 0};
      for (int b = 0; b < 4; b++) {
        if ((t >> b) & 1) acc = b_add(acc, x);
        x = b_times_x(x);
      }
      T[e] = acc;
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < seglen; b += blockDim.x) {
      const B128d lo = ld_b(s.e_lo, b);
      B128d acc{0, 0};
#pragma unroll
      for (int c = 0; c < 32; c++) {
        const uint32_t nib = (uint32_t)((c < 16 ? lo.lo >> (4 * c) : lo.hi >> (4 * (c - 16))) & 15);
        acc = b_add(acc, T[16 * c + nib]);
      }
      st_b(s.eq, ((size_t)a << s.ll) + b, acc);
    }
  }
}

// The three matrices in one pass over the pairs (j, j + n/2), j < n/2: kind 0 the rows j + n/2
// (selector t, value eq), kind 1 the rows j, kind 2 the pairs' sums. Row k of a matrix is the XOR
// of the values of the rows whose selector has bit k set. A CTA stages 256 pairs' three rows in
// shared memory (the next 256 are loaded into registers meanwhile); warp w then runs through 32
// of them with lane l owning the bits k = 4 l + q (q < 4) of all three matrices: per row, one
// selector word and one value read by broadcast, four sign-extended bit masks and sixteen masked
// XORs (one LOP3 each). The warps' sums are XOR-reduced in shared memory, then into the
// instance's matrices.
constexpr int SW_SUM_ROWS = 2048;  // pairs per block before the cap
__global__ void __launch_bounds__(SW_THREADS) k_sw_sums(const SwInst* __restrict__ I, int count) {
  __shared__ uint4 sSel[3][SW_THREADS], sVal[3][SW_THREADS];
  __shared__ uint32_t sAcc[3][128][4];
  uint32_t local, nblk;
  int i = sw_find(I, count, 1, 0, SW_SUM_ROWS, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  const size_t h = (1ull << s.l) / 2;
  for (int t = threadIdx.x; t < 3 * 128 * 4; t += blockDim.x) (&sAcc[0][0][0])[t] = 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t acc[3][4][4];
#pragma unroll
  for (int kind = 0; kind < 3; kind++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[kind][q][0] = acc[kind][q][1] = acc[kind][q][2] = acc[kind][q][3] = 0;
  // pair base + threadIdx.x: its two trace words and eq values (zeros past the pairs)
  uint64_t tl0, tl1, th0, th1;
  B128d el, eh;
  auto fetch = [&](size_t base) {
    const size_t j = base + threadIdx.x;
    tl0 = tl1 = th0 = th1 = 0;
    el = eh = B128d{0, 0};
    if (j < h) {
      tl0 = __ldg(s.w + 3 * j), tl1 = __ldg(s.w + 3 * j + 1);
      th0 = __ldg(s.w + 3 * (j + h)), th1 = __ldg(s.w + 3 * (j + h) + 1);
      el = ld_b(s.eq, j), eh = ld_b(s.eq, j + h);
    }
  };
  auto u4 = [](uint64_t lo, uint64_t hi) {
    return make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
  };
  const int sel_shift = 28 - 4 * (lane & 7);
  const size_t stride = (size_t)nblk * SW_THREADS;
  fetch((size_t)local * SW_THREADS);
  for (size_t base = (size_t)local * SW_THREADS; base < h; base += stride) {
    __syncthreads();  // the previous chunk's rows are consumed
    sSel[0][threadIdx.x] = u4(th0, th1);
    sVal[0][threadIdx.x] = u4(eh.lo, eh.hi);
    sSel[1][threadIdx.x] = u4(tl0, tl1);
    sVal[1][threadIdx.x] = u4(el.lo, el.hi);
    sSel[2][threadIdx.x] = u4(tl0 ^ th0, tl1 ^ th1);
    sVal[2][threadIdx.x] = u4(el.lo ^ eh.lo, el.hi ^ eh.hi);
    __syncthreads();
    if (base + stride < h) fetch(base + stride);
    for (int r = 0; r < 32; r++) {
      const int row = 32 * warp + r;
#pragma unroll
      for (int kind = 0; kind < 3; kind++) {
        // the lane's four selector bits moved to bits 28..31, then one mask per bit
        const uint32_t t = reinterpret_cast<const uint32_t*>(&sSel[kind][row])[lane >> 3] << sel_shift;
        const uint4 e = sVal[kind][row];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const uint32_t m = bit_mask(t, 28 + q);
          acc[kind][q][0] ^= e.x & m;
          acc[kind][q][1] ^= e.y & m;
          acc[kind][q][2] ^= e.z & m;
          acc[kind][q][3] ^= e.w & m;
        }
      }
    }
  }
#pragma unroll
  for (int kind = 0; kind < 3; kind++)
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int w = 0; w < 4; w++)
        if (acc[kind][q][w]) atomicXor(&sAcc[kind][4 * lane + q][w], acc[kind][q][w]);
  __syncthreads();
  uint32_t* m = &s.s->mat[0][0][0];
  for (int t = threadIdx.x; t < 3 * 128 * 4; t += blockDim.x) {
    uint32_t val = (&sAcc[0][0][0])[t];
    if (val) atomicXor(m + t, val);
  }
}

// One block per instance: the claim (if the statement leaves it to the prover: the trace's value
// at r_hi, sum_k v[k] x^k, crates/pcs/src/switch.rs:116-122), absorb_statement and the partials
// (crates/pcs/src/switch.rs:124-129, 147-148) staged behind the hasher's open block as one byte
// string and absorbed into the shared copy of the hasher, then the batch coordinates,
// sample_f162("labinius/switch-batch", 7) (crates/pcs/src/switch.rs:149,
// crates/pcs/src/challenge.rs:129-140).
constexpr int SW_STMT_MAX = 23 + 8 + 16 * 7 + 8 + 16 * 32 + 24 + 8 + 16 * 128;
__global__ void k_sw_statement(const SwInst* __restrict__ I) {
  const SwInst& s = I[blockIdx.x];
  SwSmall* sm = s.s;
  __shared__ HasherState sh;
  __shared__ uint64_t v[256], claim[2];
  __shared__ uint32_t stage[(64 + SW_STMT_MAX + 63) / 64 * 16];
  __shared__ uint32_t cvs[8][8];
  uint32_t last;
  uint8_t* bytes = reinterpret_cast<uint8_t*>(stage);
  dev::hs_copy(&sh, s.st);
  // v[k] is row k of the matrices over the rows j + n/2 and j < n/2 (bit m of word m / 32)
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    const uint32_t* hi = sm->mat[0][t >> 1];
    const uint32_t* lo = sm->mat[1][t >> 1];
    const int o = 2 * (t & 1);
    uint64_t x = (uint64_t)(hi[o] ^ lo[o]) | ((uint64_t)(hi[o + 1] ^ lo[o + 1]) << 32);
    v[t] = x;
    (&sm->v[0][0])[t] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    B128d acc{sm->claim[0], sm->claim[1]};
    if (!s.claim_given) {
      acc = B128d{0, 0};
      for (int k = 127; k >= 0; k--) acc = b_add(b_times_x(acc), B128d{v[2 * k], v[2 * k + 1]});
      sm->claim[0] = acc.lo;
      sm->claim[1] = acc.hi;
    }
    claim[0] = acc.lo;
    claim[1] = acc.hi;
  }
  __syncthreads();
  // the open block, then le64(15) "labinius/switch", le64(nlo) r_lo, le64(l) r_hi, le64(1) claim,
  // le64(128) partials
  const uint32_t bl = sh.buf_len, o_lo = bl + 31, o_hi = o_lo + 16 * s.nlo + 8, o_claim = o_hi + 16 * s.l + 8,
                 o_v = o_claim + 24, total = o_v + 16 * 128, padded = (total + 63) / 64 * 64;
  for (uint32_t b = threadIdx.x; b < padded; b += blockDim.x) {
    uint64_t word = 0;
    uint32_t at = 0;
    if (b < bl) {
      bytes[b] = sh.buf[b];
      continue;
    } else if (b < bl + 8) {
      word = 15, at = b - bl;
    } else if (b < bl + 23) {
      bytes[b] = (uint8_t)c_sw_label[b - bl - 8];
      continue;
    } else if (b < o_lo) {
      word = s.nlo, at = b - (bl + 23);
    } else if (b < o_hi - 8) {
      word = s.r_lo[(b - o_lo) / 8], at = (b - o_lo) % 8;
    } else if (b < o_hi) {
      word = s.l, at = b - (o_hi - 8);
    } else if (b < o_claim - 8) {
      word = s.r_hi[(b - o_hi) / 8], at = (b - o_hi) % 8;
    } else if (b < o_claim) {
      word = 1, at = b - (o_claim - 8);
    } else if (b < o_claim + 16) {
      word = claim[(b - o_claim) / 8], at = (b - o_claim) % 8;
    } else if (b < o_v) {
      word = 128, at = b - (o_v - 8);
    } else if (b < total) {
      word = v[(b - o_v) / 8], at = (b - o_v) % 8;
    }
    bytes[b] = (uint8_t)(word >> (8 * at));
  }
  __syncthreads();
  static_assert(64 + SW_STMT_MAX <= 8 * 1024 - 64, "the chunk-parallel absorb takes 8 chunks");
  last = dev::hs_absorb_staged_par(&sh, stage, total, cvs);
  const uint32_t nbl = total - last;
  for (uint32_t b = threadIdx.x; b < nbl; b += blockDim.x) sh.buf[b] = bytes[last + b];
  __syncthreads();
  // derive("labinius/switch-batch"): the open block, le64(counter), le64(21), the label
  const uint32_t dtotal = nbl + 37;
  for (uint32_t b = threadIdx.x; b < 128; b += blockDim.x) {
    uint32_t x = 0;
    if (b < nbl) x = sh.buf[b];
    else if (b < nbl + 8) x = (uint32_t)(s.counter0 >> (8 * (b - nbl))) & 0xFF;
    else if (b < nbl + 16) x = b == nbl + 8 ? 21 : 0;
    else if (b < dtotal) x = (uint8_t)c_sw_batch[b - nbl - 16];
    bytes[b] = (uint8_t)x;
  }
  if (threadIdx.x == 0) sh.buf_len = nbl;
  __syncthreads();
  if (threadIdx.x == 0) {
    XofRoot root;
    dev::hs_derive_staged(&sh, stage, dtotal, root);
    uint32_t out[48];
    for (int t = 0; t < 3; t++) dev::root_block_ool(root, t, out + 16 * t);
    for (int c = 0; c < 7; c++) {
      for (int w = 0; w < 3; w++) sm->rp[c][w] = (uint64_t)out[6 * c + 2 * w] | ((uint64_t)out[6 * c + 2 * w + 1] << 32);
      sm->rp[c][2] &= (1ull << 34) - 1;
    }
  }
  __syncthreads();
  dev::hs_copy(s.st, &sh);
}

// batch = the expansion of the 7 sampled F162 (crossfield.rs:65-76); psi[16 c + t] = the XOR of
// batch[4c + b] over the set bits b of t (crossfield.rs:112-130); and round 0's message,
// e0 = sum_k batch[k] P_k and einf = sum_k batch[k] Q_k, where P_k (bit m) is entry (m, k) of the
// matrix over j < n/2 and Q_k of the matrix over the pairs. One block of 256 threads per instance.
__global__ void __launch_bounds__(256) k_sw_batch(const SwInst* __restrict__ I) {
  const SwInst& s = I[blockIdx.x];
  __shared__ F162d t[2][128];
  __shared__ uint32_t mpq[2][128][4];
  __shared__ uint64_t red[8][6];
  for (int e = threadIdx.x; e < 2 * 128 * 4; e += blockDim.x) (&mpq[0][0][0])[e] = (&s.s->mat[1][0][0])[e];
  if (threadIdx.x == 0) t[0][0] = F162d{{1, 0, 0}};
  __syncthreads();
  int cur = 0;
  for (int round = 0; round < 7; round++) {
    int size = 1 << round;
    if ((int)threadIdx.x < size) {
      F162d x = t[cur][threadIdx.x];
      F162d h = f_mul(x, ld_f(&s.s->rp[0][0], round));
      t[cur ^ 1][2 * threadIdx.x] = f_add(x, h);
      t[cur ^ 1][2 * threadIdx.x + 1] = h;
    }
    __syncthreads();
    cur ^= 1;
  }
  for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
    int c = e >> 4, v = e & 15;
    F162d acc{{0, 0, 0}};
    for (int b = 0; b < 4; b++)
      if ((v >> b) & 1) acc = f_add(acc, t[cur][4 * c + b]);
    st_f(&s.s->psi[0][0], e, acc);
  }
  // thread k < 128: P_k, thread 128 + k: Q_k, times batch[k]
  const int k = threadIdx.x & 127, which = threadIdx.x >> 7;
  uint64_t col[2] = {0, 0};
  for (int m = 0; m < 128; m++) col[m >> 6] |= (uint64_t)((mpq[which][m][k >> 5] >> (k & 31)) & 1u) << (m & 63);
  F162d prod = f_mul(t[cur][k], F162d{{col[0], col[1], 0}});
  for (int o = 16; o > 0; o >>= 1)
    for (int q = 0; q < 3; q++) prod.w[q] ^= __shfl_xor_sync(0xffffffffu, prod.w[q], o);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < 3; q++) red[warp][q] = prod.w[q];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int half = threadIdx.x / 3, q = threadIdx.x % 3;
    uint64_t x = 0;
    for (int w = 0; w < 4; w++) x ^= red[4 * half + w][q];
    s.s->msg[3 * half + q] = x;
  }
}

__device__ __forceinline__ void load_table(F162d* dst, const uint64_t* src, int entries) {
  for (int e = threadIdx.x; e < entries; e += blockDim.x) dst[e] = ld_f(src, e);
}

__device__ __forceinline__ F162d psi_of(const F162d* __restrict__ tab, B128d e) {
  F162d acc{{0, 0, 0}};
#pragma unroll
  for (int c = 0; c < 32; c++) {
    uint32_t nib = (uint32_t)((c < 16 ? e.lo >> (4 * c) : e.hi >> (4 * (c - 16))) & 15);
    acc = f_add(acc, tab[16 * c + nib]);
  }
  return acc;
}

// x r through the round's tables: T[16 i + t] = (t x^{4i}) r, 41 nibble positions (32 when x
// has at most 128 bits).
template <int POS = 41>
__device__ __forceinline__ F162d cmul(const F162d* __restrict__ T, F162d x) {
  F162d acc{{0, 0, 0}};
#pragma unroll
  for (int i = 0; i < POS; i++) {
    uint32_t nib = (uint32_t)(x.w[i >> 4] >> (4 * (i & 15))) & 15;
    acc = f_add(acc, T[16 * i + nib]);
  }
  return acc;
}

__device__ __forceinline__ void xor_reduce_store(F162d e0, F162d ei, uint64_t* msg) {
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      e0.w[k] ^= __shfl_xor_sync(0xffffffffu, e0.w[k], o);
      ei.w[k] ^= __shfl_xor_sync(0xffffffffu, ei.w[k], o);
    }
  }
  if ((threadIdx.x & 31) == 0) {
    unsigned long long* m = reinterpret_cast<unsigned long long*>(msg);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      atomicXor(m + k, (unsigned long long)e0.w[k]);
      atomicXor(m + 3 + k, (unsigned long long)ei.w[k]);
    }
  }
}

// The transcript step of round k of one instance, on the whole block (it ends with a barrier):
// the round's message msg (six words in shared memory) recorded and absorbed, then
// sample_f162("labinius/switch-round", 1) (crates/pcs/src/switch.rs:152-159), both staged behind
// the open block of sh, the block's shared copy of the instance's transcript hasher; the challenge
// recorded and R4[i] = r x^{4i}, i < 41.
__device__ void sw_transcript_step(const SwInst& s, int k, HasherState& sh, const uint64_t* msg, F162d* R4) {
  SwSmall* sm = s.s;
  __shared__ uint32_t stage[32];
  __shared__ uint32_t last;
  uint8_t* bytes = reinterpret_cast<uint8_t*>(stage);
  if (threadIdx.x < 6) sm->rounds[k][threadIdx.x] = msg[threadIdx.x];
  // absorb_f162(&msg): the open block, le64(2), the six words
  const uint32_t bl = sh.buf_len, total = bl + 56;
  for (uint32_t b = threadIdx.x; b < 128; b += blockDim.x) {
    uint32_t x = 0;
    if (b < bl) x = sh.buf[b];
    else if (b < bl + 8) x = b == bl ? 2 : 0;
    else if (b < total) x = (uint32_t)(msg[(b - bl - 8) / 8] >> (8 * ((b - bl) % 8))) & 0xFF;
    bytes[b] = (uint8_t)x;
  }
  __syncthreads();
  if (threadIdx.x == 0) last = dev::hs_absorb_staged(&sh, stage, total);
  __syncthreads();
  const uint32_t nbl = total - last;
  for (uint32_t b = threadIdx.x; b < nbl; b += blockDim.x) sh.buf[b] = bytes[last + b];
  __syncthreads();
  // derive("labinius/switch-round"): the open block, le64(counter), le64(21), the label
  const uint64_t counter = s.counter0 + 1 + (uint64_t)k;
  const uint32_t dtotal = nbl + 37;
  for (uint32_t b = threadIdx.x; b < 128; b += blockDim.x) {
    uint32_t x = 0;
    if (b < nbl) x = sh.buf[b];
    else if (b < nbl + 8) x = (uint32_t)(counter >> (8 * (b - nbl))) & 0xFF;
    else if (b < nbl + 16) x = b == nbl + 8 ? 21 : 0;
    else if (b < dtotal) x = (uint8_t)c_sw_round[b - nbl - 16];
    bytes[b] = (uint8_t)x;
  }
  if (threadIdx.x == 0) sh.buf_len = nbl;
  __syncthreads();
  if (threadIdx.x == 0) {
    XofRoot root;
    dev::hs_derive_staged(&sh, stage, dtotal, root);
    uint32_t out[16];
    dev::root_block_ool(root, 0, out);
    F162d r;
    for (int w = 0; w < 3; w++) r.w[w] = (uint64_t)out[2 * w] | ((uint64_t)out[2 * w + 1] << 32);
    r.w[2] &= (1ull << 34) - 1;
    st_f(&sm->rr[0][0], k, r);
    for (int q = 0; q < 41; q++) {
      R4[q] = r;
      r = f_times_x4(r);
    }
  }
  __syncthreads();
}

// Entry e of the round's product tables: (t x^{4i}) r at e = 16 i + t, from R4[i] = r x^{4i}.
__device__ __forceinline__ F162d rtab_entry(const F162d* R4, int e) {
  F162d x = R4[e >> 4], acc{{0, 0, 0}};
  for (int b = 0; b < 4; b++) {
    if ((e >> b) & 1) acc = f_add(acc, x);
    x = f_times_x(x);
  }
  return acc;
}

// One block per instance whose round k is due (k below its tail): the round's transcript step;
// the message accumulators cleared; the tables of (t x^{4i}) r for the fold, and for round 0 the
// psi tables times r.
__global__ void k_sw_step(const SwInst* __restrict__ I, int k) {
  const SwInst& s = I[blockIdx.x];
  if ((uint32_t)k >= sw_tail_start(s.l)) return;
  SwSmall* sm = s.s;
  __shared__ HasherState sh;
  __shared__ F162d R4[41];
  __shared__ uint64_t msg[6];
  dev::hs_copy(&sh, s.st);
  if (threadIdx.x < 6) msg[threadIdx.x] = sm->msg[threadIdx.x];
  __syncthreads();
  if (threadIdx.x < 6) sm->msg[threadIdx.x] = 0;
  sw_transcript_step(s, k, sh, msg, R4);
  dev::hs_copy(s.st, &sh);
  if (k == 0) {
    const F162d r = R4[0];
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) st_f(&sm->rpsi[0][0], e, f_mul(ld_f(&sm->psi[0][0], e), r));
  }
  for (int e = threadIdx.x; e < 41 * 16; e += blockDim.x) st_f(&sm->rtab[0][0], e, rtab_entry(R4, e));
}

// Round k's fold with its challenge (x0 + r (x0 + x1) over the pairs (j, j + half) of tables of
// 2 half entries) and, when half >= 2, round k + 1's message over the pairs (j, j + half/2) of
// the folded tables. FIRST (k = 0) reads the tables through eq and the trace and writes the
// folded ones; later rounds fold in place.
// Out-of-line products for the rounds where a thread folds at most one pair (k_sw_fold_small,
// k_sw_fold_split, k_sw_tail): one copy of each in the kernel's code, so the few instructions each thread runs are
// fetched once per SM instead of once per inlined copy.
__device__ __noinline__ F162d f_mul_ool(F162d a, F162d b) { return f_mul(a, b); }
__device__ __noinline__ F162d cmul_ool(const F162d* T, F162d x) { return cmul<41>(T, x); }

template <bool FIRST>
__global__ void __launch_bounds__(SW_THREADS) k_sw_fold(const SwInst* __restrict__ I, int count, int k) {
  // round 0 multiplies only 128-bit words (trace pairs) by r, so it needs 32 of the 41 positions
  __shared__ F162d T[(FIRST ? 32 : 41) * 16];
  __shared__ F162d psi[FIRST ? 512 : 1];
  __shared__ F162d rpsi[FIRST ? 512 : 1];
  uint32_t local, nblk;
  int i = sw_find(I, count, 2, k, SW_THREADS, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  load_table(T, &s.s->rtab[0][0], (FIRST ? 32 : 41) * 16);
  if (FIRST) {
    load_table(psi, &s.s->psi[0][0], 512);
    load_table(rpsi, &s.s->rpsi[0][0], 512);
  }
  __syncthreads();
  const size_t half = (1ull << s.l) >> (k + 1);
  // the folded entry x (x < half) of both tables
  auto fold_at = [&](size_t x, F162d& na, F162d& np) {
    if (FIRST) {
      // psi is GF(2)-linear, so r psi(q0 + q1) reads r psi's own tables
      B128d q0 = ld_b(s.eq, x), q1 = ld_b(s.eq, x + half);
      na = f_add(psi_of(psi, q0), psi_of(rpsi, b_add(q0, q1)));
      F162d p0 = ld_word(s.w, x), p1 = ld_word(s.w, x + half);
      np = f_add(p0, cmul<32>(T, f_add(p0, p1)));
    } else {
      F162d a0 = ld_f(s.a, x), a1 = ld_f(s.a, x + half);
      na = f_add(a0, cmul(T, f_add(a0, a1)));
      F162d p0 = ld_f(s.p, x), p1 = ld_f(s.p, x + half);
      np = f_add(p0, cmul(T, f_add(p0, p1)));
    }
  };
  if (half < 2) {
    if (local == 0 && threadIdx.x == 0) {
      F162d na, np;
      fold_at(0, na, np);
      st_f(s.a, 0, na);
      st_f(s.p, 0, np);
    }
    return;
  }
  const size_t h2 = half / 2;
  F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
  for (size_t j = (size_t)local * SW_THREADS + threadIdx.x; j < h2; j += (size_t)nblk * SW_THREADS) {
    F162d na, pa, nb, pb;
    fold_at(j, na, pa);
    fold_at(j + h2, nb, pb);
    st_f(s.a, j, na);
    st_f(s.a, j + h2, nb);
    st_f(s.p, j, pa);
    st_f(s.p, j + h2, pb);
    e0 = f_add(e0, f_mul(na, pa));
    ei = f_add(ei, f_mul(f_add(na, nb), f_add(pa, pb)));
  }
  xor_reduce_store(e0, ei, &s.s->msg[0]);
}

// k_sw_fold for a round k >= 1 whose launch gives every thread at most one pair (half >= 2): the
// same arithmetic through one out-of-line copy of each product. Such rounds are bound by the
// latency of one thread's work, not by throughput.
__global__ void __launch_bounds__(SW_THREADS) k_sw_fold_small(const SwInst* __restrict__ I, int count, int k) {
  __shared__ F162d T[41 * 16];
  uint32_t local, nblk;
  int i = sw_find(I, count, 2, k, SW_THREADS, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  load_table(T, &s.s->rtab[0][0], 41 * 16);
  __syncthreads();
  const size_t half = (1ull << s.l) >> (k + 1);
  const size_t h2 = half / 2;
  F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
  for (size_t j = (size_t)local * SW_THREADS + threadIdx.x; j < h2; j += (size_t)nblk * SW_THREADS) {
    F162d na[2], np[2];
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
      const size_t x = j + h * h2;
      F162d a0 = ld_f(s.a, x), a1 = ld_f(s.a, x + half), p0 = ld_f(s.p, x), p1 = ld_f(s.p, x + half);
      na[h] = f_add(a0, cmul_ool(T, f_add(a0, a1)));
      np[h] = f_add(p0, cmul_ool(T, f_add(p0, p1)));
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      st_f(s.a, j + h * h2, na[h]);
      st_f(s.p, j + h * h2, np[h]);
    }
    e0 = f_add(e0, f_mul_ool(na[0], np[0]));
    ei = f_add(ei, f_mul_ool(f_add(na[0], na[1]), f_add(np[0], np[1])));
  }
  xor_reduce_store(e0, ei, &s.s->msg[0]);
}

// k_sw_fold_small for rounds whose pairs leave most of the GPU idle, with a pair's work spread over
// four warps: warps 4g + r of a CTA take the pairs 32 g + lane of the CTA's 64; warp role r folds
// one of the pair's four entries (entry j + (r >> 1) h2 of table a or p by r & 1) through the
// round's product tables, then roles 0 and 1 make the message's two products and roles 2 and 3
// store the folded entries (every read of them is done by then). A thread's sequential work is
// one product by r and at most one general product instead of four and two.
constexpr int SW_SPLIT_PAIRS = 64;
__global__ void __launch_bounds__(SW_THREADS) k_sw_fold_split(const SwInst* __restrict__ I, int count, int k) {
  __shared__ F162d T[41 * 16];
  __shared__ F162d N[2][4][32];
  uint32_t local, nblk;
  int i = sw_find(I, count, 2, k, SW_SPLIT_PAIRS, local, nblk);
  if (i < 0) return;
  const SwInst& s = I[i];
  load_table(T, &s.s->rtab[0][0], 41 * 16);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = warp >> 2, r = warp & 3;
  const size_t half = (1ull << s.l) >> (k + 1), h2 = half / 2;
  F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
  for (size_t base = (size_t)local * SW_SPLIT_PAIRS; base < h2; base += (size_t)nblk * SW_SPLIT_PAIRS) {
    __syncthreads();  // the tables are loaded, and the last pass is done with N
    const size_t j = base + 32 * g + lane;
    const bool on = j < h2;
    if (on) {
      const uint64_t* tab = (r & 1) ? s.p : s.a;
      const size_t x = j + (size_t)(r >> 1) * h2;
      const F162d v0 = ld_f(tab, x), v1 = ld_f(tab, x + half);
      N[g][r][lane] = f_add(v0, cmul_ool(T, f_add(v0, v1)));
    }
    __syncthreads();
    if (on) {
      const F162d na0 = N[g][0][lane], np0 = N[g][1][lane], na1 = N[g][2][lane], np1 = N[g][3][lane];
      if (r == 0) {
        e0 = f_add(e0, f_mul_ool(na0, np0));
      } else if (r == 1) {
        ei = f_add(ei, f_mul_ool(f_add(na0, na1), f_add(np0, np1)));
      } else if (r == 2) {
        st_f(s.a, j, na0);
        st_f(s.a, j + h2, na1);
      } else {
        st_f(s.p, j, np0);
        st_f(s.p, j + h2, np1);
      }
    }
  }
  xor_reduce_store(e0, ei, &s.s->msg[0]);
}

// The opened value p[0] and the evaluation point, msb_first
// (crates/pcs/src/scheme/commitment.rs:163-174): p0[i] = r_(l-1-i), p1[i] = r_(col_log-1-i).
__device__ void sw_finish(const SwInst& s) {
  SwSmall* sm = s.s;
  for (int w = 0; w < 3; w++) sm->opened[w] = s.p[w];
  if (s.p0)
    for (uint32_t q = 0; q < s.row_log; q++)
      for (int w = 0; w < 3; w++) s.p0[3 * q + w] = sm->rr[s.l - 1 - q][w];
  if (s.p1)
    for (uint32_t q = 0; q < s.col_log; q++)
      for (int w = 0; w < 3; w++) s.p1[3 * q + w] = sm->rr[s.col_log - 1 - q][w];
  sm->status = 1;
}

// One block per instance: the rounds from sw_tail_start(l) on (each its transcript step, then its
// fold and the next round's message, XOR-reduced over the block), with the hasher, the message
// and the product tables in shared memory; then the opened value and the point.
constexpr int SW_TAIL_THREADS = 256;
__global__ void __launch_bounds__(SW_TAIL_THREADS) k_sw_tail(const SwInst* __restrict__ I) {
  const SwInst& s = I[blockIdx.x];
  SwSmall* sm = s.s;
  __shared__ HasherState sh;
  __shared__ F162d R4[41];
  __shared__ F162d T[41 * 16];
  __shared__ uint64_t msg[6];
  __shared__ uint64_t red[SW_TAIL_THREADS / 32][6];
  __shared__ F162d N[2][4][32];
  const uint32_t kt = sw_tail_start(s.l);
  if (kt < s.l) {
    dev::hs_copy(&sh, s.st);
    if (threadIdx.x < 6) msg[threadIdx.x] = sm->msg[threadIdx.x];
    __syncthreads();
    for (uint32_t k = kt; k < s.l; k++) {
      sw_transcript_step(s, (int)k, sh, msg, R4);
      for (int e = threadIdx.x; e < 41 * 16; e += blockDim.x) T[e] = rtab_entry(R4, e);
      __syncthreads();
      const uint32_t half = 1u << (s.l - k - 1);
      if (half < 2) {
        if (threadIdx.x == 0) {
          F162d a0 = ld_f(s.a, 0), a1 = ld_f(s.a, 1), p0 = ld_f(s.p, 0), p1 = ld_f(s.p, 1);
          st_f(s.a, 0, f_add(a0, cmul_ool(T, f_add(a0, a1))));
          st_f(s.p, 0, f_add(p0, cmul_ool(T, f_add(p0, p1))));
        }
      } else {
        const uint32_t h2 = half / 2;
        F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
        if (h2 <= (uint32_t)SW_SPLIT_PAIRS) {
          // at most 64 pairs: a pair's four entries and two products over four warps, as
          // k_sw_fold_split does
          const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = warp >> 2, r = warp & 3;
          const uint32_t j = 32 * g + lane;
          const bool on = j < h2;
          if (on) {
            const uint64_t* tab = (r & 1) ? s.p : s.a;
            const uint32_t x = j + (uint32_t)(r >> 1) * h2;
            const F162d v0 = ld_f(tab, x), v1 = ld_f(tab, x + half);
            N[g][r][lane] = f_add(v0, cmul_ool(T, f_add(v0, v1)));
          }
          __syncthreads();
          if (on) {
            const F162d na0 = N[g][0][lane], np0 = N[g][1][lane], na1 = N[g][2][lane], np1 = N[g][3][lane];
            if (r == 0) {
              e0 = f_mul_ool(na0, np0);
            } else if (r == 1) {
              ei = f_mul_ool(f_add(na0, na1), f_add(np0, np1));
            } else if (r == 2) {
              st_f(s.a, j, na0);
              st_f(s.a, j + h2, na1);
            } else {
              st_f(s.p, j, np0);
              st_f(s.p, j + h2, np1);
            }
          }
        } else {
          for (uint32_t j = threadIdx.x; j < h2; j += blockDim.x) {
            F162d na[2], np[2];
#pragma unroll 1
            for (int h = 0; h < 2; h++) {
              const uint32_t x = j + h * h2;
              F162d a0 = ld_f(s.a, x), a1 = ld_f(s.a, x + half), p0 = ld_f(s.p, x), p1 = ld_f(s.p, x + half);
              na[h] = f_add(a0, cmul_ool(T, f_add(a0, a1)));
              np[h] = f_add(p0, cmul_ool(T, f_add(p0, p1)));
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
              st_f(s.a, j + h * h2, na[h]);
              st_f(s.p, j + h * h2, np[h]);
            }
            e0 = f_add(e0, f_mul_ool(na[0], np[0]));
            ei = f_add(ei, f_mul_ool(f_add(na[0], na[1]), f_add(np[0], np[1])));
          }
        }
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int w = 0; w < 3; w++) {
            e0.w[w] ^= __shfl_xor_sync(0xffffffffu, e0.w[w], o);
            ei.w[w] ^= __shfl_xor_sync(0xffffffffu, ei.w[w], o);
          }
        if ((threadIdx.x & 31) == 0)
#pragma unroll
          for (int w = 0; w < 3; w++) {
            red[threadIdx.x >> 5][w] = e0.w[w];
            red[threadIdx.x >> 5][3 + w] = ei.w[w];
          }
        __syncthreads();
        if (threadIdx.x < 6) {
          uint64_t x = 0;
          for (int w = 0; w < SW_TAIL_THREADS / 32; w++) x ^= red[w][threadIdx.x];
          msg[threadIdx.x] = x;
        }
      }
      __syncthreads();
    }
    dev::hs_copy(s.st, &sh);
  }
  __syncthreads();
  if (threadIdx.x == 0) sw_finish(s);
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

size_t sw_scratch_bytes(uint32_t l) {
  uint32_t lh = l / 2, ll = l - lh;
  size_t n = (size_t)1 << l, half = std::max<size_t>(n / 2, 1);
  return align256((size_t)16 << lh) + align256((size_t)16 << ll) + align256(16 * n) + 2 * align256(24 * half);
}

void sw_layout(SwInst& I, uint8_t* base) {
  I.lh = I.l / 2;
  I.ll = I.l - I.lh;
  size_t n = (size_t)1 << I.l, half = std::max<size_t>(n / 2, 1);
  I.e_hi = (uint64_t*)base;
  base += align256((size_t)16 << I.lh);
  I.e_lo = (uint64_t*)base;
  base += align256((size_t)16 << I.ll);
  I.eq = (uint64_t*)base;
  base += align256(16 * n);
  I.a = (uint64_t*)base;
  base += align256(24 * half);
  I.p = (uint64_t*)base;
}

uint64_t sw_launches(const SwInst* h, int count) {
  if (count <= 0) return 0;
  uint32_t ktmax = 0;
  bool short_eq = false, seg_eq = false;
  for (int i = 0; i < count; i++) {
    ktmax = std::max(ktmax, sw_tail_start(h[i].l));
    short_eq |= sw_units(h[i].l, 3, 0) > 0;
    seg_eq |= sw_units(h[i].l, 4, 0) > 0;
  }
  return 5 + (short_eq ? 1 : 0) + (seg_eq ? 1 : 0) + 2 * (uint64_t)ktmax;
}

cudaError_t enqueue_switch(const SwInst* d, const SwInst* h, int count, cudaStream_t st, uint64_t* launches) {
  if (count <= 0) return cudaSuccess;
  uint32_t ktmax = 0, tabmax = 0;
  for (int i = 0; i < count; i++) {
    ktmax = std::max(ktmax, sw_tail_start(h[i].l));
    tabmax = std::max(tabmax, (1u << h[i].lh) + (1u << h[i].ll));
  }
  auto blocks = [&](int stage, int k, int per) {
    uint64_t t = 0;
    for (int i = 0; i < count; i++) t += sw_blocks(sw_units(h[i].l, stage, k), per);
    return (unsigned)t;
  };
  k_sw_tables<<<dim3((tabmax + 127) / 128, count), 128, 0, st>>>(d);
  if (unsigned g = blocks(3, 0, SW_THREADS)) k_sw_eq<<<g, SW_THREADS, 0, st>>>(d, count);
  if (unsigned g = blocks(4, 0, 1)) k_sw_eq_seg<<<g, SW_THREADS, 0, st>>>(d, count);
  k_sw_sums<<<blocks(1, 0, SW_SUM_ROWS), SW_THREADS, 0, st>>>(d, count);
  k_sw_statement<<<count, 128, 0, st>>>(d);
  k_sw_batch<<<count, 256, 0, st>>>(d);
  for (uint32_t k = 0; k < ktmax; k++) {
    k_sw_step<<<count, 128, 0, st>>>(d, (int)k);
    unsigned g = blocks(2, (int)k, SW_THREADS);
    if (k == 0) {
      k_sw_fold<true><<<g, SW_THREADS, 0, st>>>(d, count, 0);
    } else {
      // a launch that gives every thread at most one pair of a round with a message to compute
      uint64_t most = 0;
      bool last = false;
      for (int i = 0; i < count; i++) {
        most = std::max(most, sw_units(h[i].l, 2, (int)k));
        last |= (uint32_t)k + 1 == h[i].l;
      }
      if (!last && most <= (uint64_t)SW_CAP * SW_SPLIT_PAIRS)
        k_sw_fold_split<<<blocks(2, (int)k, SW_SPLIT_PAIRS), SW_THREADS, 0, st>>>(d, count, (int)k);
      else if (!last && most <= (uint64_t)SW_CAP * SW_THREADS)
        k_sw_fold_small<<<g, SW_THREADS, 0, st>>>(d, count, (int)k);
      else
        k_sw_fold<false><<<g, SW_THREADS, 0, st>>>(d, count, (int)k);
    }
  }
  k_sw_tail<<<count, SW_TAIL_THREADS, 0, st>>>(d);
  if (launches) *launches += sw_launches(h, count);
  return cudaGetLastError();
}

}  // namespace lbg

using namespace lbg;

namespace {
int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

size_t al256(size_t b) { return (b + 255) / 256 * 256; }

// Bytes in front of the scratch in the entry point's workspace: the instance's small values, its
// table entry, its hasher state and its coordinates (32 slots of r_hi, then r_lo).
size_t sw_head_bytes() {
  return al256(sizeof(SwSmall)) + al256(sizeof(SwInst)) + al256(sizeof(HasherState)) + al256(39 * 16);
}
}  // namespace

void lbg_switch_release(lbg_pp* pp) {
  if (pp && pp->d_sw) {
    cudaFree(pp->d_sw);
    pp->d_sw = nullptr;
  }
}

extern "C" {

int lbg_switch_prove(const lbg_pp* pp_c, const lbg_witness* w, const uint64_t* r_lo, size_t nlo, const uint64_t* r_hi,
                     size_t l, const uint64_t claim[2], lbg_transcript* t, uint64_t* partials, uint64_t* rounds,
                     uint64_t opened[3], uint64_t* p0_out, uint64_t* p1_out) {
  if (!pp_c || !w || !r_hi || !claim || !t || !partials || !rounds || !opened || !p0_out || !p1_out ||
      (nlo && !r_lo))
    return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (l != pp->params.witness_log_len || w->n != pp->n) return fail(LBG_ERR_INVALID, "the point does not match the parameters");
  if (nlo != 0 && nlo != 7) return fail(LBG_ERR_INVALID, "a bit-level point has 7 low coordinates");
  if (l < 1 || l > 32) return fail(LBG_ERR_INVALID, "the trace has 2^1 .. 2^32 words");
  Transcript& tr = t->t;
  std::lock_guard<std::mutex> g(pp->mu);
  if (cudaSetDevice(pp->device) != cudaSuccess) return fail(LBG_ERR_CUDA, "cudaSetDevice");
  cudaStream_t st = pp->stream;
  if (!pp->d_sw) {
    if (cudaMalloc((void**)&pp->d_sw, sw_head_bytes() + sw_scratch_bytes((uint32_t)l)) != cudaSuccess) {
      cudaGetLastError();
      pp->d_sw = nullptr;
      return fail(LBG_ERR_OOM, "switch: device allocation failed");
    }
  }
  uint8_t* base = pp->d_sw;
  SwSmall* d_small = (SwSmall*)base;
  base += al256(sizeof(SwSmall));
  SwInst* d_inst = (SwInst*)base;
  base += al256(sizeof(SwInst));
  HasherState* d_st = (HasherState*)base;
  base += al256(sizeof(HasherState));
  uint64_t* d_r = (uint64_t*)base;
  base += al256(39 * 16);

  SwInst h;
  std::memset(&h, 0, sizeof(h));
  h.w = w->d;
  h.r_hi = d_r;
  h.r_lo = nlo ? d_r + 2 * 32 : nullptr;
  h.s = d_small;
  h.st = d_st;
  h.counter0 = tr.counter();
  h.l = (uint32_t)l;
  h.nlo = (uint32_t)nlo;
  h.row_log = (uint32_t)(l - pp->params.column_log_len);
  h.col_log = pp->params.column_log_len;
  h.claim_given = 1;
  sw_layout(h, base);
  HasherState hs;
  tr.state().save(hs);
  std::vector<uint64_t> rbuf(2 * 39, 0);
  std::memcpy(rbuf.data(), r_hi, l * 16);
  if (nlo) std::memcpy(rbuf.data() + 2 * 32, r_lo, nlo * 16);
  std::vector<SwSmall> out(1);
  cudaError_t e = cudaMemsetAsync(d_small, 0, sizeof(SwSmall), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_small->claim, claim, 16, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_st, &hs, sizeof(hs), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_r, rbuf.data(), rbuf.size() * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_inst, &h, sizeof(h), cudaMemcpyHostToDevice, st);
  uint64_t launches = 0;
  if (e == cudaSuccess) e = enqueue_switch(d_inst, &h, 1, st, &launches);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d_small, sizeof(SwSmall), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, d_st, sizeof(hs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("switch: ") + cudaGetErrorString(e));
  const SwSmall& o = out[0];
  if (o.status != 1) return fail(LBG_ERR_CUDA, "switch: the device pass did not complete");
  tr.state().load(hs);
  tr.set_counter(h.counter0 + 1 + l);
  std::memcpy(partials, o.v, 128 * 16);
  std::memcpy(rounds, o.rounds, l * 48);
  std::memcpy(opened, o.opened, 24);
  // EvaluationPoint::msb_first (crates/pcs/src/scheme/commitment.rs:163-174)
  size_t cl = pp->params.column_log_len, rows = l - cl;
  for (size_t i = 0; i < rows; i++) std::memcpy(p0_out + 3 * i, o.rr[l - 1 - i], 24);
  for (size_t i = 0; i < cl; i++) std::memcpy(p1_out + 3 * i, o.rr[cl - 1 - i], 24);
  return LBG_OK;
}

}  // extern "C"
