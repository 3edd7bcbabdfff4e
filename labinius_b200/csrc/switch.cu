// The cross-field switch prover on the device (crates/pcs/src/switch.rs:133-168,
// crates/pcs/src/fields/crossfield.rs, crates/pcs/src/fields/sumcheck.rs).
//
// A B128 trace committed as Witness::lifted carries a claim in B128; the switch turns it into the
// F162 claim the commitment opens at the point its sumcheck ends on. The prover's work is three
// passes over the trace and a sumcheck of l rounds:
//  * eq_hi = the expansion of r_hi (one B128 product per entry, from two half-size tables);
//  * the 128 partial evaluations v[k] = sum_j bit_k(trace_j) eq_hi[j];
//  * a_j = psi(eq_hi[j]) = sum_k bit_k(eq_hi[j]) batch[k] (byte tables of the batch in shared
//    memory), p_j = the trace word as an F162;
//  * each round sends (sum a0 p0, sum (a0 + a1)(p0 + p1)) over the index pairs (j, j + half),
//    then folds both tables with the round's challenge r: x0 + r (x0 + x1). The fold of round k
//    and the message of round k + 1 are one kernel; products by r go through 4-bit tables of
//    r x^i in shared memory.
// The transcript stays on the host (the prover's lbg_transcript): one short exchange per round.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "error.h"
#include "gf2_dev.cuh"
#include "handles.h"
#include "transcript.h"

using namespace lbg;

namespace {

int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

// Entry idx of the expansion of r[0..m): the product over rounds of r_round or 1 + r_round, by
// bit m-1-round of idx (crates/pcs/src/fields/crossfield.rs:78-98: the last coordinate is bit 0).
__global__ void k_sw_eq_tables(const B128d* __restrict__ r, int lh, int ll, B128d* __restrict__ e_hi,
                               B128d* __restrict__ e_lo) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int nh = 1 << lh, nl = 1 << ll;
  if (g >= nh + nl) return;
  bool high = g < nh;
  int idx = high ? g : g - nh;
  int m = high ? lh : ll;
  const B128d* rr = high ? r : r + lh;
  B128d acc{1, 0};
  for (int round = 0; round < m; round++) {
    B128d f = rr[round];
    if (!((idx >> (m - 1 - round)) & 1)) f.lo ^= 1;
    acc = b_mul(acc, f);
  }
  (high ? e_hi : e_lo)[idx] = acc;
}

__global__ void k_sw_eq(const B128d* __restrict__ e_hi, const B128d* __restrict__ e_lo, int ll, size_t n,
                        B128d* __restrict__ eq) {
  size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  eq[j] = b_mul(e_hi[j >> ll], e_lo[j & ((1ull << ll) - 1)]);
}

// v[k] = sum_j bit_k(trace_j) eq[j]: thread (sub, m) of a CTA adds, for its rows j, eq[j] into
// the 8 partial sums of bits 8m .. 8m+7; the 16 row groups are then XOR-reduced and added to v.
__global__ void __launch_bounds__(256) k_sw_partials(const uint64_t* __restrict__ W, const B128d* __restrict__ eq,
                                                     size_t n, unsigned long long* __restrict__ v) {
  __shared__ uint64_t red[16][128][2];
  const int sub = threadIdx.x >> 4, m = threadIdx.x & 15;
  uint64_t S[8][2];
#pragma unroll
  for (int r = 0; r < 8; r++) S[r][0] = S[r][1] = 0;
  for (size_t j = (size_t)blockIdx.x * 16 + sub; j < n; j += (size_t)gridDim.x * 16) {
    uint64_t word = __ldg(W + 3 * j + (m >> 3));
    uint32_t byte = (uint32_t)(word >> (8 * (m & 7))) & 0xFF;
    B128d e = eq[j];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      uint64_t msk = 0 - (uint64_t)((byte >> r) & 1);
      S[r][0] ^= e.lo & msk;
      S[r][1] ^= e.hi & msk;
    }
  }
#pragma unroll
  for (int r = 0; r < 8; r++) {
    red[sub][8 * m + r][0] = S[r][0];
    red[sub][8 * m + r][1] = S[r][1];
  }
  __syncthreads();
  if (threadIdx.x < 128) {
    uint64_t a = 0, b = 0;
    for (int s = 0; s < 16; s++) {
      a ^= red[s][threadIdx.x][0];
      b ^= red[s][threadIdx.x][1];
    }
    atomicXor(v + 2 * threadIdx.x, (unsigned long long)a);
    atomicXor(v + 2 * threadIdx.x + 1, (unsigned long long)b);
  }
}

// batch = the expansion of the 7 sampled F162 (crossfield.rs:65-76); psi[c][t] = the XOR of
// batch[8c + b] over the set bits b of t (crossfield.rs:112-130). One CTA of 256 threads.
__global__ void k_sw_batch(const F162d* __restrict__ rp, F162d* __restrict__ batch, F162d* __restrict__ psi) {
  __shared__ F162d t[2][128];
  if (threadIdx.x == 0) t[0][0] = F162d{{1, 0, 0}};
  __syncthreads();
  int cur = 0;
  for (int round = 0; round < 7; round++) {
    int size = 1 << round;
    if ((int)threadIdx.x < size) {
      F162d x = t[cur][threadIdx.x];
      F162d h = f_mul(x, rp[round]);
      t[cur ^ 1][2 * threadIdx.x] = f_add(x, h);
      t[cur ^ 1][2 * threadIdx.x + 1] = h;
    }
    __syncthreads();
    cur ^= 1;
  }
  if (threadIdx.x < 128) batch[threadIdx.x] = t[cur][threadIdx.x];
  for (int e = threadIdx.x; e < 16 * 256; e += blockDim.x) {
    int c = e >> 8, v = e & 255;
    F162d acc{{0, 0, 0}};
    for (int b = 0; b < 8; b++)
      if ((v >> b) & 1) acc = f_add(acc, t[cur][8 * c + b]);
    psi[e] = acc;
  }
}

__device__ __forceinline__ void xor_reduce_store(F162d e0, F162d ei, unsigned long long* msg) {
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      e0.w[k] ^= __shfl_xor_sync(0xffffffffu, e0.w[k], o);
      ei.w[k] ^= __shfl_xor_sync(0xffffffffu, ei.w[k], o);
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      atomicXor(msg + k, (unsigned long long)e0.w[k]);
      atomicXor(msg + 3 + k, (unsigned long long)ei.w[k]);
    }
  }
}

__device__ __forceinline__ F162d psi_of(const F162d* __restrict__ tab, B128d e) {
  F162d acc{{0, 0, 0}};
#pragma unroll
  for (int c = 0; c < 16; c++) {
    uint32_t byte = (uint32_t)((c < 8 ? e.lo >> (8 * c) : e.hi >> (8 * (c - 8))) & 0xFF);
    acc = f_add(acc, tab[c * 256 + byte]);
  }
  return acc;
}

// a and p of every index, and round 0's message over the pairs (j, j + n/2).
__global__ void __launch_bounds__(256) k_sw_init(const uint64_t* __restrict__ W, const B128d* __restrict__ eq,
                                                 const F162d* __restrict__ psi_g, size_t n, F162d* __restrict__ a,
                                                 F162d* __restrict__ p, unsigned long long* __restrict__ msg) {
  extern __shared__ F162d psi[];  // [16][256]
  for (int e = threadIdx.x; e < 16 * 256; e += blockDim.x) psi[e] = psi_g[e];
  __syncthreads();
  const size_t h = n / 2;
  F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < h; j += (size_t)gridDim.x * blockDim.x) {
    F162d a0 = psi_of(psi, eq[j]), a1 = psi_of(psi, eq[j + h]);
    F162d p0{{W[3 * j], W[3 * j + 1], 0}}, p1{{W[3 * (j + h)], W[3 * (j + h) + 1], 0}};
    a[j] = a0;
    a[j + h] = a1;
    p[j] = p0;
    p[j + h] = p1;
    e0 = f_add(e0, f_mul(a0, p0));
    ei = f_add(ei, f_mul(f_add(a0, a1), f_add(p0, p1)));
  }
  xor_reduce_store(e0, ei, msg);
}

// x r through 4-bit tables: T[i][t] = (t x^{4i}) r, 41 nibble positions.
__device__ __forceinline__ F162d cmul(const F162d* __restrict__ T, F162d x) {
  F162d acc{{0, 0, 0}};
#pragma unroll
  for (int i = 0; i < 41; i++) {
    uint32_t nib = (uint32_t)(x.w[i >> 4] >> (4 * (i & 15))) & 15;
    acc = f_add(acc, T[16 * i + nib]);
  }
  return acc;
}

// Fold both tables with r (x0 + r (x0 + x1) over the pairs (j, j + half)); when half >= 2, also
// the next round's message over the pairs (j, j + half/2) of the folded tables.
__global__ void __launch_bounds__(256) k_sw_round(F162d* __restrict__ a, F162d* __restrict__ p, size_t half,
                                                  const F162d* __restrict__ rr, unsigned long long* __restrict__ msg) {
  __shared__ F162d R[164];
  __shared__ F162d T[41 * 16];
  if (threadIdx.x == 0) {
    F162d x = *rr;
    for (int k = 0; k < 164; k++) {
      R[k] = x;
      x = f_times_x(x);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 41 * 16; e += blockDim.x) {
    int i = e >> 4, t = e & 15;
    F162d acc{{0, 0, 0}};
    for (int b = 0; b < 4; b++)
      if ((t >> b) & 1) acc = f_add(acc, R[4 * i + b]);
    T[e] = acc;
  }
  __syncthreads();
  if (half < 2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a[0] = f_add(a[0], cmul(T, f_add(a[0], a[1])));
      p[0] = f_add(p[0], cmul(T, f_add(p[0], p[1])));
    }
    return;
  }
  const size_t h2 = half / 2;
  F162d e0{{0, 0, 0}}, ei{{0, 0, 0}};
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < h2; j += (size_t)gridDim.x * blockDim.x) {
    F162d x0 = a[j], x1 = a[j + half], y0 = a[j + h2], y1 = a[j + h2 + half];
    F162d na = f_add(x0, cmul(T, f_add(x0, x1))), nb = f_add(y0, cmul(T, f_add(y0, y1)));
    F162d u0 = p[j], u1 = p[j + half], v0 = p[j + h2], v1 = p[j + h2 + half];
    F162d pa = f_add(u0, cmul(T, f_add(u0, u1))), pb = f_add(v0, cmul(T, f_add(v0, v1)));
    a[j] = na;
    a[j + h2] = nb;
    p[j] = pa;
    p[j + h2] = pb;
    e0 = f_add(e0, f_mul(na, pa));
    ei = f_add(ei, f_mul(f_add(na, nb), f_add(pa, pb)));
  }
  xor_reduce_store(e0, ei, msg);
}

unsigned grid_for(size_t threads, int block) {
  size_t g = (threads + block - 1) / block;
  return (unsigned)std::max<size_t>(1, std::min<size_t>(g, 148 * 16));
}

}  // namespace

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
  if (l < 1) return fail(LBG_ERR_INVALID, "an empty trace");
  Transcript& tr = t->t;
  // absorb_statement (crates/pcs/src/switch.rs:124-129)
  tr.absorb_bytes((const uint8_t*)"labinius/switch", 15);
  tr.absorb_b128(r_lo, nlo);
  tr.absorb_b128(r_hi, l);
  tr.absorb_b128(claim, 1);

  std::lock_guard<std::mutex> g(pp->mu);
  if (cudaSetDevice(pp->device) != cudaSuccess) return fail(LBG_ERR_CUDA, "cudaSetDevice");
  cudaStream_t st = pp->stream;
  size_t n = pp->n;
  int lh = (int)(l / 2), ll = (int)(l - lh);
  B128d *d_r = nullptr, *d_ehi = nullptr, *d_elo = nullptr, *d_eq = nullptr;
  F162d *d_rp = nullptr, *d_batch = nullptr, *d_psi = nullptr, *d_a = nullptr, *d_p = nullptr, *d_rr = nullptr;
  unsigned long long *d_v = nullptr, *d_msg = nullptr;
  auto release = [&]() {
    void* ptrs[] = {d_r, d_ehi, d_elo, d_eq, d_rp, d_batch, d_psi, d_a, d_p, d_rr, d_v, d_msg};
    for (void* q : ptrs) cudaFree(q);
  };
  if (cudaMalloc((void**)&d_r, l * 16) != cudaSuccess || cudaMalloc((void**)&d_ehi, ((size_t)1 << lh) * 16) != cudaSuccess ||
      cudaMalloc((void**)&d_elo, ((size_t)1 << ll) * 16) != cudaSuccess || cudaMalloc((void**)&d_eq, n * 16) != cudaSuccess ||
      cudaMalloc((void**)&d_rp, 7 * 24) != cudaSuccess || cudaMalloc((void**)&d_batch, 128 * 24) != cudaSuccess ||
      cudaMalloc((void**)&d_psi, 4096 * 24) != cudaSuccess || cudaMalloc((void**)&d_a, n * 24) != cudaSuccess ||
      cudaMalloc((void**)&d_p, n * 24) != cudaSuccess || cudaMalloc((void**)&d_rr, 24) != cudaSuccess ||
      cudaMalloc((void**)&d_v, 128 * 16) != cudaSuccess || cudaMalloc((void**)&d_msg, 48) != cudaSuccess) {
    cudaGetLastError();
    release();
    return fail(LBG_ERR_OOM, "switch: device allocation failed");
  }
  std::vector<uint64_t> r_pp(3 * l);
  uint64_t msg[6];
  cudaError_t e = cudaMemcpyAsync(d_r, r_hi, l * 16, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_sw_eq_tables<<<grid_for(((size_t)1 << lh) + ((size_t)1 << ll), 128), 128, 0, st>>>(d_r, lh, ll, d_ehi, d_elo);
    k_sw_eq<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_ehi, d_elo, ll, n, d_eq);
    e = cudaMemsetAsync(d_v, 0, 128 * 16, st);
  }
  if (e == cudaSuccess) {
    k_sw_partials<<<grid_for(n, 16), 256, 0, st>>>(w->d, d_eq, n, d_v);
    e = cudaMemcpyAsync(partials, d_v, 128 * 16, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    // the batch (crates/pcs/src/switch.rs:149-150)
    tr.absorb_b128(partials, 128);
    uint64_t rp[21];
    tr.sample_f162("labinius/switch-batch", rp, 7);
    e = cudaMemcpyAsync(d_rp, rp, 7 * 24, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) {
    k_sw_batch<<<1, 256, 0, st>>>(d_rp, d_batch, d_psi);
    e = cudaMemsetAsync(d_msg, 0, 48, st);
  }
  if (e == cudaSuccess) {
    size_t smem = 4096 * sizeof(F162d);
    cudaFuncSetAttribute(k_sw_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_sw_init<<<grid_for(n / 2, 256), 256, smem, st>>>(w->d, d_eq, d_psi, n, d_a, d_p, d_msg);
    e = cudaMemcpyAsync(msg, d_msg, 48, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  for (size_t round = 0; round < l && e == cudaSuccess; round++) {
    // the round's message, its challenge (crates/pcs/src/switch.rs:152-159)
    tr.absorb_f162(msg, 2);
    uint64_t r[3];
    tr.sample_f162("labinius/switch-round", r, 1);
    std::memcpy(rounds + 6 * round, msg, 48);
    std::memcpy(r_pp.data() + 3 * round, r, 24);
    size_t half = n >> (round + 1);
    e = cudaMemcpyAsync(d_rr, r, 24, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_msg, 0, 48, st);
    if (e == cudaSuccess) {
      k_sw_round<<<half >= 2 ? grid_for(half / 2, 256) : 1, 256, 0, st>>>(d_a, d_p, half, d_rr, d_msg);
      e = cudaMemcpyAsync(msg, d_msg, 48, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(opened, d_p, 24, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  release();
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("switch: ") + cudaGetErrorString(e));
  // EvaluationPoint::msb_first (crates/pcs/src/scheme/commitment.rs:163-174)
  size_t cl = pp->params.column_log_len, rows = l - cl;
  for (size_t i = 0; i < rows; i++) std::memcpy(p0_out + 3 * i, r_pp.data() + 3 * (l - 1 - i), 24);
  for (size_t i = 0; i < cl; i++) std::memcpy(p1_out + 3 * i, r_pp.data() + 3 * (cl - 1 - i), 24);
  return LBG_OK;
}

}  // extern "C"
