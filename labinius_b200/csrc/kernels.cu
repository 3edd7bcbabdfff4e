// Kernels of the B200 prover path. Launch wrappers at the bottom dispatch on the prime index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "kernels.cuh"
#include "tcgen05.cuh"
#include "launch.h"
#include "transcript_dev.h"

namespace lbg {

// =============================================================================================
// Key expansion: A from xorshift64* (crates/pcs/src/rng.rs:6-19, crates/pcs/src/key.rs:63-80)
// =============================================================================================
// Draw d of limb k's stream is the state after d + 1 steps; thread (b, j) produces the 32 draws
// (b * 648 + j) * 32 + p, p < 32, i.e. row j of ring elements 32 b + p. The start state is reached
// with the GF(2) jump matrices T^(2^t) (64 columns each).
__global__ void k_key_expand(const uint64_t* __restrict__ jumps, uint64_t state0, uint32_t q,
                             int nb, int16_t* __restrict__ A /* [len_ring][648] */) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nb * N648) return;
  int b = gid / N648, j = gid % N648;
  uint64_t d0 = ((uint64_t)b * N648 + j) * 32;
  uint64_t s = state0;
  for (int t = 0; t < 40; t++) {
    if (!((d0 >> t) & 1)) continue;
    const uint64_t* M = jumps + t * 64;
    uint64_t r = 0;
    for (int c = 0; c < 64; c++) r ^= M[c] & (0 - ((s >> c) & 1));
    s = r;
  }
  int16_t half = (int16_t)((q - 1) / 2);
  for (int p = 0; p < 32; p++) {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    uint64_t out = s * 0x2545F4914F6CDD1Dull;
    uint32_t below = (uint32_t)(((out >> 32) * (uint64_t)q) >> 32);
    A[(size_t)(32 * b + p) * N648 + j] = (int16_t)((int16_t)below - half);
  }
}

// The key in component form: for ring element i and leaf j of the 162-point tree,
// Ahat[i][j] = (a_0, a_1, a_2, a_3, theta^v a_1, theta^v a_2, theta^v a_3, 0), the R_162 slot
// values of A_i's four components (the decomposition of crates/pcs/src/ring/mod.rs:217-426
// applied to the key), centered.
template <int PI>
__global__ void k_key_components(const int16_t* __restrict__ A, const DevPrime* __restrict__ D,
                                 int len_ring, int4* __restrict__ Ahat /* [len_ring][162][2] */) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= len_ring * N162) return;
  constexpr int32_t q = Pr<PI>::q;
  int i = gid / N162, s = gid % N162;
  const int16_t* a = A + (size_t)i * N648;
  uint32_t e[4];
  for (int t = 0; t < 4; t++) {
    int32_t x = a[D->key_rows[s][t]];
    e[t] = (uint32_t)(x < 0 ? x + q : x);
  }
  uint32_t y[4];
  for (int k = 0; k < 4; k++) {
    uint64_t acc = 0;
    for (int t = 0; t < 4; t++) acc += (uint64_t)D->key_D[s][k][t] * e[t];
    y[k] = (uint32_t)(acc % q);
  }
  int leaf = D->pow3_to_leaf[s];
  uint32_t th = D->theta_leaf[leaf];
  int4 lo, hi;
  lo.x = center<PI>(y[0]);
  lo.y = center<PI>(y[1]);
  lo.z = center<PI>(y[2]);
  lo.w = center<PI>(y[3]);
  hi.x = center<PI>(mulmod<PI>(th, y[1]));
  hi.y = center<PI>(mulmod<PI>(th, y[2]));
  hi.z = center<PI>(mulmod<PI>(th, y[3]));
  hi.w = 0;
  Ahat[((size_t)i * N162 + leaf) * 2] = lo;
  Ahat[((size_t)i * N162 + leaf) * 2 + 1] = hi;
}

// =============================================================================================
// Commit: Y_j(v) = sum_i Ahat_i(v) (x) What_{j,i}(v) per column j and leaf v
// =============================================================================================
// CTA: 16 columns x a chunk of ring elements, four ring elements per step, 256 threads.
//  phase A: thread t transforms F162 number t of the step's tile (column t / 16, F162 t % 16 of
//           the column's 16) into smem What[ii][v][jj][k] (u16, in [0, 2q));
//  phase B: lane l of warp w serves column l % 16 and the leaves v = 2 (w + 8 u) + l / 16; it
//           accumulates Y_0..Y_3 of those leaves: 16 multiply-adds per (ring element, leaf).
// Both global inputs arrive by asynchronous copies into shared memory: the step's key tile (the
// four ring elements' Ahat, 20.7 KB contiguous) while phase A transforms, the next step's witness
// tile while phase B multiplies.
constexpr int CT = 16;   // columns per CTA
constexpr int RT = 4;    // ring elements per step
constexpr int VPT = 11;  // leaves per thread (8 warps x 2 halves x 11 >= 162)
constexpr int WROW = RT * 12 + 2;          // staged witness words per column, padded to 16 bytes
constexpr int LUT_BYTES = NTT_LUT_U16 * 2;  // the transform's window tables
constexpr int AT_BYTES = RT * N162 * 32;   // the step's key tile

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// all but the newest `N` of this thread's committed groups have landed
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int PI>
__device__ __forceinline__ void commit_phase_a_store(uint16_t* __restrict__ wt, int ii, int k, int jj,
                                                     const uint32_t idx[7], const uint8_t* lut) {
  uint32_t v[27];
#define LBG_BLOCK(TAU)                                                                 \
  ntt_block<PI, TAU>(idx, lut, v);                                                     \
  _Pragma("unroll") for (int x = 0; x < 27; x++) wt[(((ii * N162) + TAU * 27 + x) * CT + jj) * 4 + k] = (uint16_t)v[x];
  LBG_BLOCK(0)
  LBG_BLOCK(1)
  LBG_BLOCK(2)
  LBG_BLOCK(3)
  LBG_BLOCK(4)
  LBG_BLOCK(5)
#undef LBG_BLOCK
}

// Ring elements between two fold-backs of the signed accumulators: one ring element adds at most
// 4 products |Ahat| |What| < (q-1)/2 * 2q per lane, and a fold-back leaves |acc| < 2q.
template <int PI>
struct CommitRed {
  static constexpr int raw = (int)((2147483647ull - 2ull * Pr<PI>::q) /
                                   ((uint64_t)4 * ((Pr<PI>::q - 1) / 2) * (2 * Pr<PI>::q)));
  static constexpr int value = raw < 1 ? 1 : raw;
};

template <int PI, bool KEEP>
__global__ void __launch_bounds__(256, 2)
    k_commit(const uint64_t* __restrict__ W, size_t wdim, const int4* __restrict__ Ahat,
             const DevPrime* __restrict__ D, int cols, int len_ring, int chunk,
             int32_t* __restrict__ partial /* [nchunks][cols][162][4] */,
             uint16_t* __restrict__ keep /* null, or the kept transform [cols][162][wdim] */) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint16_t* lut = (uint16_t*)smem;                        // NTT_LUT_U16 u16
  uint64_t* wtile = (uint64_t*)(smem + LUT_BYTES);        // CT rows of WROW u64 (two pad words)
  uint16_t* wt = (uint16_t*)(smem + LUT_BYTES + CT * WROW * 8);  // RT * 162 * CT * 4 u16
  int4* atile = (int4*)(smem + LUT_BYTES + CT * WROW * 8 + RT * N162 * CT * 4 * 2);  // [RT][162][2]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int j0 = blockIdx.x * CT;
  const int i_begin = blockIdx.y * chunk;
  const int i_end = min(len_ring, i_begin + chunk);
  load_ntt_lut<PI>(lut, D);
  const int jj_b = lane & 15, half = lane >> 4;
  // the witness tile of the step at i0: column jj's 12 * nsteps words in place, zeros past the
  // columns and ring elements of this CTA (plain stores to words no copy targets)
  auto stage_witness = [&](int i0) {
    const int words = 12 * min(RT, i_end - i0);
    for (int x = tid; x < CT * RT * 12; x += 256) {
      int jj = x / (RT * 12), wd = x % (RT * 12);
      int j = j0 + jj;
      if (j < cols && wd < words)
        cp_async8(wtile + jj * WROW + wd, W + ((size_t)j * wdim + (size_t)4 * i0) * 3 + wd);
      else
        wtile[jj * WROW + wd] = 0;
    }
  };
  if (i_begin < i_end) stage_witness(i_begin);
  cp_async_commit();

  int32_t acc[VPT][4];
#pragma unroll
  for (int u = 0; u < VPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0;
  constexpr int RED = CommitRed<PI>::value;
  int since = 0;

  for (int i0 = i_begin; i0 < i_end; i0 += RT) {
    const int nsteps = min(RT, i_end - i0);
    __syncthreads();  // the previous step's phase B is done with the key tile
    {
      const int4* src = Ahat + (size_t)i0 * N162 * 2;
      for (int x = tid; x < nsteps * N162 * 2; x += 256) cp_async16(atile + x, src + x);
    }
    cp_async_commit();
    cp_async_wait<1>();  // this step's witness tile
    __syncthreads();
    {
      // lanes run over columns, so a warp's What stores hit 16 distinct banks
      int jj = tid & 15, g = tid >> 4;  // column, F162 within the column's tile
      const uint64_t* e = wtile + jj * WROW + g * 3;
      uint32_t idx[7];
      f162_windows(e[0], e[1], e[2], idx);
      commit_phase_a_store<PI>(wt, g >> 2, g & 3, jj, idx, (const uint8_t*)lut);
    }
    __syncthreads();
    if (i0 + RT < i_end) stage_witness(i0 + RT);
    cp_async_commit();
    if constexpr (KEEP) {
      // the kept transform (the fold's input) in blocks of 16 positions: keep[j][p / 16][v][p % 16],
      // p = 4 i + k, so this tile of a column is one contiguous 5184-byte block; a lane pair writes
      // one leaf's 16 positions (32 bytes)
      for (int x = tid; x < CT * N162 * 2; x += 256) {
        int h = x & 1, jj = (x >> 1) & (CT - 1), v = x >> 5;
        int j = j0 + jj;
        if (j >= cols || 2 * h >= nsteps) continue;
        uint2 a = *(const uint2*)(wt + ((((2 * h) * N162) + v) * CT + jj) * 4);
        uint16_t* dst = keep + ((size_t)j * (wdim / 16) + i0 / 4) * (N162 * 16) + v * 16 + 8 * h;
        if (2 * h + 1 < nsteps) {
          uint2 b = *(const uint2*)(wt + ((((2 * h + 1) * N162) + v) * CT + jj) * 4);
          *(uint4*)dst = make_uint4(a.x, a.y, b.x, b.y);
        } else {
          *(uint2*)dst = a;
        }
      }
    }
    cp_async_wait<1>();  // this step's key tile
    __syncthreads();
    for (int ii = 0; ii < nsteps; ii++) {
      const int4* ah = atile + ii * N162 * 2;
#pragma unroll
      for (int u = 0; u < VPT; u++) {
        int v = 2 * (warp + 8 * u) + half;
        if (v < N162) {
          uint2 wv = *(const uint2*)(wt + (((ii * N162) + v) * CT + jj_b) * 4);
          int32_t w0 = wv.x & 0xFFFF, w1 = wv.x >> 16, w2 = wv.y & 0xFFFF, w3 = wv.y >> 16;
          int4 lo = ah[2 * v], hi = ah[2 * v + 1];
          acc[u][0] += lo.x * w0 + hi.x * w3 + hi.y * w2 + hi.z * w1;
          acc[u][1] += lo.y * w0 + lo.x * w1 + hi.y * w3 + hi.z * w2;
          acc[u][2] += lo.z * w0 + lo.y * w1 + lo.x * w2 + hi.z * w3;
          acc[u][3] += lo.w * w0 + lo.z * w1 + lo.y * w2 + lo.x * w3;
        }
      }
      if (++since >= RED) {
        since = 0;
#pragma unroll
        for (int u = 0; u < VPT; u++)
#pragma unroll
          for (int c = 0; c < 4; c++) acc[u][c] = red_signed<PI>(acc[u][c]);
      }
    }
  }
  const int j = j0 + jj_b;
  if (j < cols) {
#pragma unroll
    for (int u = 0; u < VPT; u++) {
      int v = 2 * (warp + 8 * u) + half;
      if (v < N162) {
        int4 o;
        o.x = (int)red_signed_full<PI>(acc[u][0]);
        o.y = (int)red_signed_full<PI>(acc[u][1]);
        o.z = (int)red_signed_full<PI>(acc[u][2]);
        o.w = (int)red_signed_full<PI>(acc[u][3]);
        ((int4*)partial)[((size_t)blockIdx.y * cols + j) * N162 + v] = o;
      }
    }
  }
}

// Sum the chunk partials, center, and write the reference layout C[col][row][limb][s].
template <int PI>
__global__ void k_commit_finish(const int32_t* __restrict__ partial, int nchunks, int cols,
                                const DevPrime* __restrict__ D, int limb, int limbs,
                                int16_t* __restrict__ C) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= cols * N162) return;
  int j = gid / N162, s = gid % N162;
  int v = D->pow3_to_leaf[s];
  uint64_t acc[4] = {0, 0, 0, 0};
  for (int c = 0; c < nchunks; c++) {
    int4 p = ((const int4*)partial)[((size_t)c * cols + j) * N162 + v];
    acc[0] += (uint32_t)p.x;
    acc[1] += (uint32_t)p.y;
    acc[2] += (uint32_t)p.z;
    acc[3] += (uint32_t)p.w;
  }
  for (int row = 0; row < 4; row++)
    C[(((size_t)j * 4 + row) * limbs + limb) * N162 + s] = center<PI>((uint32_t)(acc[row] % Pr<PI>::q));
}

// =============================================================================================
// Commit on the tensor cores: the 162-point binary transform as a kind::i8 multiply
// =============================================================================================
// The transform of an F162 is linear in its bits: What(v) = sum_m bit_m T[m][v] with
// T[m][v] = theta^{E[v] m} mod q. A step's 128 F162 (32 columns x the 4 positions of one ring
// element) are the rows of an M = 128, N = 176, K = 384 multiply whose A row holds bit m at K-byte
// m and 128 bit_m at K-byte 192 + m, and whose B (shared memory for the whole kernel) holds T split
// as lo + 128 hi (tc_transform_operand): the s32 accumulator is the exact transform, < 2^22.
//
// Row r of a step is column jj = 8 (r / 32) + r % 8 of the tile and position k = (r / 8) % 4 of
// the ring element, so that the 16x256b tensor-memory load hands each thread the four positions
// of one column at two leaves: the module product's operands arrive in registers, with no pass
// through shared memory.
//
// The kernel is persistent: CTA b takes the work items b, b + gridDim.x, ... (an item is a tile of
// 32 columns x a chunk of ring elements, partial[chunk][column] its output), and the steps of all
// its items, one ring element each, form one pipeline of two warp roles (slot g % 2 of each
// mbarrier pair serves step g; every wait is bounded):
//   producer (warp 12, one lane) copies step g's key tile into buffer g % 2 once step g - 2's is
//            released (kempty; completion counted on kfull) and writes step g + 1's cursor, then,
//            at named barrier 1, issues step g's 12 K-steps into tensor-memory accumulator g % 2
//            and commits them to mma;
//   compute (warps 0-11) per step g: expand step g's witness words (wtile g % 2, landed on wfull)
//            into A buffer g % 2 and meet the producer (named barrier 1); start the 8-byte copies
//            of step g + 1's words (cp.async, one word a thread, counted on wfull); read step
//            g - 1's accumulator, warp w the lanes of quadrant w % 4 (columns 8 (w % 4) .. + 7)
//            and leaves [56 (w / 4), + 56): thread t column 8 (w % 4) + t / 4 at 14 leaves,
//            reduced to [0, 2q), times the key, 16 multiply-adds per (leaf, column) into 56
//            registers; release the key tile. After an item's last step each thread writes its
//            column's sums and clears its registers.
// A buffer g % 2 is free for step g once step g - 2's multiply is done, which every compute warp
// saw before reading that step's accumulator; accumulator g % 2 is free once every compute warp
// has passed named barrier 1 of step g. Rows of columns past the last are zero.
// CW compute warps. 12: three leaf ranges of 56 leaves (14 a thread) and a producer warp (13 warps,
// 128 registers). 16: four ranges of 48, 40, 40, 40 leaves (at most 12 a thread) and no producer
// warp: thread 0 issues the key copies and the multiplies after each step's barrier (16 warps, 128
// registers: a 17th warp would cost the registers of four, which allocate in groups of four warps).
template <int CW>
struct TccShape {
  static constexpr int CTHREADS = CW * 32;
  static constexpr bool PRODUCER = CW == 12;  // a warp of its own issues the copies and multiplies
  static constexpr int THREADS = CTHREADS + (PRODUCER ? 32 : 0);
  static constexpr int LPT = CW == 12 ? 14 : 12;  // leaves per compute thread (at most)
  static_assert(CW == 12 || CW == 16, "twelve or sixteen compute warps");
  // first leaf of leaf range `part`, and the number of eight-leaf chunks in it
  __device__ static int base(int part) { return CW == 12 ? 56 * part : (part == 0 ? 0 : 8 + 40 * part); }
  __device__ static int chunks(int part) { return CW == 12 ? 7 : (part == 0 ? 6 : 5); }
};
constexpr int TCC_CTHREADS = 384;                      // the default: compute warps 0-11
constexpr int TCC_THREADS = TCC_CTHREADS + 32;         // and the producer warp (13 warps: 128 registers)
constexpr int TCC_CT = 32;                             // columns per item
constexpr int TCC_RT = 1;                              // ring elements per step
constexpr int TCC_LPT = 14;                            // leaves per compute thread
constexpr int TCC_A_BYTES = 128 * TC_KBYTES;           // 128 rows x 384 bytes
constexpr int TCC_AT_BYTES = N162 * 32;                // a step's key tile
constexpr int TCC_WT_BYTES = 128 * 24;                 // a step's witness words (three per row)
constexpr int TCC_OFF_A = TC_B_BYTES;                  // two A buffers
constexpr int TCC_OFF_AT = TCC_OFF_A + 2 * TCC_A_BYTES;        // two key tiles
constexpr int TCC_OFF_WT = TCC_OFF_AT + 2 * TCC_AT_BYTES;      // two witness tiles
constexpr int TCC_OFF_BAR = TCC_OFF_WT + 2 * TCC_WT_BYTES;
constexpr int TCC_OFF_CUR = TCC_OFF_BAR + 128;         // four step cursors
constexpr int TCC_SMEM = TCC_OFF_CUR + 4 * 32 + 1024;  // + barriers, tensor-memory slot, flag, cursors, alignment
constexpr uint32_t TCC_TMEM_COLS = 512;                // two accumulators at columns 0 and 256
constexpr long long TC_WAIT_BUDGET = 2000000000ll;     // cycles (about a second) before a timeout

static_assert(TCC_OFF_A % TC_ATOM == 0 && TCC_A_BYTES % TC_ATOM == 0 && TCC_OFF_AT % 16 == 0 &&
                  TCC_OFF_WT % 16 == 0 && TCC_OFF_BAR % 8 == 0 && TCC_OFF_CUR % 16 == 0,
              "alignment");
static_assert(TCC_SMEM <= 232448, "shared memory per CTA");
static_assert(TCC_CTHREADS == 3 * 128 && 3 * 56 >= N162 && 48 + 3 * 40 >= N162,
              "four quadrants x three or four leaf ranges; the first 384 compute threads copy the rows' words");

// A device-wide flag set by a tensor-core kernel whose bounded wait ran out (never in practice:
// what it waits for takes microseconds). The host reads and clears it.
__device__ int g_tc_timeout = 0;

// The thread's part of the A operand: row tid % 128, its NC chunks c_k = tid / 128 + (threads / 128) k
// of 16 bits (bits 16 c_k ..) expanded to bytes at their swizzled offsets in the bit plane and in the
// times-128 plane, from the row's F162 words (zero when !valid; at most 34 bits in the third word).
template <int NC>
__device__ __forceinline__ void tc_build_row_inline(uint8_t* sA, int tid, int threads, const uint64_t* e,
                                                    bool valid = true) {
  const int r = tid & 127, step = threads >> 7;
  const uint64_t w0 = valid ? e[0] : 0, w1 = valid ? e[1] : 0, w2 = valid ? e[2] & ((1ull << 34) - 1) : 0;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const int c = (tid >> 7) + step * k;
    const uint64_t word = (c >> 2) == 0 ? w0 : (c >> 2) == 1 ? w1 : w2;
    const uint32_t u = (uint32_t)(word >> (16 * (c & 3))) & 0xFFFFu;
    uint4 b;
    b.x = ((u & 15u) * 0x00204081u) & 0x01010101u;
    b.y = (((u >> 4) & 15u) * 0x00204081u) & 0x01010101u;
    b.z = (((u >> 8) & 15u) * 0x00204081u) & 0x01010101u;
    b.w = (((u >> 12) & 15u) * 0x00204081u) & 0x01010101u;
    *(uint4*)(sA + tc_swizzled_offset(r, 16 * c, 128)) = b;
    *(uint4*)(sA + tc_swizzled_offset(r, 16 * c + 192, 128)) = make_uint4(b.x << 7, b.y << 7, b.z << 7, b.w << 7);
  }
}

// Issue the 12 K-steps of one 128 x 176 x 384 transform multiply and commit them to `bar`.
__device__ __forceinline__ void tc_transform_mma(uint32_t d_tmem, uint32_t sA_u, uint32_t sB_u, uint64_t* bar) {
  constexpr uint32_t IDESC = tc::idesc_u8(128, TC_LEAVES);
#pragma unroll
  for (int kk = 0; kk < TC_KBYTES / 32; kk++) {
    // K-step kk: atom kk / 4, 32-byte step kk % 4 inside it
    const uint32_t a = sA_u + (kk >> 2) * (128 * 128) + (kk & 3) * 32;
    const uint32_t b = sB_u + (kk >> 2) * (TC_LEAVES * 128) + (kk & 3) * 32;
    tc::mma_i8(d_tmem, tc::smem_desc_sw128(a, TC_ATOM), tc::smem_desc_sw128(b, TC_ATOM), IDESC, kk > 0);
  }
  tc::commit_to(bar);
}

// A bounded mbarrier wait that records a timeout in the CTA's flag and is skipped once it is set.
__device__ __forceinline__ void tc_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  if (*abort) return;
  if (!tc::mbar_wait(bar, parity, TC_WAIT_BUDGET)) *abort = 1;
}

// The CTA's work items in order, each a run of steps: item `it` is column tile it % col_tiles
// and ring-element chunk it / col_tiles.
struct TcItems {
  int first, stride, total, col_tiles, chunk, len_ring;
  __device__ int steps(int it) const {
    const int i0 = (it / col_tiles) * chunk;
    const int i1 = min(len_ring, i0 + chunk);
    return i1 > i0 ? (i1 - i0 + TCC_RT - 1) / TCC_RT : 0;
  }
};

// A position in that sequence, with the item's bounds computed once when the item starts (one
// division per item rather than several per step): step st of item it covers ring elements
// [i, min(i + TCC_RT, iend)) of columns [j0, j0 + TCC_CT).
struct TcCursor {
  int it, st, steps, j0, i, iend, ci;
  __device__ void load(const TcItems& I, int item) {
    it = item;
    st = 0;
    steps = 0;
    while (it < I.total) {
      ci = it / I.col_tiles;
      const int i0 = ci * I.chunk, i1 = min(I.len_ring, i0 + I.chunk);
      if (i1 > i0) {
        j0 = (it - ci * I.col_tiles) * TCC_CT;
        i = i0;
        iend = i1;
        steps = (i1 - i0 + TCC_RT - 1) / TCC_RT;
        return;
      }
      it += I.stride;
    }
  }
  __device__ void advance(const TcItems& I) {
    if (++st < steps) {
      i += TCC_RT;
      return;
    }
    load(I, it + I.stride);
  }
  __device__ int n() const { return min(TCC_RT, iend - i); }  // ring elements in this step
  __device__ bool last() const { return st + 1 == steps; }
  __device__ bool valid(const TcItems& I) const { return it < I.total; }
};

template <int PI, int CW>
__global__ void __launch_bounds__(TccShape<CW>::THREADS, 1)
    k_commit_tc(const uint64_t* __restrict__ W, size_t wdim, const int4* __restrict__ Ahat,
                const uint8_t* __restrict__ tcb, int cols, int len_ring, int chunk, int nchunks,
                int32_t* __restrict__ partial /* [nchunks][cols][162][4] */) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);  // swizzle atoms
  uint8_t* sB = smem;
  uint8_t* sA = smem + TCC_OFF_A;                       // [2] A operands
  int4* atile = (int4*)(smem + TCC_OFF_AT);             // [2][162][2] key tiles
  uint64_t* wtile = (uint64_t*)(smem + TCC_OFF_WT);     // [2][128][3] witness words of the rows
  uint64_t* wfull = (uint64_t*)(smem + TCC_OFF_BAR);    // [2] words landed (cp.async, every compute thread)
  uint64_t* mma = wfull + 2;                            // [2] multiply done (tcgen05.commit)
  uint64_t* kfull = wfull + 4;                          // [2] key tile landed (bulk copy)
  uint64_t* kempty = wfull + 6;                         // [2] key tile read (compute warps)
  uint64_t* bfull = wfull + 8;                          // the transform operand landed
  uint32_t* tslot = (uint32_t*)(wfull + 9);
  volatile int* abort = (volatile int*)(wfull + 10);
  // step g's cursor in slot g % 4: the producer writes step g + 1's before named barrier 1 of step
  // g; the compute warps read step g + 1's (word copies) and step g - 1's (item end) after it
  TcCursor* curs = (TcCursor*)(smem + TCC_OFF_CUR);
  using Sh = TccShape<CW>;
  constexpr int CTHREADS = Sh::CTHREADS, THREADS = Sh::THREADS, LPT = Sh::LPT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int col_tiles = (cols + TCC_CT - 1) / TCC_CT;
  const TcItems items{(int)blockIdx.x, (int)gridDim.x, col_tiles * nchunks, col_tiles, chunk, len_ring};
  int S = 0;  // the CTA's steps
  for (int it = items.first; it < items.total; it += items.stride) S += items.steps(it);

  if (tid == 0) {
    for (int b = 0; b < 2; b++) {
      tc::mbar_init(&wfull[b], CTHREADS);
      tc::mbar_init(&mma[b], 1);
      tc::mbar_init(&kfull[b], 1);
      tc::mbar_init(&kempty[b], CTHREADS / 32);
    }
    tc::mbar_init(bfull, 1);
    *abort = 0;
    curs[0].load(items, items.first);
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, TCC_TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (Sh::PRODUCER && warp == CTHREADS / 32) {
    // ---------------- producer (one lane) ----------------
    const uint32_t sA_u = tc::smem_u32(sA), sB_u = tc::smem_u32(sB);
    TcCursor cur = curs[0];
    if (lane == 0 && S > 0) {
      tc::mbar_arrive_expect_tx(bfull, TC_B_BYTES);
      for (int x = 0; x < 4; x++)
        tc::bulk_g2s(sB + x * (TC_B_BYTES / 4), tcb + x * (TC_B_BYTES / 4), TC_B_BYTES / 4, bfull);
    }
    for (int g = 0; g < S; g++) {
      const int b = g & 1;
      TcCursor nxt = cur;
      nxt.advance(items);
      if (lane == 0) {
        // step g's key tile into buffer b, released by step g - 2's module product
        if (g >= 2) tc_wait(&kempty[b], ((g - 2) >> 1) & 1, abort);
        tc::mbar_arrive_expect_tx(&kfull[b], TCC_AT_BYTES);
        tc::bulk_g2s(atile + b * (N162 * 2), Ahat + (size_t)cur.i * N162 * 2, TCC_AT_BYTES, &kfull[b]);
        curs[(g + 1) & 3] = nxt;
      }
      __syncwarp();
      tc::named_sync(1, THREADS);  // step g's A operand is built
      if (lane == 0) {
        tc::fence_after_sync();
        if (g == 0) tc_wait(bfull, 0, abort);
        if (!*abort)
          tc_transform_mma(tmem + (uint32_t)b * 256u, sA_u + (uint32_t)b * TCC_A_BYTES, sB_u, &mma[b]);
        else
          tc::mbar_arrive(&mma[b]);
      }
      __syncwarp();
      cur = nxt;
    }
    if (lane == 0) {
      // the last key copies and multiplies have landed before the CTA winds down (bounded waits
      // that ignore the abort flag: nothing of this CTA may still be in flight at its exit)
      for (int g = S - 2 < 0 ? 0 : S - 2; g < S; g++) {
        tc::mbar_wait(&kfull[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
        tc::mbar_wait(&mma[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
      }
    }
  } else if (S > 0) {
    // ---------------- compute ----------------
    const int quad = warp & 3, part = warp >> 2;
    const int jq = 8 * quad + (lane >> 2);               // the thread's column in the tile
    const int v0 = Sh::base(part) + 2 * (lane & 3);      // its leaves: v0 + 8 c + l, c < chunks, l < 2
    const int nlv = 2 * Sh::chunks(part);                // its leaf slots
    // the word this thread copies for every step: word wx of row wr (column wj, position wk)
    const int wr = tid / 3, wx = tid - 3 * (tid / 3);
    const int wj = 8 * (wr >> 5) + (wr & 7), wk = (wr >> 3) & 3;
    auto copy_words = [&](const TcCursor& c, int b) {
      if (tid < 384 && c.j0 + wj < cols)
        tc::cp_async8(wtile + (b * 128 + wr) * 3 + wx, W + ((size_t)(c.j0 + wj) * wdim + (size_t)4 * c.i + wk) * 3 + wx);
      tc::cp_async_arrive(&wfull[b]);
    };
    const int r = tid & 127;
    const int rj = 8 * (r >> 5) + (r & 7);  // the built row's column
    int32_t acc[LPT][4];
#pragma unroll
    for (int u = 0; u < LPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0;
    constexpr int RED = CommitRed<PI>::value;
    int since = 0;
    // one leaf's module product: positions w0..w3 of the column's ring element, key (lo, hi)
    auto product = [&](int32_t(&a)[4], uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, const int4* ah) {
      const int32_t w0 = (int32_t)red_half<PI>(x0), w1 = (int32_t)red_half<PI>(x1);
      const int32_t w2 = (int32_t)red_half<PI>(x2), w3 = (int32_t)red_half<PI>(x3);
      const int4 lo = ah[0], hi = ah[1];
      a[0] += lo.x * w0 + hi.x * w3 + hi.y * w2 + hi.z * w1;
      a[1] += lo.y * w0 + lo.x * w1 + hi.y * w3 + hi.z * w2;
      a[2] += lo.z * w0 + lo.y * w1 + lo.x * w2 + hi.z * w3;
      a[3] += lo.w * w0 + lo.z * w1 + lo.y * w2 + lo.x * w3;
    };
    // without a producer warp, thread 0 keeps the cursor sequence and issues, after step g's
    // barrier, step g's key copy into buffer g % 2 (its last reader, step g - 2's module product,
    // finished before that barrier) and step g's multiply
    TcCursor pcur;
    if (!Sh::PRODUCER && tid == 0) {
      pcur = curs[0];
      tc::mbar_arrive_expect_tx(bfull, TC_B_BYTES);
      for (int x = 0; x < 4; x++)
        tc::bulk_g2s(sB + x * (TC_B_BYTES / 4), tcb + x * (TC_B_BYTES / 4), TC_B_BYTES / 4, bfull);
    }
    copy_words(curs[0], 0);
    for (int g = 0; g <= S; g++) {
      if (g < S) {
        const int b = g & 1;
        if (!Sh::PRODUCER && tid == 0) {
          // step g + 1's cursor, read after this step's barrier (its slot's last reader was step
          // g - 3's module product, before the previous barrier)
          pcur.advance(items);
          curs[(g + 1) & 3] = pcur;
        }
        tc_wait(&wfull[b], (g >> 1) & 1, abort);  // step g's words
        tc_build_row_inline<12 * 128 / CTHREADS>(sA + b * TCC_A_BYTES, tid, CTHREADS,
                                                   wtile + (b * 128 + r) * 3, curs[g & 3].j0 + rj < cols);
        tc::fence_async_shared();
        tc::fence_before_sync();
        tc::named_sync(1, THREADS);  // meets the producer: lockstep, even when a wait timed out
        if (!Sh::PRODUCER && tid == 0) {
          tc::fence_after_sync();
          if (g == 0) tc_wait(bfull, 0, abort);
          if (!*abort) {
            tc::mbar_arrive_expect_tx(&kfull[b], TCC_AT_BYTES);
            tc::bulk_g2s(atile + b * (N162 * 2), Ahat + (size_t)curs[g & 3].i * N162 * 2, TCC_AT_BYTES, &kfull[b]);
            tc_transform_mma(tmem + (uint32_t)b * 256u, tc::smem_u32(sA) + (uint32_t)b * TCC_A_BYTES,
                             tc::smem_u32(sB), &mma[b]);
          } else {
            tc::mbar_arrive(&kfull[b]);
            tc::mbar_arrive(&mma[b]);
          }
        }
        if (g + 1 < S) copy_words(curs[(g + 1) & 3], (g + 1) & 1);
      }
      if (g >= 1) {
        const int b = (g - 1) & 1;
        const uint32_t par = ((g - 1) >> 1) & 1;
        const TcCursor& prev = curs[(g - 1) & 3];
        tc_wait(&mma[b], par, abort);    // step g - 1's accumulator
        tc_wait(&kfull[b], par, abort);  // step g - 1's key tile
        tc::fence_after_sync();
        // lanes 32 quad .. + 15 hold positions 0-1 of the quadrant's 8 columns, + 16 .. 31 positions 2-3
        const uint32_t ta = tmem + (uint32_t)b * 256u + ((uint32_t)(32 * quad) << 16) + Sh::base(part);
        const uint32_t tb = ta + (16u << 16);
        const int4* kt = atile + b * (N162 * 2) + 2 * v0;  // the key at the thread's first leaf
        // chunk pairs (16 leaves, all below 162) by x2 loads: x[0..7] positions 0-1, x[8..15] positions 2-3
        auto pair = [&](int cp) {
          uint32_t x[16];
          tc::tmem_ld16x256_x2_nowait(ta + 16 * cp, x);
          tc::tmem_ld16x256_x2_nowait(tb + 16 * cp, x + 8);
          tc::tmem_wait_ld(x);
#pragma unroll
          for (int h = 0; h < 2; h++)
#pragma unroll
            for (int l = 0; l < 2; l++)
              product(acc[2 * (2 * cp + h) + l], x[4 * h + l], x[4 * h + 2 + l], x[8 + 4 * h + l],
                      x[8 + 4 * h + 2 + l], kt + 2 * (8 * (2 * cp + h) + l));
        };
        // a last single chunk by x1 loads; the last leaf range's pads (leaves 162 - 167) use leaf
        // 161's key, unused
        auto single = [&](int c) {
          uint32_t x[8];
          tc::tmem_ld16x256_x1_nowait(ta + 8 * c, x);
          tc::tmem_ld16x256_x1_nowait(tb + 8 * c, x + 4);
          tc::tmem_wait_ld(x);
#pragma unroll
          for (int l = 0; l < 2; l++)
            product(acc[2 * c + l], x[l], x[2 + l], x[4 + l], x[6 + l], kt + 2 * (min(v0 + 8 * c + l, N162 - 1) - v0));
        };
        if (CW == 12) {
#pragma unroll
          for (int cp = 0; cp < 3; cp++) pair(cp);
          single(6);
        } else {
          pair(0);
          pair(1);
          if (part == 0)
            pair(2);
          else
            single(4);
        }
        tc::fence_before_sync();
        tc::fence_async_shared();  // this warp's reads of the key tile precede the next bulk copy into it
        if (Sh::PRODUCER) {
          __syncwarp();
          if (lane == 0) tc::mbar_arrive(&kempty[b]);
        }
        if (++since >= RED) {
          since = 0;
#pragma unroll
          for (int u = 0; u < LPT; u++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[u][c] = red_signed<PI>(acc[u][c]);
        }
        if (prev.last()) {
          // the item's last step: the column's sums out, the registers cleared
          const int j = prev.j0 + jq;
          if (j < cols) {
            int4* dst = (int4*)partial + ((size_t)prev.ci * cols + j) * N162;
#pragma unroll
            for (int u = 0; u < LPT; u++) {
              const int v = v0 + 8 * (u >> 1) + (u & 1);
              if (u < nlv && v < N162) {
                int4 o;
                o.x = (int)red_signed_full<PI>(acc[u][0]);
                o.y = (int)red_signed_full<PI>(acc[u][1]);
                o.z = (int)red_signed_full<PI>(acc[u][2]);
                o.w = (int)red_signed_full<PI>(acc[u][3]);
                dst[v] = o;
              }
            }
          }
#pragma unroll
          for (int u = 0; u < LPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0;
          since = 0;
        }
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy of this thread outlives the CTA
    if (!Sh::PRODUCER && tid == 0) {
      // as the producer warp does: the last key copies and multiplies have landed (bounded waits
      // that ignore the abort flag)
      for (int g = S - 2 < 0 ? 0 : S - 2; g < S; g++) {
        tc::mbar_wait(&kfull[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
        tc::mbar_wait(&mma[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCC_TMEM_COLS);
  if (tid == 0 && *abort) atomicExch(&g_tc_timeout, 1);
}

// =============================================================================================
// Fold: v_p = sum_j c_j(-Y) w_{j,p}(Y) in Z_q[Y]/(Y^162 - Y^81 + 1), one F162 position p at a time
// =============================================================================================
// Challenge slot values: chat[j][leaf] = c_j(-theta^{E[leaf]}) (crates/pcs/src/fold.rs:287-335).
template <int PI>
__global__ void k_challenge_slots(const lbg_challenge_d* __restrict__ ch, int r,
                                  const DevPrime* __restrict__ D, uint32_t* __restrict__ chat) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= r * N162) return;
  int j = gid / N162, leaf = gid % N162;
  constexpr uint32_t q = Pr<PI>::q;
  const lbg_challenge_d& c = ch[j];
  uint32_t acc = 0;
  uint32_t w = c.weight > 32 ? 32 : c.weight;
  for (uint32_t t = 0; t < w; t++) {
    uint32_t p = c.positions[t];
    if (p >= N162) continue;
    uint32_t x = D->chal[p * N162 + leaf];
    acc += ((c.signs >> t) & 1) ? (q - x) : x;
  }
  chat[(size_t)j * N162 + leaf] = acc % q;
}

constexpr int FP = 32;  // positions per CTA
constexpr int FJ = 8;   // columns per step
constexpr int VPW = 21; // leaves per warp (8 warps, 162 leaves)

// The inverse transforms of a CTA's FP positions' sums vh[FP][162] (shared memory), four positions
// at a time by 54 threads each, centred into the folded witness (position p is coefficient
// 4m + p % 4 of ring element p / 4). Every thread of the CTA calls it.
template <int PI>
__device__ __forceinline__ void fold_positions_out(uint32_t* vh, size_t p0, size_t wdim, const DevPrime* D,
                                                   int16_t* v_out) {
  const int tid = threadIdx.x, g = tid / 54, jj = tid - 54 * g;
  for (int r = 0; r < FP / 4; r++) intt162_group<PI>(vh + (g < 4 ? 4 * r + g : 0) * N162, g < 4 ? jj : 54, *D);
  for (int e = tid; e < FP * N162; e += blockDim.x) {
    const int pl = e / N162, m = e - pl * N162;
    const size_t p = p0 + pl;
    if (p < wdim) v_out[(p / 4) * N648 + 4 * m + (p % 4)] = center<PI>(vh[pl * N162 + m]);
  }
}

// Columns between two fold-backs of the unsigned accumulators: a column adds one product
// chat * What < q * 2q per lane, and a fold-back leaves acc < 2q.
template <int PI>
struct FoldRed {
  static constexpr int raw = (int)((4294967295ull - 2ull * Pr<PI>::q) / (2ull * Pr<PI>::q * Pr<PI>::q));
  static constexpr int value = raw < 1 ? 1 : raw;
};

template <int PI>
__device__ __forceinline__ void fold_phase_a_store(uint16_t* __restrict__ wt, int jj, int lane,
                                                   const uint32_t idx[7], const uint8_t* lut) {
  uint32_t v[27];
#define LBG_BLOCK(TAU)                  \
  ntt_block<PI, TAU>(idx, lut, v);      \
  _Pragma("unroll") for (int x = 0; x < 27; x++) wt[((jj * N162) + TAU * 27 + x) * FP + lane] = (uint16_t)v[x];
  LBG_BLOCK(0)
  LBG_BLOCK(1)
  LBG_BLOCK(2)
  LBG_BLOCK(3)
  LBG_BLOCK(4)
  LBG_BLOCK(5)
#undef LBG_BLOCK
}

// One CTA: 32 F162 positions x the columns [c_begin, c_end), eight columns per step.
//  phase A: warp w transforms the F162 of column c + w at its lane's position into smem;
//  phase B: warp w owns the leaves v = w + 8 u; lane = position; one multiply-add per (column, leaf).
// The next step's witness words are loaded into registers while this step runs, and the step's
// challenge slot values arrive in shared memory by cp.async while phase A transforms.
// Split mode: the CTA's sums, reduced to [0, q), are added into vhat[p][v] (u32, zeroed by the
// caller; with at most 2^16 column splits the total stays below 2^32) and k_fold_finish inverts.
// Direct mode (one split): the CTA inverts its 32 positions itself and writes v, no vhat.
template <int PI, bool DIRECT>
__global__ void __launch_bounds__(256, 2)
    k_fold(const uint64_t* __restrict__ W, size_t wdim, int cols, int cols_per_split,
           const uint32_t* __restrict__ chat, const DevPrime* __restrict__ D, uint32_t* __restrict__ vhat,
           int16_t* __restrict__ v_out, const int* __restrict__ split_inst) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint16_t* lut = (uint16_t*)smem;
  uint16_t* wt = (uint16_t*)(smem + LUT_BYTES);  // FJ * 162 * FP u16
  uint32_t* ctile = (uint32_t*)(smem + LUT_BYTES + FJ * N162 * FP * 2);  // [FJ][162]: the step's chat
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t p0 = (size_t)blockIdx.x * FP;
  const int c_begin = blockIdx.y * cols_per_split;
  const int c_end = min(cols, c_begin + cols_per_split);
  load_ntt_lut<PI>(lut, D);
  uint32_t acc[VPW];
#pragma unroll
  for (int u = 0; u < VPW; u++) acc[u] = 0;
  constexpr int RED = FoldRed<PI>::value;
  int since = 0;
  // warp w's F162 of the step at j0: column j0 + w at the lane's position (zero past the range)
  auto load_w = [&](int j0, uint64_t& e0, uint64_t& e1, uint64_t& e2) {
    const int j = j0 + warp;
    const size_t p = p0 + lane;
    e0 = e1 = e2 = 0;
    if (j < c_end && p < wdim) {
      const uint64_t* e = W + ((size_t)j * wdim + p) * 3;
      e0 = e[0];
      e1 = e[1];
      e2 = e[2];
    }
  };
  uint64_t e0, e1, e2;
  load_w(c_begin, e0, e1, e2);
  for (int j0 = c_begin; j0 < c_end; j0 += FJ) {
    const int nj = min(FJ, c_end - j0);
    __syncthreads();  // the previous step's phase B is done with wt and ctile
    for (int x = tid; x < nj * N162; x += 256) cp_async4(ctile + x, chat + (size_t)j0 * N162 + x);
    cp_async_commit();
    {
      uint32_t idx[7];
      f162_windows(e0, e1, e2, idx);
      load_w(j0 + FJ, e0, e1, e2);
      fold_phase_a_store<PI>(wt, warp, lane, idx, (const uint8_t*)lut);
    }
    cp_async_wait<0>();
    __syncthreads();
    for (int jj = 0; jj < nj; jj++) {
      const uint32_t* ch = ctile + jj * N162;
#pragma unroll
      for (int u = 0; u < VPW; u++) {
        int v = warp + 8 * u;
        if (v < N162) acc[u] += ch[v] * (uint32_t)wt[((jj * N162) + v) * FP + lane];
      }
      if (++since >= RED) {
        since = 0;
#pragma unroll
        for (int u = 0; u < VPW; u++) acc[u] = red_half<PI>(acc[u]);
      }
    }
  }
  if (!DIRECT) {
    const size_t p = p0 + lane;
    // many instances: split s belongs to instance split_inst[s], whose sums start at inst * wdim
    if (split_inst) vhat += (size_t)split_inst[blockIdx.y] * wdim * N162;
    if (p < wdim) {
#pragma unroll
      for (int u = 0; u < VPW; u++) {
        int v = warp + 8 * u;
        if (v < N162) atomicAdd(vhat + p * N162 + v, red_full<PI>(acc[u]));
      }
    }
    return;
  }
  __syncthreads();
  uint32_t* vh = (uint32_t*)wt;  // [FP][162] u32, 20.7 KB of the 83 KB stage
#pragma unroll
  for (int u = 0; u < VPW; u++) {
    int v = warp + 8 * u;
    if (v < N162) vh[lane * N162 + v] = red_full<PI>(acc[u]);
  }
  __syncthreads();
  fold_positions_out<PI>(vh, p0, wdim, D, v_out);
}

// The fold from the kept transform (keep[j][p / 16][v][p % 16], written by the commit at the base
// limb): the same sums as k_fold without transforming each F162 again. Per step the CTA streams
// the two 5184-byte blocks of its 32 positions for FJ columns into shared memory (16-byte loads);
// then warp w owns the leaves v = w + 8 u and lane = position, as in k_fold.
template <int PI, bool DIRECT>
__global__ void __launch_bounds__(256, 2)
    k_fold_kept(const uint16_t* __restrict__ keep, size_t wdim, int cols, int cols_per_split,
                const uint32_t* __restrict__ chat, const DevPrime* __restrict__ D, uint32_t* __restrict__ vhat,
                int16_t* __restrict__ v_out, const int* __restrict__ split_inst) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint16_t* st = (uint16_t*)smem;  // [FJ][2 blocks][162][16] u16
  constexpr int BLK = N162 * 16;   // u16 per block
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t p0 = (size_t)blockIdx.x * FP;
  const size_t p = p0 + lane;
  const bool inside = p < wdim;
  const int c_begin = blockIdx.y * cols_per_split;
  const int c_end = min(cols, c_begin + cols_per_split);
  const size_t nblk = wdim / 16, b0 = p0 / 16;
  const int blocks = (int)min((size_t)2, nblk - b0);
  uint32_t acc[VPW];
#pragma unroll
  for (int u = 0; u < VPW; u++) acc[u] = 0;
  constexpr int RED = FoldRed<PI>::value;
  int since = 0;
  for (int j0 = c_begin; j0 < c_end; j0 += FJ) {
    const int nj = min(FJ, c_end - j0);
    __syncthreads();
    const int per_col = blocks * BLK / 8;  // uint4 per column
    for (int x = tid; x < nj * per_col; x += 256) {
      int jj = x / per_col, o = x - jj * per_col;
      const uint4* src = (const uint4*)(keep + ((size_t)(j0 + jj) * nblk + b0) * BLK);
      ((uint4*)(st + (size_t)jj * 2 * BLK))[o] = __ldg(src + o);
    }
    __syncthreads();
    const int off = (lane >> 4) * BLK + (lane & 15);
    for (int jj = 0; jj < nj; jj++) {
      const uint32_t* ch = chat + (size_t)(j0 + jj) * N162;
      const uint16_t* sj = st + (size_t)jj * 2 * BLK + off;
#pragma unroll
      for (int u = 0; u < VPW; u++) {
        int v = warp + 8 * u;
        if (v < N162) acc[u] += __ldg(ch + v) * (uint32_t)sj[v * 16];
      }
      if (++since >= RED) {
        since = 0;
#pragma unroll
        for (int u = 0; u < VPW; u++) acc[u] = red_half<PI>(acc[u]);
      }
    }
  }
  if constexpr (!DIRECT) {
    if (split_inst) vhat += (size_t)split_inst[blockIdx.y] * wdim * N162;
    if (inside) {
#pragma unroll
      for (int u = 0; u < VPW; u++) {
        int v = warp + 8 * u;
        if (v < N162) atomicAdd(vhat + p * N162 + v, red_full<PI>(acc[u]));
      }
    }
  } else {
    __syncthreads();
    uint32_t* vh = (uint32_t*)smem;  // [FP][162] u32, 20.7 KB of the stage
#pragma unroll
    for (int u = 0; u < VPW; u++) {
      int v = warp + 8 * u;
      if (v < N162) vh[lane * N162 + v] = red_full<PI>(acc[u]);
    }
    __syncthreads();
    fold_positions_out<PI>(vh, p0, wdim, D, v_out);
  }
}

// =============================================================================================
// Fold on the tensor cores: the base limb's transforms by the same kind::i8 multiply
// =============================================================================================
// A work item is 128 consecutive positions p of the witness x a split of columns [c0, c1); the
// kernel is persistent (CTA b takes items b, b + gridDim.x, ...) and all its items' steps, one
// column each, form one pipeline of two warp roles:
//   producer (warp 12)  loads step g + 1's 128 F162 (3 KB, one bulk copy counted on mbarrier
//            full[(g + 1) % 2]) and issues step g's multiply into tensor-memory accumulator g % 2
//            (mbarrier mma[g % 2]) as soon as its A operand (buffer g % 2) is built;
//   compute (warps 0-11) per step g: expand step g's words into A buffer g % 2 and meet the
//            producer (named barrier 1); read step g - 1's accumulator (warp w: the lanes of
//            quadrant w % 4 = positions, leaves [56 (w / 4), + 56) up to 162), reduce to [0, 2q)
//            and add chat_j(v) What_{j,p}(v) into per-thread accumulators; load step g + 1's chat
//            row into ctile[(g + 1) % 3].
// After an item's last column its sums, reduced to [0, q), are added into the transposed scratch
// vhat_t[v][p] (u32, zeroed by the caller; a warp's 32 positions are one coalesced atomic add; at
// most 2^16 splits keep the total below 2^32) and k_fold_finish_t inverts.
constexpr int TCF_CTHREADS = 384;  // 12 compute warps: with the producer, 128 registers a thread
constexpr int TCF_THREADS = TCF_CTHREADS + 32;
constexpr int TCF_ROWS = 128;
constexpr int TCF_WT_BYTES = TCF_ROWS * 24;  // one step's witness words
constexpr int TCF_OFF_A = TC_B_BYTES;        // two A buffers
constexpr int TCF_OFF_WTILE = TCF_OFF_A + 2 * TCC_A_BYTES;
constexpr int TCF_OFF_CT = TCF_OFF_WTILE + 2 * TCF_WT_BYTES;
constexpr int TCF_OFF_BAR = TCF_OFF_CT + 3 * 176 * 4;
constexpr int TCF_OFF_CUR = TCF_OFF_BAR + 64;  // four step cursors
constexpr int TCF_SMEM = TCF_OFF_CUR + 4 * 32 + 1024;
constexpr uint32_t TCF_TMEM_COLS = 512;
static_assert(TCF_OFF_A % TC_ATOM == 0 && (TCF_OFF_A + TCC_A_BYTES) % TC_ATOM == 0 && TCF_OFF_WTILE % 16 == 0 && TCF_OFF_CT % 16 == 0 && TCF_OFF_BAR % 8 == 0, "alignment");
static_assert(TCF_SMEM <= 232448, "shared memory per CTA");

// A position in a CTA's fold items (item it: position tile it % tiles, column split it / tiles;
// step st is column c0 + st), the item's bounds computed once when it starts.
struct TcfCursor {
  int it, st, n, c0, tile, split;
  __device__ void load(int item, int stride, int total, int tiles, int cols, int cols_per_split) {
    it = item;
    st = 0;
    n = 0;
    while (it < total) {
      split = it / tiles;
      c0 = split * cols_per_split;
      n = min(cols, c0 + cols_per_split) - c0;
      if (n > 0) {
        tile = it - split * tiles;
        return;
      }
      n = 0;
      it += stride;
    }
  }
};

template <int PI>
__global__ void __launch_bounds__(TCF_THREADS, 1)
    k_fold_tc(const uint64_t* __restrict__ W, size_t wdim, int cols, int cols_per_split,
              const uint32_t* __restrict__ chat, const uint8_t* __restrict__ tcb, uint32_t* __restrict__ vhat_t,
              const int* __restrict__ split_inst) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);  // swizzle atoms
  uint8_t* sB = smem;
  uint8_t* sA = smem + TCF_OFF_A;
  uint64_t* wtile = (uint64_t*)(smem + TCF_OFF_WTILE);
  uint32_t* ctile = (uint32_t*)(smem + TCF_OFF_CT);  // [3][176]
  uint64_t* full = (uint64_t*)(smem + TCF_OFF_BAR);  // [2]: step g's words
  uint64_t* mma = full + 2;                          // [2]: step g's multiply done
  uint64_t* bfull = full + 4;
  uint32_t* tslot = (uint32_t*)(full + 5);
  volatile int* abort = (volatile int*)(full + 6);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = (int)((wdim + TCF_ROWS - 1) / TCF_ROWS);
  const int splits = (cols + cols_per_split - 1) / cols_per_split;
  const int total = tiles * splits;
  auto advance = [&](TcfCursor& c) {
    if (++c.st < c.n) return;
    c.load(c.it + (int)gridDim.x, (int)gridDim.x, total, tiles, cols, cols_per_split);
  };
  // step g's cursor in slot g % 4: the producer writes step g + 1's before named barrier 1 of step
  // g; the compute warps read step g + 1's (chat row) and step g - 1's (item end) after it
  TcfCursor* curs = (TcfCursor*)(smem + TCF_OFF_CUR);
  int S = 0;
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    const int c0 = (it / tiles) * cols_per_split;
    S += max(0, min(cols, c0 + cols_per_split) - c0);
  }

  if (tid == 0) {
    for (int b = 0; b < 5; b++) tc::mbar_init(&full[b], 1);
    *abort = 0;
    curs[0].load(blockIdx.x, (int)gridDim.x, total, tiles, cols, cols_per_split);
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, TCF_TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (warp == TCF_CTHREADS / 32) {
    // ---------------- producer ----------------
    auto load_words = [&](const TcfCursor& c, int b) {
      const size_t p0 = (size_t)c.tile * TCF_ROWS;
      tc::mbar_arrive_expect_tx(&full[b], TCF_WT_BYTES);
      tc::bulk_g2s(wtile + b * (TCF_ROWS * 3), W + ((size_t)(c.c0 + c.st) * wdim + p0) * 3, TCF_WT_BYTES, &full[b]);
    };
    const uint32_t sA_u = tc::smem_u32(sA), sB_u = tc::smem_u32(sB);
    TcfCursor cur = curs[0];
    if (lane == 0 && S > 0) {
      tc::mbar_arrive_expect_tx(bfull, TC_B_BYTES);
      for (int x = 0; x < 4; x++)
        tc::bulk_g2s(sB + x * (TC_B_BYTES / 4), tcb + x * (TC_B_BYTES / 4), TC_B_BYTES / 4, bfull);
      load_words(cur, 0);
    }
    for (int g = 0; g < S; g++) {
      TcfCursor nxt = cur;
      advance(nxt);
      // step g + 1's words into buffer (g + 1) % 2, whose step g - 1 the compute warps have expanded
      if (lane == 0) {
        if (nxt.it < total) load_words(nxt, (g + 1) & 1);
        curs[(g + 1) & 3] = nxt;
      }
      __syncwarp();
      tc::named_sync(1, TCF_THREADS);  // step g's A operand is built
      if (lane == 0) {
        tc::fence_after_sync();
        if (g == 0) tc_wait(bfull, 0, abort);
        if (!*abort)
          tc_transform_mma(tmem + (uint32_t)(g & 1) * 256u, sA_u + (uint32_t)(g & 1) * TCC_A_BYTES, sB_u, &mma[g & 1]);
        else
          tc::mbar_arrive(&mma[g & 1]);
      }
      __syncwarp();
      cur = nxt;
    }
  } else if (S > 0) {
    // ---------------- compute ----------------
    const int quad = warp & 3, part = warp >> 2;
    const int v0 = 56 * part;  // leaves v0 .. v0 + 55 (v0 + 49 for the last part)
    const int row = 32 * quad + lane;
    uint32_t acc[56];
#pragma unroll
    for (int i = 0; i < 56; i++) acc[i] = 0;
    constexpr int RED = FoldRed<PI>::value;
    int since = 0;
    // step 0's chat row
    if (tid < N162) ctile[tid] = chat[(size_t)curs[0].c0 * N162 + tid];
    tc::named_sync(2, TCF_CTHREADS);
    for (int g = 0; g <= S; g++) {
      uint32_t cnext = 0;  // step g + 1's chat row, stored at the end of the iteration
      const bool has_next = g + 1 < S && tid < N162;
      if (g < S) {
        tc_wait(&full[g & 1], (g >> 1) & 1, abort);                   // step g's words
        if (g >= 2) tc_wait(&mma[g & 1], ((g - 2) >> 1) & 1, abort);  // A buffer g % 2 free
        tc_build_row_inline<12 * 128 / TCF_CTHREADS>(sA + (g & 1) * TCC_A_BYTES, tid, TCF_CTHREADS,
                                                   wtile + (g & 1) * (TCF_ROWS * 3) + (tid & 127) * 3);
        tc::fence_async_shared();
        tc::fence_before_sync();
        tc::named_sync(1, TCF_THREADS);  // meets the producer: lockstep, even when a wait timed out
      }
      if (has_next) {
        const TcfCursor& nxt = curs[(g + 1) & 3];
        cnext = __ldg(chat + (size_t)(nxt.c0 + nxt.st) * N162 + tid);
      }
      if (g >= 1) {
        const TcfCursor& prev = curs[(g - 1) & 3];
        tc_wait(&mma[(g - 1) & 1], ((g - 1) >> 1) & 1, abort);  // step g - 1's accumulator
        tc::fence_after_sync();
        const uint32_t taddr = tmem + (uint32_t)((g - 1) & 1) * 256u + ((uint32_t)(32 * quad) << 16);
        const uint32_t* ch = ctile + ((g - 1) % 3) * 176;
        // leaves v0 .. v0 + 47 in three batches of 16 (two loads, one wait), then v0 + 48 .. v0 + 55
        // (the last part: its leaves 160-161)
#pragma unroll
        for (int bt = 0; bt < 3; bt++) {
          uint32_t x[16];
          tc::tmem_ld8_nowait(taddr + v0 + 16 * bt, x);
          tc::tmem_ld8_nowait(taddr + v0 + 16 * bt + 8, x + 8);
          tc::tmem_wait_ld(x);
#pragma unroll
          for (int i = 0; i < 16; i += 4) {
            const uint4 c4 = *(const uint4*)(ch + v0 + 16 * bt + i);
            acc[16 * bt + i] += c4.x * red_half<PI>(x[i]);
            acc[16 * bt + i + 1] += c4.y * red_half<PI>(x[i + 1]);
            acc[16 * bt + i + 2] += c4.z * red_half<PI>(x[i + 2]);
            acc[16 * bt + i + 3] += c4.w * red_half<PI>(x[i + 3]);
          }
        }
        if (part < 2) {
          uint32_t x[8];
          tc::tmem_ld8_nowait(taddr + v0 + 48, x);
          tc::tmem_wait_ld(x);
#pragma unroll
          for (int i = 0; i < 8; i += 4) {
            const uint4 c4 = *(const uint4*)(ch + v0 + 48 + i);
            acc[48 + i] += c4.x * red_half<PI>(x[i]);
            acc[49 + i] += c4.y * red_half<PI>(x[i + 1]);
            acc[50 + i] += c4.z * red_half<PI>(x[i + 2]);
            acc[51 + i] += c4.w * red_half<PI>(x[i + 3]);
          }
        } else {
          uint32_t y[2];
          tc::tmem_ld2(taddr + 160, y);  // the last part's leaves 160 and 161
          acc[48] += ch[160] * red_half<PI>(y[0]);
          acc[49] += ch[161] * red_half<PI>(y[1]);
        }
        tc::fence_before_sync();
        if (++since >= RED) {
          since = 0;
#pragma unroll
          for (int i = 0; i < 56; i++) acc[i] = red_half<PI>(acc[i]);
        }
        if (prev.st + 1 == prev.n) {
          // the item's last column: its sums into vhat_t, a warp's 32 positions per add
          const size_t p0 = (size_t)prev.tile * TCF_ROWS;
          uint32_t* dst = vhat_t + (split_inst ? (size_t)split_inst[prev.split] * wdim * N162 : 0) + p0 + row;
          if (p0 + row < wdim) {
#pragma unroll
            // one pointer walked by an opaque stride, so that the 56 addresses are not hoisted
            // out of the step loop into registers
            size_t stride = wdim;
            asm volatile("" : "+l"(stride));
            uint32_t* d = dst + (size_t)v0 * stride;
            for (int i = 0; i < 56; i++, d += stride)
              if (part < 2 || i < 50) atomicAdd(d, red_full<PI>(acc[i]));
          }
#pragma unroll
          for (int i = 0; i < 56; i++) acc[i] = 0;
          since = 0;
        }
      }
      if (has_next) ctile[((g + 1) % 3) * 176 + tid] = cnext;
      tc::named_sync(2, TCF_CTHREADS);  // the chat row of step g + 1 is in place
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCF_TMEM_COLS);
  if (tid == 0 && *abort) atomicExch(&g_tc_timeout, 1);
}

// The inverse transform of each position's sums from the transposed scratch vhat_t (per instance
// [162][wdim]), centred into the folded witness, as k_fold_finish.
// =============================================================================================
// Fold as one tensor-core product per column: the challenge folded into the transform operand
// =============================================================================================
// v^_p(v) = sum_j c^_j(v) w^_{j,p}(v) = sum_j sum_m bit_m(W[j][p]) G_j[m][v] with
// G_j[m][v] = c^_j(v) T[m][v] mod q: the challenge weight moves from the CUDA cores into the
// multiply's B operand. k_fold_operand builds G_j for every column in the transform operand's layout
// (lo + 128 hi, K-major, 128-byte swizzle); k_fold_gm then accumulates, for 128 positions, the
// product of the bits (the commit's A operand, bits and 128 x bits) with G_j over all the columns
// of a work item in one tensor-memory accumulator (below 2^31 for at most 512 columns: 512 x 162 x
// (q - 1) < 2^31 for every prime here), and reads it back once per item. The CUDA cores only expand
// the bits and reduce each item's sums.
constexpr int GM_MAX_COLS_PER_SPLIT = 512;

// One thread per (column j, row v of N, 16-byte chunk c of K): the chunk's 16 bytes of G_j.
template <int PI>
__global__ void k_fold_operand(const uint32_t* __restrict__ chat /* [cols][162] */, int cols,
                               const uint8_t* __restrict__ tcb /* T: the operand, then u16 rows */,
                               uint8_t* __restrict__ G) {
  constexpr uint32_t q = Pr<PI>::q;
  const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  constexpr int CHUNKS = TC_KBYTES / 16;  // 24
  if (gid >= (size_t)cols * TC_LEAVES * CHUNKS) return;
  const int c = (int)(gid % CHUNKS);
  const int v = (int)((gid / CHUNKS) % TC_LEAVES);
  const int j = (int)(gid / ((size_t)CHUNKS * TC_LEAVES));
  const int kb0 = 16 * c;
  const bool hi = kb0 >= 192;
  uint32_t bytes[4] = {0, 0, 0, 0};
  const int m0 = hi ? kb0 - 192 : kb0;
  if (v < N162 && m0 < N162) {
    const uint32_t cv = chat[(size_t)j * N162 + v];
    // T[m0 .. m0 + 15][v]: 32 bytes of the plain table after the operand (zero past m = 161)
    const uint4* trow = reinterpret_cast<const uint4*>(tcb + TC_B_BYTES) + ((size_t)v * TC_LEAVES + m0) / 8;
    const uint4 ta = trow[0], tb = trow[1];
    const uint32_t tw[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
    for (int x = 0; x < 16; x++) {
      const uint32_t t = (tw[x >> 1] >> (16 * (x & 1))) & 0xFFFFu;
      const uint32_t g = red_full<PI>(cv * t);
      bytes[x >> 2] |= (hi ? g >> 7 : g & 127u) << (8 * (x & 3));
    }
  }
  *(uint4*)(G + (size_t)j * TC_B_BYTES + tc_swizzled_offset(v, kb0, TC_LEAVES)) =
      make_uint4(bytes[0], bytes[1], bytes[2], bytes[3]);
}

// A position in a CTA's k_fold_gm items, as TcfCursor, with the accumulator the item uses (the
// CTA's items alternate between two).
struct GmCursor {
  TcfCursor c;
  int acc;
};

// Persistent over items (128 positions x a column split), one column a step, two warp roles:
//   producer (warp 12, one lane): for step g, once step g - 2's multiply is done, copies G_j into B
//            buffer g % 2 and step g + 1's witness words into wtile (g + 1) % 2 (bulk copies), writes
//            step g + 1's cursor, meets the compute warps (named barrier 1), then issues step g's
//            multiply into the item's accumulator (accumulating after the item's first K-step);
//   compute (warps 0-11) for step g: once step g - 1's multiply is done (the A buffer is free), add
//            the sums of an item that step g - 1 ended into vhat_t (warp w: the lanes of quadrant
//            w % 4 = positions, leaves [56 (w / 4), + 56)), then expand step g's words into A and
//            meet the producer.
constexpr int GM_THREADS = TCF_THREADS;  // 12 compute warps and the producer warp
constexpr int GM_OFF_A = 2 * TC_B_BYTES;  // two B buffers, then one A buffer
constexpr int GM_OFF_WT = GM_OFF_A + TCC_A_BYTES;
constexpr int GM_OFF_BAR = GM_OFF_WT + 2 * TCF_WT_BYTES;
constexpr int GM_OFF_CUR = GM_OFF_BAR + 64;
constexpr int GM_SMEM = GM_OFF_CUR + 4 * (int)sizeof(GmCursor) + 1024;
static_assert(GM_OFF_A % TC_ATOM == 0 && TC_B_BYTES % TC_ATOM == 0 && GM_OFF_WT % 16 == 0 && GM_OFF_BAR % 8 == 0 &&
                  GM_OFF_CUR % 8 == 0,
              "alignment");
static_assert(GM_SMEM <= 232448, "shared memory per CTA");

// Issue the 12 K-steps of one column's 128 x 176 x 384 multiply (accumulating unless `first`) and
// commit them to `bar`.
__device__ __forceinline__ void gm_mma(uint32_t d_tmem, uint32_t sA_u, uint32_t sB_u, bool first, uint64_t* bar) {
  constexpr uint32_t IDESC = tc::idesc_u8(128, TC_LEAVES);
#pragma unroll
  for (int kk = 0; kk < TC_KBYTES / 32; kk++) {
    const uint32_t a = sA_u + (kk >> 2) * (128 * 128) + (kk & 3) * 32;
    const uint32_t b = sB_u + (kk >> 2) * (TC_LEAVES * 128) + (kk & 3) * 32;
    tc::mma_i8(d_tmem, tc::smem_desc_sw128(a, TC_ATOM), tc::smem_desc_sw128(b, TC_ATOM), IDESC,
               (first && kk == 0) ? 0u : 1u);
  }
  tc::commit_to(bar);
}

template <int PI>
__global__ void __launch_bounds__(GM_THREADS, 1)
    k_fold_gm(const uint64_t* __restrict__ W, size_t wdim, int cols, int cols_per_split,
              const uint8_t* __restrict__ G, uint32_t* __restrict__ vhat_t,
              const int* __restrict__ split_inst /* null: one instance */) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);  // swizzle atoms
  uint8_t* sB = smem;                                                           // [2] G_j
  uint8_t* sA = smem + GM_OFF_A;
  uint64_t* wtile = (uint64_t*)(smem + GM_OFF_WT);  // [2][128][3]
  uint64_t* wfull = (uint64_t*)(smem + GM_OFF_BAR);  // [2]: step g's words landed
  uint64_t* bfull = wfull + 2;                       // [2]: step g's G_j landed
  uint64_t* mma = wfull + 4;                         // [2]: step g's multiply done
  uint32_t* tslot = (uint32_t*)(wfull + 6);
  volatile int* abort = (volatile int*)(wfull + 7);
  GmCursor* curs = (GmCursor*)(smem + GM_OFF_CUR);  // step g's cursor in slot g % 4
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = (int)((wdim + TCF_ROWS - 1) / TCF_ROWS);
  const int splits = (cols + cols_per_split - 1) / cols_per_split;
  const int total = tiles * splits;
  int S = 0;
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    const int c0 = (it / tiles) * cols_per_split;
    S += max(0, min(cols, c0 + cols_per_split) - c0);
  }
  auto advance = [&](GmCursor& g) {
    if (++g.c.st < g.c.n) return;
    g.c.load(g.c.it + (int)gridDim.x, (int)gridDim.x, total, tiles, cols, cols_per_split);
    g.acc ^= 1;
  };

  if (tid == 0) {
    for (int b = 0; b < 6; b++) tc::mbar_init(&wfull[b], 1);
    *abort = 0;
    curs[0].c.load(blockIdx.x, (int)gridDim.x, total, tiles, cols, cols_per_split);
    curs[0].acc = 0;
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, TCF_TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (warp == TCF_CTHREADS / 32) {
    // ---------------- producer (one lane) ----------------
    auto load_words = [&](const GmCursor& g, int b) {
      const size_t p0 = (size_t)g.c.tile * TCF_ROWS;
      tc::mbar_arrive_expect_tx(&wfull[b], TCF_WT_BYTES);
      tc::bulk_g2s(wtile + b * (TCF_ROWS * 3), W + ((size_t)(g.c.c0 + g.c.st) * wdim + p0) * 3, TCF_WT_BYTES,
                   &wfull[b]);
    };
    const uint32_t sA_u = tc::smem_u32(sA), sB_u = tc::smem_u32(sB);
    GmCursor cur = curs[0];
    if (lane == 0 && S > 0) load_words(cur, 0);
    for (int g = 0; g < S; g++) {
      const int b = g & 1;
      GmCursor nxt = cur;
      advance(nxt);
      if (lane == 0) {
        // G_j of step g into B buffer b, whose last reader was step g - 2's multiply
        if (g >= 2) tc_wait(&mma[b], ((g - 2) >> 1) & 1, abort);
        const int j = cur.c.c0 + cur.c.st;
        tc::mbar_arrive_expect_tx(&bfull[b], TC_B_BYTES);
        for (int x = 0; x < 4; x++)
          tc::bulk_g2s(sB + b * TC_B_BYTES + x * (TC_B_BYTES / 4), G + (size_t)j * TC_B_BYTES + x * (TC_B_BYTES / 4),
                       TC_B_BYTES / 4, &bfull[b]);
        // step g + 1's words into wtile (g + 1) % 2, whose step g - 1 the compute warps expanded
        if (g + 1 < S) load_words(nxt, (g + 1) & 1);
        curs[(g + 1) & 3] = nxt;
      }
      __syncwarp();
      tc::named_sync(1, GM_THREADS);  // step g's A operand is built
      if (lane == 0) {
        tc::fence_after_sync();
        tc_wait(&bfull[b], (g >> 1) & 1, abort);
        if (!*abort)
          gm_mma(tmem + (uint32_t)cur.acc * 256u, sA_u, sB_u + (uint32_t)b * TC_B_BYTES, cur.c.st == 0, &mma[b]);
        else
          tc::mbar_arrive(&mma[b]);
      }
      __syncwarp();
      cur = nxt;
    }
    if (lane == 0) {
      // the last copies and multiplies have landed before the CTA winds down (bounded waits that
      // ignore the abort flag)
      for (int g = S - 2 < 0 ? 0 : S - 2; g < S; g++) {
        tc::mbar_wait(&bfull[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
        tc::mbar_wait(&mma[g & 1], (g >> 1) & 1, TC_WAIT_BUDGET);
      }
    }
  } else if (S > 0) {
    // ---------------- compute ----------------
    const int quad = warp & 3, part = warp >> 2;
    const int v0 = 56 * part;  // leaves v0 .. v0 + 55 (v0 + 49 for the last part)
    const int row = 32 * quad + lane;
    // the sums of the item that step s ended, from its accumulator into vhat_t
    auto drain = [&](int s) {
      const GmCursor& it = curs[s & 3];
      const uint32_t taddr = tmem + (uint32_t)it.acc * 256u + ((uint32_t)(32 * quad) << 16) + v0;
      const size_t p0 = (size_t)it.c.tile * TCF_ROWS;
      uint32_t* d = vhat_t + (split_inst ? (size_t)split_inst[it.c.split] * wdim * N162 : 0) + p0 + row +
                    (size_t)v0 * wdim;
      const bool inside = p0 + row < wdim;
#pragma unroll
      for (int bt = 0; bt < 7; bt++) {
        uint32_t x[8];
        tc::tmem_ld8(taddr + 8 * bt, x);
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int v = v0 + 8 * bt + i;
          if (inside && v < N162) atomicAdd(d + (size_t)(8 * bt + i) * wdim, red_full<PI>(x[i]));
        }
      }
    };
    for (int g = 0; g < S; g++) {
      if (g >= 1) {
        tc_wait(&mma[(g - 1) & 1], ((g - 1) >> 1) & 1, abort);  // step g - 1's multiply: A is free
        tc::fence_after_sync();
        const GmCursor& prev = curs[(g - 1) & 3];
        if (prev.c.st + 1 == prev.c.n) drain(g - 1);
      }
      tc_wait(&wfull[g & 1], (g >> 1) & 1, abort);  // step g's words
      tc_build_row_inline<12 * 128 / TCF_CTHREADS>(sA, tid, TCF_CTHREADS, wtile + (g & 1) * (TCF_ROWS * 3) + (tid & 127) * 3);
      tc::fence_async_shared();
      tc::fence_before_sync();
      tc::named_sync(1, GM_THREADS);  // meets the producer: lockstep, even when a wait timed out
    }
    // the last item's sums
    tc_wait(&mma[(S - 1) & 1], ((S - 1) >> 1) & 1, abort);
    tc::fence_after_sync();
    drain(S - 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCF_TMEM_COLS);
  if (tid == 0 && *abort) atomicExch(&g_tc_timeout, 1);
}

template <int PI>
__global__ void __launch_bounds__(216) k_fold_finish_t(const uint32_t* __restrict__ vhat_t, size_t wdim,
                                                       size_t positions, const DevPrime* __restrict__ D,
                                                       int16_t* __restrict__ v_out /* [len_ring][648] */) {
  __shared__ uint32_t xs[4][N162];
  const int g = threadIdx.x / 54, j = threadIdx.x - 54 * g;
  const size_t p = (size_t)blockIdx.x * 4 + g;
  const size_t inst = p / wdim, pl = p - inst * wdim;
  const uint32_t* src = vhat_t + inst * wdim * N162 + pl;
  for (int v = j; v < N162; v += 54) xs[g][v] = p < positions ? src[(size_t)v * wdim] % Pr<PI>::q : 0;
  __syncthreads();
  intt162_group<PI>(xs[g], j, *D);
  if (p < positions) {
    const size_t i = p / 4;
    const int k = (int)(p % 4);
    for (int m = j; m < N162; m += 54) v_out[i * N648 + 4 * m + k] = center<PI>(xs[g][m]);
  }
}

// The inverse transform of each position's sums, centred, into the folded witness: position
// p = 4 i + k gives coefficients 4 m + k of ring element i (crates/pcs/src/fold.rs:620-677).
template <int PI>
__global__ void __launch_bounds__(216) k_fold_finish(const uint32_t* __restrict__ vhat, size_t wdim,
                                                     const DevPrime* __restrict__ D,
                                                     int16_t* __restrict__ v_out /* [len_ring][648] */) {
  // four positions per CTA, 54 threads each: the inverse 162-point transform in shared memory
  __shared__ uint32_t xs[4][N162];
  const int g = threadIdx.x / 54, j = threadIdx.x - 54 * g;
  const size_t p = (size_t)blockIdx.x * 4 + g;
  for (int v = j; v < N162; v += 54) xs[g][v] = p < wdim ? vhat[p * N162 + v] % Pr<PI>::q : 0;
  __syncthreads();
  intt162_group<PI>(xs[g], j, *D);
  if (p < wdim) {
    const size_t i = p / 4;
    const int k = (int)(p % 4);
    for (int m = j; m < N162; m += 54) v_out[i * N648 + 4 * m + k] = center<PI>(xs[g][m]);
  }
}

// Verifier::fold_commitment: out[row][limb][s] = sum_j chat_j(s) C_j[row][limb][s]
// (crates/pcs/src/scheme/verifier.rs:114-146).
template <int PI>
__global__ void __launch_bounds__(1024) k_fold_commitment(const int16_t* __restrict__ C, int cols, int limb, int limbs,
                                                          const uint32_t* __restrict__ chat,
                                                          const DevPrime* __restrict__ D, int16_t* __restrict__ out) {
  // CTA (slot group, row): lane = slot (consecutive slots, coalesced loads of C), warp w sums the
  // columns w, w + 32, ...; the 32 warps' sums are added in shared memory
  __shared__ uint32_t part[32][33];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.y, s = blockIdx.x * 32 + lane;
  constexpr int32_t q = Pr<PI>::q;
  uint64_t acc = 0;
  if (s < N162) {
    const int leaf = D->pow3_to_leaf[s];
    for (int j = warp; j < cols; j += 32) {
      int32_t c = C[(((size_t)j * 4 + row) * limbs + limb) * N162 + s];
      uint32_t cm = (uint32_t)(c < 0 ? c + q : c);
      acc += (uint64_t)chat[(size_t)j * N162 + leaf] * cm;
    }
  }
  part[warp][lane] = (uint32_t)(acc % q);
  __syncthreads();
  if (warp == 0 && s < N162) {
    uint32_t t = 0;
    for (int w = 0; w < 32; w++) t += part[w][lane];
    out[(row * limbs + limb) * N162 + s] = center<PI>(t % q);
  }
}

// =============================================================================================
// Bit-drop (crates/pcs/src/bd/digits.rs:121-181): per limb, the coefficients of each column's
// commitment (component d's coefficients are coefficients 4m + d), then Garner digits.
// =============================================================================================
template <int PI>
__global__ void __launch_bounds__(216) k_column_residues(const int16_t* __restrict__ C, int cols, int limb, int limbs,
                                                         const DevPrime* __restrict__ D,
                                                         uint16_t* __restrict__ res /* [cols*648] */) {
  // one column per CTA, 54 threads per component: the inverse 162-point transform in shared memory
  __shared__ uint32_t xs[4][N162];
  const int d = threadIdx.x / 54, t = threadIdx.x - 54 * d;
  const int j = blockIdx.x;
  constexpr int32_t q = Pr<PI>::q;
  for (int s = t; s < N162; s += 54) {
    int32_t c = C[(((size_t)j * 4 + d) * limbs + limb) * N162 + s];
    xs[d][D->pow3_to_leaf[s]] = (uint32_t)(c < 0 ? c + q : c);
  }
  __syncthreads();
  intt162_group<PI>(xs[d], t, *D);
  for (int m = t; m < N162; m += 54) res[(size_t)j * N648 + 4 * m + d] = (uint16_t)xs[d][m];
}

// The recursive opening's residues (crates/pcs/src/recursion/limbs.rs:379-398, drain_batch :311-325):
// for one limb, vector l (component l) holds each column's coefficients 4m + l, centred, times
// (-1)^m, cut into three chunks of 54 (chunk b of column j is polynomial b * cols + j, positions
// 0..53; the rest of the 64 positions and the padding polynomials are zero). One thread per output
// coefficient; `res` is the limb's coefficients in [0, q) as k_column_residues leaves them.
__global__ void k_recursion_residues(const uint16_t* __restrict__ res, int cols, size_t polys, int32_t q,
                                     int16_t* __restrict__ out /* [4][polys][64] */) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * polys * 64) return;
  const int pos = (int)(i & 63);
  const size_t poly = (i >> 6) % polys;
  const int l = (int)((i >> 6) / polys);
  int32_t v = 0;
  if (pos < 54 && poly < (size_t)3 * cols) {
    const int b = (int)(poly / cols), j = (int)(poly - (size_t)b * cols);
    const int m = 54 * b + pos;
    int32_t c = res[(size_t)j * N648 + 4 * m + l];
    if (c > (q - 1) / 2) c -= q;
    v = (m & 1) ? -c : c;
  }
  out[i] = (int16_t)v;
}

// Prover::commit_left_expansion's vector u (crates/pcs/src/scheme/prover.rs:95-115): chunk b of the
// lift of row value j (its bits 54 b .. 54 b + 53 as 0/1 coefficients, crates/pcs/src/recursion/
// binary.rs:49-51, chunk.rs:76-86) at polynomial b * cols + j; the rest zero. One thread per output
// coefficient.
__global__ void k_left_expansion(const uint64_t* __restrict__ u /* [cols][3] */, int cols, size_t rank,
                                 int16_t* __restrict__ out /* [rank][64] */) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rank * 64) return;
  const int pos = (int)(i & 63);
  const size_t poly = i >> 6;
  int16_t v = 0;
  if (pos < 54 && poly < (size_t)3 * cols) {
    const int b = (int)(poly / cols), j = (int)(poly - (size_t)b * cols);
    const int bit = 54 * b + pos;
    v = (int16_t)((u[(size_t)j * 3 + (bit >> 6)] >> (bit & 63)) & 1);
  }
  out[i] = v;
}

__global__ void k_garner(const uint16_t* __restrict__ res, size_t count, int limbs, GarnerConsts g,
                         uint16_t* __restrict__ top, uint16_t* __restrict__ digits) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t base = res[i];
  top[i] = (uint16_t)((base + (1u << (g.dropped_bits - 1))) >> g.dropped_bits);
  uint32_t mixed[7];
  mixed[0] = base;
  for (int k = 1; k < limbs; k++) {
    uint32_t q = g.q[k];
    uint32_t x = res[(size_t)k * count + i];
    for (int m = 0; m < k; m++)
      x = (uint32_t)((uint64_t)((x + q - mixed[m] % q) % q) * g.inv[k][m] % q);
    mixed[k] = x;
    digits[(size_t)(k - 1) * count + i] = (uint16_t)x;
  }
}

// The bit-dropped residual (crates/pcs/src/bd/residual.rs:66-130) on the device.
// k_bd_columns: the columns rebuilt from the top bits and the Garner digits modulo limb `limb`
// ((top << dropped_bits) + q_0 (d_1 + q_1 (d_2 + ...)), crates/pcs/src/simd/bd.rs:5-36), in the
// commitment's component form: component d of column j is the forward 162-point transform of
// coefficients 4m + d, written at C[j][d][limb][slot] centred (the inverse of k_column_residues).
template <int PI>
__global__ void __launch_bounds__(216) k_bd_columns(const uint16_t* __restrict__ top, const uint16_t* __restrict__ digits, int cols, int limb,
                             GarnerConsts g, int limbs, const DevPrime* __restrict__ D, int16_t* __restrict__ C) {
  // one column per CTA, 54 threads per component, the transform in shared memory
  __shared__ uint32_t xs[4][N162];
  const int d = threadIdx.x / 54, t = threadIdx.x - 54 * d;
  const int j = blockIdx.x;
  constexpr uint32_t q = Pr<PI>::q;
  const size_t count = (size_t)cols * N648;
  for (int m = t; m < N162; m += 54) {
    const size_t at = (size_t)j * N648 + 4 * m + d;
    uint32_t inner = 0;
    if (limbs > 1) {
      inner = digits[(size_t)(limbs - 2) * count + at] % q;
      for (int k = limbs - 3; k >= 0; k--) inner = (digits[(size_t)k * count + at] + inner * g.q[k + 1]) % q;
    }
    xs[d][m] = (uint32_t)((((uint64_t)top[at] << g.dropped_bits) + (uint64_t)inner * g.q[0]) % q);
  }
  __syncthreads();
  ntt162_group<PI>(xs[d], t, *D);
  for (int s = t; s < N162; s += 54)
    C[(((size_t)j * 4 + d) * limbs + limb) * N162 + s] = center<PI>(xs[d][D->pow3_to_leaf[s]]);
}

// k_bd_inverse: A v - the folded commitment for one limb, diff[row][leaf], back to the 648
// coefficients (row d holds coefficients 4m + d), modulo the limb.
template <int PI>
__global__ void k_bd_inverse(const uint32_t* __restrict__ diff, const DevPrime* __restrict__ D, uint32_t* __restrict__ res) {
  const int d = threadIdx.x;
  if (d >= 4) return;
  uint32_t x[N162];
  for (int leaf = 0; leaf < N162; leaf++) x[leaf] = diff[d * N162 + leaf];
  intt162_serial<PI>(x, *D);
  for (int m = 0; m < N162; m++) res[4 * m + d] = x[m];
}

// k_bd_normsq: the Garner recombination of the limbs' residues res[limb][648] and the squared norm
// of the centred integers (crates/pcs/src/bd/digits.rs:229-260), one CTA, out = the 128-bit sum
// as two words, low first.
__global__ void k_bd_normsq(const uint32_t* __restrict__ res, int limbs, GarnerConsts g, unsigned long long* out) {
  __shared__ unsigned __int128 red[1024];
  const int i = threadIdx.x;
  unsigned __int128 sq = 0;
  if (i < N648) {
    uint64_t mixed[7];
    unsigned __int128 modulus = 1;
    for (int k = 0; k < limbs; k++) {
      const uint64_t q = g.q[k];
      uint64_t x = res[(size_t)k * N648 + i] % q;
      for (int m = 0; m < k; m++) x = (x + q - mixed[m] % q) % q * g.inv[k][m] % q;
      mixed[k] = x;
      modulus *= q;
    }
    unsigned __int128 value = 0;
    for (int k = limbs - 1; k >= 0; k--) value = value * g.q[k] + mixed[k];
    unsigned __int128 mag = value > modulus / 2 ? modulus - value : value;
    sq = mag * mag;
  }
  red[i] = sq;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (i < o) red[i] += red[i + o];
    __syncthreads();
  }
  if (i == 0) {
    out[0] = (unsigned long long)red[0];
    out[1] = (unsigned long long)(red[0] >> 64);
  }
}

// =============================================================================================
// Row evaluation over F162 (crates/pcs/src/eval.rs:51-63, 171-193)
// =============================================================================================
// eq(p, i) = prod_k (p_k if bit k of i else 1 + p_k).
__global__ void k_eq_table(const uint64_t* __restrict__ p, int n, size_t count, int instances,
                           uint64_t* __restrict__ eq) {
  size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= count * (size_t)instances) return;
  // instances one after another: instance g / count's table from its own point
  size_t inst = g / count, i = g % count;
  p += inst * (size_t)n * 3;
  eq += inst * count * 3;
  F162d x{{1, 0, 0}};
  for (int k = 0; k < n; k++) {
    F162d pk{{p[3 * k], p[3 * k + 1], p[3 * k + 2]}};
    if (!((i >> k) & 1)) pk.w[0] ^= 1;
    x = f_mul(x, pk);
  }
  eq[3 * i] = x.w[0];
  eq[3 * i + 1] = x.w[1];
  eq[3 * i + 2] = x.w[2];
}

// Row evaluation by the method of four Russians over 8-row groups (crates/pcs/src/eval.rs:136-193
// computes the same sums one row at a time): u_j = sum_b x^b S_{j,b} mod x^162 + x^81 + 1 with
// S_{j,b} = XOR of eq[i] over the rows i whose W[i][j] has bit b set. Bit b of the 8 rows of a
// group, read as an 8-bit index, selects the XOR of their eq values to add to S_{j,b}; the index
// is split into two nibbles looked up in two 16-entry tables (rows 0-3 and 4-7 of the group), so
// a table is 16 entries of 3 words stored as three 128-byte word planes: the lanes' lookups hit
// distinct banks or the same address, never a conflict. A thread owns one byte position m of one
// column (bits 8m .. 8m+7): it gathers the 8 rows' bytes, transposes the 8x8 bit block and makes
// 16 lookups. The witness rows of the CTA's columns and their eq values arrive in stages of 32
// rows by cp.async, one stage ahead, coalesced (a column's rows are contiguous). CTAs split the
// rows; partial results are combined with atomic XORs into u (zeroed first).
constexpr int RE_COLS = 12;      // columns per CTA (12 x 21 byte positions = 252 threads)
constexpr int RE_THREADS = 256;
constexpr int RE_ROWS = 32;      // rows per stage (4 groups)
constexpr int RE_WS = RE_ROWS * 3 + 3;  // staged words per column, padded so that columns start 6 banks apart

__device__ __forceinline__ uint64_t transpose8x8(uint64_t x) {
  // byte k bit r -> byte r bit k
  uint64_t t;
  t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x = x ^ t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x = x ^ t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x = x ^ t ^ (t << 28);
  return x;
}

__global__ void __launch_bounds__(RE_THREADS) k_row_eval(const uint64_t* __restrict__ W, int wdim, int cols,
                                                         const uint64_t* __restrict__ eq_all,
                                                         const int4* __restrict__ tiles, int groups_per_split,
                                                         unsigned long long* __restrict__ u) {
  __shared__ uint64_t Ws[2][RE_COLS][RE_WS];         // the stage's witness rows, per column
  __shared__ uint64_t Es[2][RE_ROWS][3];             // the stage's eq values
  __shared__ uint64_t TL[RE_ROWS / 8][2][3][16];     // per group: two nibble tables, word planes
  __shared__ uint64_t Q[RE_COLS][21][4];
  int4 tile;
  if (tiles) tile = tiles[blockIdx.x];
  else tile = make_int4(RE_COLS * blockIdx.x, min(RE_COLS, cols - RE_COLS * (int)blockIdx.x), 0, 0);
  const uint64_t* eq = eq_all + (size_t)tile.z * wdim * 3;
  const int t = threadIdx.x;
  const int c = t / 21, m = t - 21 * (t / 21);
  const bool active = c < tile.y;
  const int limb = m >> 3, sh = 8 * (m & 7);
  const int G = wdim >> 3;
  const int g0 = blockIdx.y * groups_per_split, g1 = min(G, g0 + groups_per_split);
  const int r0 = 8 * g0, r1 = 8 * g1;
  uint64_t S[8][3];
#pragma unroll
  for (int r = 0; r < 8; r++) S[r][0] = S[r][1] = S[r][2] = 0;
  // stage at row i0 into buffer b: each column's 3 * rows words, and the rows' eq values
  auto stage = [&](int i0, int b) {
    const int words = 3 * min(RE_ROWS, r1 - i0);
    for (int x = t; x < tile.y * words; x += RE_THREADS) {
      const int cc = x / words, wd = x - cc * words;
      cp_async8(&Ws[b][cc][wd], W + ((size_t)(tile.x + cc) * wdim + i0) * 3 + wd);
    }
    for (int x = t; x < words; x += RE_THREADS) cp_async8(&Es[b][0][0] + x, eq + (size_t)i0 * 3 + x);
  };
  if (r0 < r1) stage(r0, 0);
  cp_async_commit();
  for (int i0 = r0, cur = 0; i0 < r1; i0 += RE_ROWS, cur ^= 1) {
    const int ngroups = min(RE_ROWS, r1 - i0) >> 3;
    cp_async_wait<0>();
    __syncthreads();  // the stage has landed, and the previous stage's lookups are done
    if (t < 32 * ngroups) {
      // entry e of the half-table h of group q: the XOR of eq over rows 8q + 4h + k, k the set bits of e
      const int q = t >> 5, h = (t >> 4) & 1, e = t & 15;
      uint64_t a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint64_t msk = 0 - (uint64_t)((e >> k) & 1);
        const uint64_t* x = Es[cur][8 * q + 4 * h + k];
        a0 ^= x[0] & msk;
        a1 ^= x[1] & msk;
        a2 ^= x[2] & msk;
      }
      TL[q][h][0][e] = a0;
      TL[q][h][1][e] = a1;
      TL[q][h][2][e] = a2;
    }
    if (i0 + RE_ROWS < r1) stage(i0 + RE_ROWS, cur ^ 1);
    cp_async_commit();
    __syncthreads();  // the tables are complete
    if (active) {
      for (int q = 0; q < ngroups; q++) {
        // this group's 8 bit rows of the thread's byte position, transposed: byte r = bit 8m + r
        // of the 8 rows
        uint64_t x = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) x |= ((Ws[cur][c][(8 * q + k) * 3 + limb] >> sh) & 0xFF) << (8 * k);
        x = transpose8x8(x);
#pragma unroll
        for (int r = 0; r < 8; r++) {
          const uint32_t idx = (uint32_t)(x >> (8 * r));
          const uint32_t lo = idx & 15, hi = (idx >> 4) & 15;
#pragma unroll
          for (int w = 0; w < 3; w++) S[r][w] ^= TL[q][0][w][lo] ^ TL[q][1][w][hi];
        }
      }
    }
  }
  // this thread's share of sum_b x^b S_b: bits 8m + r, placed from word `limb` on
  if (active) {
    uint64_t q4[4] = {0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < 8; r++) {
      if (8 * m + r >= 162) break;
      int bs = sh + r;
#pragma unroll
      for (int w = 0; w < 3; w++) {
        q4[w] ^= S[r][w] << bs;
        if (bs) q4[w + 1] ^= S[r][w] >> (64 - bs);
      }
    }
#pragma unroll
    for (int w = 0; w < 4; w++) Q[c][m][w] = q4[w];
  }
  __syncthreads();
  if (active && m == 0) {
    uint64_t P[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int mm = 0; mm < 21; mm++) {
      int ws = mm >> 3;
      for (int w = 0; w < 4; w++) P[ws + w] ^= Q[c][mm][w];
    }
    // reduce bits 322..162 by x^162 = x^81 + 1
    for (int bit = 322; bit >= 162; bit--) {
      if ((P[bit >> 6] >> (bit & 63)) & 1) {
        P[bit >> 6] ^= 1ull << (bit & 63);
        int a = bit - 162, b = bit - 81;
        P[a >> 6] ^= 1ull << (a & 63);
        P[b >> 6] ^= 1ull << (b & 63);
      }
    }
    unsigned long long* dst = u + 3 * (size_t)(tile.x + c);
    atomicXor(dst, (unsigned long long)P[0]);
    atomicXor(dst + 1, (unsigned long long)P[1]);
    atomicXor(dst + 2, (unsigned long long)P[2]);
  }
}

// claim(u, p1) = sum_j eq(p1, j) u_j: one thread per column, XOR-reduced per warp, then one
// atomic XOR per warp into out (zeroed by the caller).
__global__ void k_claim(const uint64_t* __restrict__ u, int cols, const uint64_t* __restrict__ p1, int n,
                        unsigned long long* __restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t a0 = 0, a1 = 0, a2 = 0;
  if (j < cols) {
    F162d x{{1, 0, 0}};
    for (int k = 0; k < n; k++) {
      F162d pk{{p1[3 * k], p1[3 * k + 1], p1[3 * k + 2]}};
      if (!((j >> k) & 1)) pk.w[0] ^= 1;
      x = f_mul(x, pk);
    }
    F162d y = f_mul(x, F162d{{u[3 * j], u[3 * j + 1], u[3 * j + 2]}});
    a0 = y.w[0];
    a1 = y.w[1];
    a2 = y.w[2];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a0 ^= __shfl_xor_sync(0xffffffffu, a0, o);
    a1 ^= __shfl_xor_sync(0xffffffffu, a1, o);
    a2 ^= __shfl_xor_sync(0xffffffffu, a2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicXor(out, (unsigned long long)a0);
    atomicXor(out + 1, (unsigned long long)a1);
    atomicXor(out + 2, (unsigned long long)a2);
  }
}

// The claims of all instances of a batch at once: one thread per column; a warp whose columns
// belong to one instance XOR-reduces and adds once, a warp over several instances adds per thread.
__global__ void k_claims(const RoundInst* __restrict__ inst, const int* __restrict__ col_inst,
                         const uint64_t* __restrict__ u, int total_cols, const uint64_t* __restrict__ p1,
                         unsigned long long* __restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int ii = j < total_cols ? col_inst[j] : -1;
  uint64_t a0 = 0, a1 = 0, a2 = 0;
  if (ii >= 0) {
    const RoundInst& I = inst[ii];
    int jj = j - (int)I.col_off;
    const uint64_t* p = p1 + 3 * 32 * ii;
    F162d x{{1, 0, 0}};
    for (int k = 0; k < (int)I.col_log; k++) {
      F162d pk{{p[3 * k], p[3 * k + 1], p[3 * k + 2]}};
      if (!((jj >> k) & 1)) pk.w[0] ^= 1;
      x = f_mul(x, pk);
    }
    F162d y = f_mul(x, F162d{{u[3 * j], u[3 * j + 1], u[3 * j + 2]}});
    a0 = y.w[0];
    a1 = y.w[1];
    a2 = y.w[2];
  }
  int i0 = __shfl_sync(0xffffffffu, ii, 0);
  bool uniform = __all_sync(0xffffffffu, ii == i0 || ii < 0);
  if (uniform) {
    for (int o = 16; o > 0; o >>= 1) {
      a0 ^= __shfl_xor_sync(0xffffffffu, a0, o);
      a1 ^= __shfl_xor_sync(0xffffffffu, a1, o);
      a2 ^= __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0 && i0 >= 0) {
      atomicXor(out + 3 * i0, (unsigned long long)a0);
      atomicXor(out + 3 * i0 + 1, (unsigned long long)a1);
      atomicXor(out + 3 * i0 + 2, (unsigned long long)a2);
    }
  } else if (ii >= 0) {
    atomicXor(out + 3 * ii, (unsigned long long)a0);
    atomicXor(out + 3 * ii + 1, (unsigned long long)a1);
    atomicXor(out + 3 * ii + 2, (unsigned long long)a2);
  }
}

// =============================================================================================
// The reference's 648-point transform (crates/pcs/src/scalar.rs:35-84) and its inverse (:123-177)
// for splitting primes, on general coefficients in [0, q): the NTT microbenchmark. 81 threads per
// ring element, E elements per CTA, three register stages joined through shared memory:
//   A: thread r holds indices r + 81k (k < 8): level 0 (the Phi split, stride 324) and the
//      radix-2 levels 1, 2 (strides 162, 81); afterwards x[k] sits in level-3 sub-ring k.
//   B: thread (k, t < 9) of sub-ring k holds 81k + t + 9a + 27b: radix-3 levels 3 (stride 27,
//      twiddle k) and 4 (stride 9, twiddle 3k + b).
//   C: thread g < 72 (a 9-block) holds 9g + c + 3d: levels 5 (stride 3, twiddle g) and 6
//      (stride 1, twiddle 3g + d).
// Forward values stay unreduced (Shoup products in [0, 2q), every level adds at most 6q, under
// 32q < 2^20 at the end) and are reduced once; the inverse's butterflies end in Shoup products,
// so its values stay in [0, 2q).
// =============================================================================================
constexpr int NTT_E = 4;  // ring elements per CTA

template <int PI>
__device__ __forceinline__ void bfly3_inv(uint32_t& y0, uint32_t& y1, uint32_t& y2, const Twiddle& t,
                                          const Ntt648Tables& T) {
  // a0 = (y0 + y1 + y2) / 3, a1 = (y0 + w^2 y1 + w y2) z^-1 / 3, a2 = (y0 + w y1 + w^2 y2) z^-2 / 3
  constexpr uint32_t q = Pr<PI>::q;
  uint32_t d = mul_shoup(y2 + 2 * q - y1, T.omega, T.omega_s, q);  // w (y2 - y1)
  uint32_t s1 = y0 + 2 * q - y1 + d;                              // y0 - y1 + w (y2 - y1)
  uint32_t s2 = y0 + 4 * q - y2 - d;                              // y0 - y2 - w (y2 - y1)
  uint32_t a0 = mul_shoup(y0 + y1 + y2, T.inv3, T.inv3s, q);
  y1 = mul_shoup(s1, t.z, t.zs, q);
  y2 = mul_shoup(s2, t.z2, t.z2s, q);
  y0 = a0;
}

template <int PI>
__global__ void __launch_bounds__(81 * NTT_E) k_ntt648_fwd(const uint16_t* __restrict__ in, uint16_t* __restrict__ out,
                                                           size_t count, const Ntt648Tables* __restrict__ Tg) {
  constexpr uint32_t q = Pr<PI>::q;
  __shared__ uint32_t s[NTT_E][N648];
  const Ntt648Tables& T = *Tg;
  const uint32_t om = T.omega, oms = T.omega_s;
  const int tid = threadIdx.x;
  size_t e0 = (size_t)blockIdx.x * NTT_E;
  {
    int e = tid / 81, r = tid - 81 * (tid / 81);
    size_t el = e0 + e;
    if (el < count) {
      const uint16_t* a = in + el * N648;
      uint32_t x[8];
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = a[r + 81 * k];
#pragma unroll
      for (int k = 0; k < 4; k++) {  // level 0: (a0 + z6 a1, a0 + a1 - z6 a1)
        uint32_t t = mul_shoup(x[k + 4], T.z6, T.z6s, q);
        uint32_t a0 = x[k];
        x[k] = a0 + t;
        x[k + 4] = a0 + x[k + 4] + 2 * q - t;
      }
#pragma unroll
      for (int sr = 0; sr < 2; sr++)  // level 1, sub-ring sr: pairs (4sr + k, 4sr + k + 2)
#pragma unroll
        for (int k = 0; k < 2; k++) {
          uint32_t t = mul_shoup(x[4 * sr + k + 2], T.f1[sr][0], T.f1[sr][1], q);
          uint32_t a0 = x[4 * sr + k];
          x[4 * sr + k] = a0 + t;
          x[4 * sr + k + 2] = a0 + 2 * q - t;
        }
#pragma unroll
      for (int sr = 0; sr < 4; sr++) {  // level 2, sub-ring sr: pair (2sr, 2sr + 1)
        uint32_t t = mul_shoup(x[2 * sr + 1], T.f2[sr][0], T.f2[sr][1], q);
        uint32_t a0 = x[2 * sr];
        x[2 * sr] = a0 + t;
        x[2 * sr + 1] = a0 + 2 * q - t;
      }
#pragma unroll
      for (int k = 0; k < 8; k++) s[e][r + 81 * k] = x[k];
    }
  }
  __syncthreads();
  if (tid < 72 * NTT_E) {
    int e = tid / 72, j = tid - 72 * (tid / 72), k = j / 9, t = j - 9 * (j / 9);
    if (e0 + e < count) {
      uint32_t y[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) y[a][b] = s[e][81 * k + t + 9 * a + 27 * b];
      Twiddle t3 = T.f3[k];
#pragma unroll
      for (int a = 0; a < 3; a++) bfly3<PI>(y[a][0], y[a][1], y[a][2], t3, om, oms);
#pragma unroll
      for (int b = 0; b < 3; b++) bfly3<PI>(y[0][b], y[1][b], y[2][b], T.f4[3 * k + b], om, oms);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) s[e][81 * k + t + 9 * a + 27 * b] = y[a][b];
    }
  }
  __syncthreads();
  if (tid < 72 * NTT_E) {
    int e = tid / 72, g = tid - 72 * (tid / 72);
    if (e0 + e < count) {
      uint32_t z[3][3];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) z[c][d] = s[e][9 * g + c + 3 * d];
      Twiddle t5 = T.f5[g];
#pragma unroll
      for (int c = 0; c < 3; c++) bfly3<PI>(z[c][0], z[c][1], z[c][2], t5, om, oms);
#pragma unroll
      for (int d = 0; d < 3; d++) bfly3<PI>(z[0][d], z[1][d], z[2][d], T.f6[3 * g + d], om, oms);
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) s[e][9 * g + 3 * d + c] = red_full<PI>(z[c][d]);
    }
  }
  __syncthreads();
  // coalesced write-back, two values per 32-bit word
  uint32_t* o32 = reinterpret_cast<uint32_t*>(out + e0 * N648);
  size_t words = (size_t)min((size_t)NTT_E, count - e0) * (N648 / 2);
  for (size_t w = tid; w < words; w += blockDim.x) {
    int e = (int)(w / (N648 / 2)), p = (int)(w - (size_t)e * (N648 / 2));
    o32[w] = s[e][2 * p] | (s[e][2 * p + 1] << 16);
  }
}

template <int PI>
__global__ void __launch_bounds__(81 * NTT_E) k_ntt648_inv(const uint16_t* __restrict__ in, uint16_t* __restrict__ out,
                                                           size_t count, const Ntt648Tables* __restrict__ Tg) {
  constexpr uint32_t q = Pr<PI>::q;
  __shared__ uint32_t s[NTT_E][N648];
  const Ntt648Tables& T = *Tg;
  const int tid = threadIdx.x;
  size_t e0 = (size_t)blockIdx.x * NTT_E;
  if (tid < 72 * NTT_E) {  // levels 6, 5
    int e = tid / 72, g = tid - 72 * (tid / 72);
    size_t el = e0 + e;
    if (el < count) {
      const uint16_t* v = in + el * N648 + 9 * g;
      uint32_t z[3][3];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) z[c][d] = v[c + 3 * d];
#pragma unroll
      for (int d = 0; d < 3; d++) bfly3_inv<PI>(z[0][d], z[1][d], z[2][d], T.i6[3 * g + d], T);
      Twiddle t5 = T.i5[g];
#pragma unroll
      for (int c = 0; c < 3; c++) bfly3_inv<PI>(z[c][0], z[c][1], z[c][2], t5, T);
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) s[e][9 * g + c + 3 * d] = z[c][d];
    }
  }
  __syncthreads();
  if (tid < 72 * NTT_E) {  // levels 4, 3
    int e = tid / 72, j = tid - 72 * (tid / 72), k = j / 9, t = j - 9 * (j / 9);
    if (e0 + e < count) {
      uint32_t y[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) y[a][b] = s[e][81 * k + t + 9 * a + 27 * b];
#pragma unroll
      for (int b = 0; b < 3; b++) bfly3_inv<PI>(y[0][b], y[1][b], y[2][b], T.i4[3 * k + b], T);
      Twiddle t3 = T.i3[k];
#pragma unroll
      for (int a = 0; a < 3; a++) bfly3_inv<PI>(y[a][0], y[a][1], y[a][2], t3, T);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) s[e][81 * k + t + 9 * a + 27 * b] = y[a][b];
    }
  }
  __syncthreads();
  {  // levels 2, 1, 0
    int e = tid / 81, r = tid - 81 * (tid / 81);
    size_t el = e0 + e;
    if (el < count) {
      uint32_t x[8];
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = s[e][r + 81 * k];
#pragma unroll
      for (int sr = 0; sr < 4; sr++) {  // (y0 + y1) / 2, (y0 - y1) z^-1 / 2
        uint32_t y0 = x[2 * sr], y1 = x[2 * sr + 1];
        x[2 * sr] = mul_shoup(y0 + y1, T.inv2, T.inv2s, q);
        x[2 * sr + 1] = mul_shoup(y0 + 2 * q - y1, T.i2[sr][0], T.i2[sr][1], q);
      }
#pragma unroll
      for (int sr = 0; sr < 2; sr++)
#pragma unroll
        for (int k = 0; k < 2; k++) {
          uint32_t y0 = x[4 * sr + k], y1 = x[4 * sr + k + 2];
          x[4 * sr + k] = mul_shoup(y0 + y1, T.inv2, T.inv2s, q);
          x[4 * sr + k + 2] = mul_shoup(y0 + 2 * q - y1, T.i1[sr][0], T.i1[sr][1], q);
        }
#pragma unroll
      for (int k = 0; k < 4; k++) {  // a1 = (y0 - y1) det, a0 = y0 - z6 a1
        uint32_t y0 = x[k], y1 = x[k + 4];
        uint32_t a1 = mul_shoup(y0 + 2 * q - y1, T.det, T.dets, q);
        uint32_t a0 = y0 + 2 * q - mul_shoup(a1, T.z6, T.z6s, q);
        x[k] = red_full<PI>(a0);
        x[k + 4] = red_full<PI>(a1);
      }
      uint16_t* a = out + el * N648;
#pragma unroll
      for (int k = 0; k < 8; k++) a[r + 81 * k] = (uint16_t)x[k];
    }
  }
}

// =============================================================================================
// The verifier (crates/pcs/src/scheme/verifier.rs:157-231): the norm of v, A v on every limb against
// the folded commitment, the binary check, the claim and the folded row value
// =============================================================================================
// Per ring element, the reference's 16 lane sums of squares (crates/pcs/src/simd/norm.rs:9-50):
// lane l adds x[32b + 2l]^2 + x[32b + 2l + 1]^2 over the 32-coefficient blocks b (the last block's
// 8 coefficients fall in lanes 0..3). A lane sum that reaches 2^31 wraps the reference's i32 lanes,
// which rejects. worst = the largest 16-bit absolute value (|-32768| stays negative and never wins).
__global__ void __launch_bounds__(256) k_v_norm(const int16_t* __restrict__ v, size_t len_ring,
                                                VerifyFlags* __restrict__ f) {
  // a warp per ring element: warp lane t sums the squares of coefficients t, t + 32, ...; the
  // reference's lane L is warp lanes 2L and 2L + 1
  const size_t e = (size_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int t = threadIdx.x & 31;
  if (e >= len_ring) return;
  const int16_t* x = v + e * N648;
  uint64_t sq = 0;
  int worst = 0;
  for (int i = t; i < N648; i += 32) {
    const int xi = x[i];
    sq += (uint64_t)(xi * xi);
    const int a = xi == -32768 ? -32768 : (xi < 0 ? -xi : xi);
    worst = a > worst ? a : worst;
  }
  int wrapped = sq + __shfl_xor_sync(0xffffffffu, sq, 1) >= (1ull << 31);
  for (int o = 16; o > 0; o >>= 1) {
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
    worst = max(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    wrapped |= __shfl_xor_sync(0xffffffffu, wrapped, o);
  }
  if (t == 0) {
    if (wrapped) atomicOr(&f->wrapped, 1);
    atomicMax(&f->worst, worst);
    atomicAdd(&f->normsq, (unsigned long long)sq);
  }
}

// The 162-point transform of every component of every ring element of v, modulo one limb:
// vhat[leaf][i][k] (component k of ring element i holds coefficients 4m + k).
template <int PI>
__global__ void __launch_bounds__(216) k_v_transform(const int16_t* __restrict__ v, size_t len_ring,
                                                     const DevPrime* __restrict__ D, uint32_t* __restrict__ vhat) {
  // one ring element per CTA, 54 threads per component, the transform in shared memory
  __shared__ uint32_t xs[4][N162];
  const int k = threadIdx.x / 54, t = threadIdx.x - 54 * k;
  const size_t i = blockIdx.x;
  constexpr int32_t q = Pr<PI>::q;
  for (int m = t; m < N162; m += 54) {
    int32_t c = v[i * N648 + 4 * m + k] % q;
    xs[k][m] = (uint32_t)(c < 0 ? c + q : c);
  }
  __syncthreads();
  ntt162_group<PI>(xs[k], t, *D);
  for (int leaf = t; leaf < N162; leaf += 54) vhat[((size_t)leaf * len_ring + i) * 4 + k] = xs[k][leaf];
}

// A v at one leaf (one CTA per leaf): Y_k'(leaf) = sum_i the module product of the key's
// components with v's (the commit's algebra), compared with the folded commitment's slot; with
// `diff`, Y - fc modulo q is written to diff[row][leaf] instead.
template <int PI>
__global__ void __launch_bounds__(256) k_v_mac(const uint32_t* __restrict__ vhat, size_t len_ring,
                                               const int4* __restrict__ Ahat, const DevPrime* __restrict__ D,
                                               int limb, int limbs, const int16_t* __restrict__ fc,
                                               VerifyFlags* __restrict__ f, uint32_t* __restrict__ diff) {
  const int leaf = blockIdx.x;
  long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (size_t i = threadIdx.x; i < len_ring; i += blockDim.x) {
    uint4 w = ((const uint4*)vhat)[(size_t)leaf * len_ring + i];
    int4 lo = __ldg(Ahat + (i * N162 + leaf) * 2), hi = __ldg(Ahat + (i * N162 + leaf) * 2 + 1);
    long long w0 = w.x, w1 = w.y, w2 = w.z, w3 = w.w;
    a0 += lo.x * w0 + hi.x * w3 + hi.y * w2 + hi.z * w1;
    a1 += lo.y * w0 + lo.x * w1 + hi.y * w3 + hi.z * w2;
    a2 += lo.z * w0 + lo.y * w1 + lo.x * w2 + hi.z * w3;
    a3 += lo.w * w0 + lo.z * w1 + lo.y * w2 + lo.x * w3;
  }
  __shared__ long long red[4][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    a3 += __shfl_xor_sync(0xffffffffu, a3, o);
  }
  if (lane == 0) {
    red[0][warp] = a0;
    red[1][warp] = a1;
    red[2][warp] = a2;
    red[3][warp] = a3;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    constexpr long long q = Pr<PI>::q;
    int s = D->leaf_to_pow3[leaf];
    for (int row = 0; row < 4; row++) {
      long long y = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) y += red[row][w];
      y %= q;
      if (y < 0) y += q;
      const int16_t c = fc[(row * limbs + limb) * N162 + s];
      if (diff)
        diff[row * N162 + leaf] = (uint32_t)((y + q - (c < 0 ? c + q : c)) % q);
      else if (center<PI>((uint32_t)y) != c)
        atomicOr(&f->mismatch, 1);
    }
  }
}

// components_mod_2 (crates/pcs/src/eval.rs:205-230): F162 4m + k holds the parities of
// coefficients 4p + k of ring element m, bit p.
__global__ void k_v_parity(const int16_t* __restrict__ v, size_t len_ring, uint64_t* __restrict__ W) {
  size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= len_ring * 4) return;
  size_t m = g >> 2;
  int k = (int)(g & 3);
  uint64_t w[3] = {0, 0, 0};
  for (int p = 0; p < N162; p++)
    if (v[m * N648 + 4 * p + k] & 1) w[p >> 6] |= 1ull << (p & 63);
  W[3 * g] = w[0];
  W[3 * g + 1] = w[1];
  W[3 * g + 2] = w[2];
}

// fold_binary (crates/pcs/src/eval.rs:195-200): sum_j (c_j mod 2) u_j, c_j mod 2 the F162 with
// bits at the challenge's positions (crates/pcs/src/challenge.rs:274-281); out zeroed first.
__global__ void k_fold_binary(const uint64_t* __restrict__ u, const lbg_challenge_d* __restrict__ ch, int r,
                              unsigned long long* __restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t a0 = 0, a1 = 0, a2 = 0;
  if (j < r) {
    F162d c{{0, 0, 0}};
    uint32_t wgt = ch[j].weight > 32 ? 32 : ch[j].weight;
    for (uint32_t t = 0; t < wgt; t++) {
      uint32_t p = ch[j].positions[t];
      if (p < N162) c.w[p >> 6] |= 1ull << (p & 63);
    }
    F162d y = f_mul(c, F162d{{u[3 * j], u[3 * j + 1], u[3 * j + 2]}});
    a0 = y.w[0];
    a1 = y.w[1];
    a2 = y.w[2];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a0 ^= __shfl_xor_sync(0xffffffffu, a0, o);
    a1 ^= __shfl_xor_sync(0xffffffffu, a1, o);
    a2 ^= __shfl_xor_sync(0xffffffffu, a2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicXor(out, (unsigned long long)a0);
    atomicXor(out + 1, (unsigned long long)a1);
    atomicXor(out + 2, (unsigned long long)a2);
  }
}

// =============================================================================================
// Witness generation: keyed BLAKE3 XOF of "labinius/witness" (crates/pcs/src/scheme/witness.rs:66-87)
// =============================================================================================
__device__ __forceinline__ uint32_t rotr32(uint32_t x, int n) { return __funnelshift_r(x, x, n); }
__device__ __forceinline__ void g_mix(uint32_t* s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
  s[a] += s[b] + x;
  s[d] = rotr32(s[d] ^ s[a], 16);
  s[c] += s[d];
  s[b] = rotr32(s[b] ^ s[c], 12);
  s[a] += s[b] + y;
  s[d] = rotr32(s[d] ^ s[a], 8);
  s[c] += s[d];
  s[b] = rotr32(s[b] ^ s[c], 7);
}
__constant__ uint8_t c_b3_sched[7][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8},
    {3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1},
    {10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6},
    {12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4},
    {9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7},
    {11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13},
};

// Output block t of a single-block root node (key words, message words, length, flags).
__device__ __forceinline__ void xof_block(const XofRoot& root, size_t t, uint32_t o[16]) {
  const uint32_t IV[4] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au};
  uint32_t s[16];
  for (int i = 0; i < 8; i++) s[i] = root.cv[i];
  for (int i = 0; i < 4; i++) s[8 + i] = IV[i];
  s[12] = (uint32_t)t;
  s[13] = (uint32_t)((uint64_t)t >> 32);
  s[14] = root.block_len;
  s[15] = root.flags;
  for (int r = 0; r < 7; r++) {
    const uint8_t* w = c_b3_sched[r];
    g_mix(s, 0, 4, 8, 12, root.m[w[0]], root.m[w[1]]);
    g_mix(s, 1, 5, 9, 13, root.m[w[2]], root.m[w[3]]);
    g_mix(s, 2, 6, 10, 14, root.m[w[4]], root.m[w[5]]);
    g_mix(s, 3, 7, 11, 15, root.m[w[6]], root.m[w[7]]);
    g_mix(s, 0, 5, 10, 15, root.m[w[8]], root.m[w[9]]);
    g_mix(s, 1, 6, 11, 12, root.m[w[10]], root.m[w[11]]);
    g_mix(s, 2, 7, 8, 13, root.m[w[12]], root.m[w[13]]);
    g_mix(s, 3, 4, 9, 14, root.m[w[14]], root.m[w[15]]);
  }
  for (int i = 0; i < 8; i++) {
    o[i] = s[i] ^ s[i + 8];
    o[i + 8] = s[i + 8] ^ root.cv[i];
  }
}

__global__ void k_xof_blocks(XofRoot root, size_t nbytes, uint8_t* __restrict__ out) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t * 64 >= nbytes) return;
  uint32_t o[16];
  xof_block(root, t, o);
  size_t base = t * 64;
  for (int i = 0; i < 64; i++)
    if (base + i < nbytes) out[base + i] = (uint8_t)(o[i >> 2] >> (8 * (i & 3)));
}

// A B128 trace from the XOF (16 bytes per element, little-endian), lifted as it is produced:
// block t holds elements 4t .. 4t+3, written as F162 [lo, hi, 0] (crates/pcs/src/fields/scalar.rs:72-74).
// Witness::random's words (crates/pcs/src/scheme/witness.rs:66-87): XOF block t is bytes 64 t .. 64 t +
// 63 of the F162 array, the third limb of every element masked to 34 bits on the way (the word at
// byte 20 of an element keeps its low two bits, the one at byte 16 is bits 0-31 of the limb), and
// the block written as four 16-byte stores (16-byte aligned: W from cudaMalloc, instances at whole
// columns).
__global__ void k_xof_f162(XofRoot root, size_t n, uint64_t* __restrict__ W) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nbytes = 24 * n;
  if (t * 64 >= nbytes) return;
  uint32_t o[16];
  xof_block(root, t, o);
  const int r0 = (int)(t % 3) * 16;  // 64 t mod 24
#pragma unroll
  for (int w = 0; w < 16; w++)
    if ((r0 + 4 * w) % 24 == 20) o[w] &= 3u;
  uint8_t* out = reinterpret_cast<uint8_t*>(W) + t * 64;
  if (t * 64 + 64 <= nbytes) {
#pragma unroll
    for (int q = 0; q < 4; q++)
      reinterpret_cast<uint4*>(out)[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  } else {
    // the last, partial block: whole words (24 n is a multiple of 8)
    for (int w = 0; w < 16 && t * 64 + 4 * w < nbytes; w++) reinterpret_cast<uint32_t*>(out)[w] = o[w];
  }
}

__global__ void k_xof_lifted(XofRoot root, size_t n, uint64_t* __restrict__ W) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t * 4 >= n) return;
  uint32_t o[16];
  xof_block(root, t, o);
  if (4 * t + 4 <= n) {
    // four whole elements, 96 bytes from byte 96 t: six 16-byte stores
    uint4* d = reinterpret_cast<uint4*>(W + 12 * t);
    d[0] = make_uint4(o[0], o[1], o[2], o[3]);
    d[1] = make_uint4(0, 0, o[4], o[5]);
    d[2] = make_uint4(o[6], o[7], 0, 0);
    d[3] = make_uint4(o[8], o[9], o[10], o[11]);
    d[4] = make_uint4(0, 0, o[12], o[13]);
    d[5] = make_uint4(o[14], o[15], 0, 0);
    return;
  }
  for (int k = 0; k < 4; k++) {
    size_t e = 4 * t + k;
    if (e >= n) break;
    W[3 * e] = (uint64_t)o[4 * k] | ((uint64_t)o[4 * k + 1] << 32);
    W[3 * e + 1] = (uint64_t)o[4 * k + 2] | ((uint64_t)o[4 * k + 3] << 32);
    W[3 * e + 2] = 0;
  }
}

__global__ void k_mask_f162(uint64_t* __restrict__ W, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) W[3 * i + 2] &= (1ull << 34) - 1;
}

// Witness::lifted: F162 = [lo, hi, 0] (crates/pcs/src/fields/scalar.rs:72-74).
__global__ void k_lift_b128(const uint64_t* __restrict__ b, size_t n, uint64_t* __restrict__ W) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    W[3 * i] = b[2 * i];
    W[3 * i + 1] = b[2 * i + 1];
    W[3 * i + 2] = 0;
  }
}

// =============================================================================================
// launch wrappers
// =============================================================================================
// The forward transform as persistent CTAs for 16-byte aligned buffers: a CTA loops over groups
// of four ring elements, with the transform's twiddles in shared memory once per CTA, the next
// group's coefficients arriving by cp.async (81 16-byte chunks a ring element) while this group is
// transformed, and the results written back as 16-byte stores. (The same scheme for the inverse
// measured slower than k_ntt648_inv, whose first levels read their nine consecutive coefficients
// straight from global memory.)
constexpr int NTT_TW = 8 + 24 + 72 + 216;  // the radix-3 twiddles of levels 3..6, in table order

template <int PI>
__global__ void __launch_bounds__(81 * NTT_E, 5) k_ntt648_fwd_p(const uint16_t* __restrict__ in, uint16_t* __restrict__ out,
                                                             size_t count, const Ntt648Tables* __restrict__ Tg) {
  constexpr uint32_t q = Pr<PI>::q;
  __shared__ __align__(16) uint16_t sin[2][NTT_E * N648];
  __shared__ __align__(16) uint16_t sout[NTT_E * N648];
  __shared__ uint32_t s[NTT_E][N648];
  __shared__ Twiddle tw[NTT_TW];  // f3 at 0, f4 at 8, f5 at 32, f6 at 104
  const Ntt648Tables& T = *Tg;
  const int tid = threadIdx.x;
  for (int x = tid; x < NTT_TW; x += blockDim.x)
    tw[x] = x < 8 ? T.f3[x] : x < 32 ? T.f4[x - 8] : x < 104 ? T.f5[x - 32] : T.f6[x - 104];
  const uint32_t om = T.omega, oms = T.omega_s, z6 = T.z6, z6s = T.z6s;
  uint32_t f1[2][2], f2[4][2];
#pragma unroll
  for (int a = 0; a < 2; a++) f1[a][0] = T.f1[a][0], f1[a][1] = T.f1[a][1];
#pragma unroll
  for (int a = 0; a < 4; a++) f2[a][0] = T.f2[a][0], f2[a][1] = T.f2[a][1];
  const int ea = tid / 81, ra = tid - 81 * ea;                         // phase A: element, residue
  const int eb = tid / 72, jb = tid - 72 * eb, kb = jb / 9, tb = jb - 9 * kb;  // phases B, C
  const size_t groups = (count + NTT_E - 1) / NTT_E;
  auto stage = [&](size_t g, int b) {
    const size_t e0 = g * NTT_E;
    const int chunks = (int)min((size_t)NTT_E, count - e0) * (N648 / 8);
    if (tid < chunks) cp_async16(&sin[b][8 * tid], in + e0 * N648 + 8 * tid);
  };
  if ((size_t)blockIdx.x < groups) stage(blockIdx.x, 0);
  cp_async_commit();
  int b = 0;
  for (size_t g = blockIdx.x; g < groups; g += gridDim.x, b ^= 1) {
    const size_t e0 = g * NTT_E;
    const int nel = (int)min((size_t)NTT_E, count - e0);
    if (g + gridDim.x < groups) stage(g + gridDim.x, b ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (ea < nel) {  // level 0 and the radix-2 levels 1, 2
      uint32_t x[8];
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = sin[b][ea * N648 + ra + 81 * k];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint32_t t = mul_shoup(x[k + 4], z6, z6s, q);
        uint32_t a0 = x[k];
        x[k] = a0 + t;
        x[k + 4] = a0 + x[k + 4] + 2 * q - t;
      }
#pragma unroll
      for (int sr = 0; sr < 2; sr++)
#pragma unroll
        for (int k = 0; k < 2; k++) {
          uint32_t t = mul_shoup(x[4 * sr + k + 2], f1[sr][0], f1[sr][1], q);
          uint32_t a0 = x[4 * sr + k];
          x[4 * sr + k] = a0 + t;
          x[4 * sr + k + 2] = a0 + 2 * q - t;
        }
#pragma unroll
      for (int sr = 0; sr < 4; sr++) {
        uint32_t t = mul_shoup(x[2 * sr + 1], f2[sr][0], f2[sr][1], q);
        uint32_t a0 = x[2 * sr];
        x[2 * sr] = a0 + t;
        x[2 * sr + 1] = a0 + 2 * q - t;
      }
#pragma unroll
      for (int k = 0; k < 8; k++) s[ea][ra + 81 * k] = x[k];
    }
    __syncthreads();
    if (tid < 72 * NTT_E && eb < nel) {  // radix-3 levels 3, 4
      uint32_t y[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) y[a][c] = s[eb][81 * kb + tb + 9 * a + 27 * c];
      const Twiddle t3 = tw[kb];
#pragma unroll
      for (int a = 0; a < 3; a++) bfly3<PI>(y[a][0], y[a][1], y[a][2], t3, om, oms);
#pragma unroll
      for (int c = 0; c < 3; c++) bfly3<PI>(y[0][c], y[1][c], y[2][c], tw[8 + 3 * kb + c], om, oms);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) s[eb][81 * kb + tb + 9 * a + 27 * c] = y[a][c];
    }
    __syncthreads();
    if (tid < 72 * NTT_E && eb < nel) {  // radix-3 levels 5, 6, reduced to [0, q)
      const int gg = jb;
      uint32_t z[3][3];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) z[c][d] = s[eb][9 * gg + c + 3 * d];
      const Twiddle t5 = tw[32 + gg];
#pragma unroll
      for (int c = 0; c < 3; c++) bfly3<PI>(z[c][0], z[c][1], z[c][2], t5, om, oms);
#pragma unroll
      for (int d = 0; d < 3; d++) bfly3<PI>(z[0][d], z[1][d], z[2][d], tw[104 + 3 * gg + d], om, oms);
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) sout[eb * N648 + 9 * gg + 3 * d + c] = (uint16_t)red_full<PI>(z[c][d]);
    }
    __syncthreads();
    if (tid < nel * (N648 / 8))
      *reinterpret_cast<uint4*>(out + e0 * N648 + 8 * tid) = *reinterpret_cast<const uint4*>(&sout[8 * tid]);
  }
}

#define LBG_DISPATCH(pi, CALL)                 \
  switch (pi) {                                \
    case 0: { constexpr int P = 0; CALL; } break; \
    case 1: { constexpr int P = 1; CALL; } break; \
    case 2: { constexpr int P = 2; CALL; } break; \
    case 3: { constexpr int P = 3; CALL; } break; \
    case 4: { constexpr int P = 4; CALL; } break; \
    case 5: { constexpr int P = 5; CALL; } break; \
    case 6: { constexpr int P = 6; CALL; } break; \
    default: return cudaErrorInvalidValue;     \
  }

static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

cudaError_t upload_hot(int pi, const HotPrime& h) {
  cudaError_t e = cudaMemcpyToSymbol(c_hot, &h, sizeof(HotPrime), sizeof(HotPrime) * pi, cudaMemcpyHostToDevice);
  // landed before any stream's kernels read it (the copy runs on the legacy default stream)
  return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

cudaError_t launch_key_expand(const uint64_t* jumps, uint64_t state0, uint32_t q, int nb, int16_t* A,
                              cudaStream_t st) {
  size_t n = (size_t)nb * N648;
  k_key_expand<<<blocks_for(n, 128), 128, 0, st>>>(jumps, state0, q, nb, A);
  return cudaGetLastError();
}

cudaError_t launch_key_components(int pi, const int16_t* A, const DevPrime* D, int len_ring, int4* Ahat,
                                  cudaStream_t st) {
  size_t n = (size_t)len_ring * N162;
  LBG_DISPATCH(pi, (k_key_components<P><<<blocks_for(n, 128), 128, 0, st>>>(A, D, len_ring, Ahat)));
  return cudaGetLastError();
}

size_t commit_smem_bytes() { return LUT_BYTES + CT * WROW * 8 + RT * N162 * CT * 4 * 2 + AT_BYTES; }

// The commit's transforms run on the tensor cores (k_commit_tc) unless LBG_COMMIT_KERNEL=scalar
// selects the CUDA cores (k_commit) (both are exact; the switch is for comparing them). The commit
// that keeps the base limb's transform for the fold always runs the CUDA-core kernel.
bool commit_tc_enabled() {
  static const bool on = [] {
    const char* e = getenv("LBG_COMMIT_KERNEL");
    return !(e && std::string(e) == "scalar");
  }();
  return on;
}

// Compute warps of the tensor-core commit: the calling thread's choice (set_commit_warps, the batch
// autotuner's), else 12 unless LBG_COMMIT_WARPS=16 (both exact).
static thread_local int t_commit_warps = 0;
void set_commit_warps(int warps) { t_commit_warps = (warps == 12 || warps == 16) ? warps : 0; }
static int commit_tc_warps() {
  static const int w = [] {
    const char* e = getenv("LBG_COMMIT_WARPS");
    return (e && std::string(e) == "16") ? 16 : 12;
  }();
  return t_commit_warps ? t_commit_warps : w;
}

int commit_blocks_per_sm(int pi) {
  int n = 0;
  const bool tcm = commit_tc_enabled();
  size_t smem = tcm ? (size_t)TCC_SMEM : commit_smem_bytes();
  cudaError_t e = cudaErrorInvalidValue;
  switch (pi) {
#define LBG_OCC(I)                                                                                        \
  case I:                                                                                                 \
    if (tcm) {                                                                                            \
      cudaFuncSetAttribute(k_commit_tc<I, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_commit_tc<I, 12>, TCC_THREADS, smem);       \
    } else {                                                                                              \
      cudaFuncSetAttribute(k_commit<I, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_commit<I, false>, 256, smem);               \
    }                                                                                                     \
    break;
    LBG_OCC(0) LBG_OCC(1) LBG_OCC(2) LBG_OCC(3) LBG_OCC(4) LBG_OCC(5) LBG_OCC(6)
#undef LBG_OCC
  }
  return (e == cudaSuccess && n > 0) ? n : 1;
}
int commit_cols_per_cta() { return commit_tc_enabled() ? TCC_CT : CT; }
// Chunks are whole steps of the scalar kernel (RT ring elements); the tensor-core kernel takes any.
int commit_ring_per_step() { return RT; }

int tc_timeout_take() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_timeout, sizeof(int)) != cudaSuccess) return -1;
  if (v) {
    int z = 0;
    cudaMemcpyToSymbol(g_tc_timeout, &z, sizeof(int));
  }
  return v;
}

static int sm_count() {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

// The most CTAs (one per SM) the persistent tensor-core kernels launched from this host thread
// take; 0: every SM. A server gives its large requests' slot fewer than all SMs so that a slot of
// small requests finds SMs free instead of waiting for a whole persistent launch to end.
static thread_local int t_persistent_cap = 0;
void set_persistent_cap(int ctas) { t_persistent_cap = ctas > 0 ? ctas : 0; }
static int persistent_ctas() {
  const int n = sm_count();
  return t_persistent_cap > 0 && t_persistent_cap < n ? t_persistent_cap : n;
}

cudaError_t launch_commit(int pi, const uint64_t* W, size_t wdim, const int4* Ahat, const DevPrime* D, int cols,
                          int len_ring, int chunk, int nchunks, int32_t* partial, cudaStream_t st, uint16_t* keep,
                          const uint8_t* tcb) {
  if (keep) {
    dim3 grid((cols + CT - 1) / CT, nchunks);
    size_t smem = commit_smem_bytes();
    LBG_DISPATCH(pi, ({
                   cudaFuncSetAttribute(k_commit<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                   k_commit<P, true><<<grid, 256, smem, st>>>(W, wdim, Ahat, D, cols, len_ring, chunk, partial, keep);
                 }));
  } else if (tcb && commit_tc_enabled()) {
    // persistent: one CTA per SM (at most one per work item) over the column tiles x chunks
    const long items = (long)((cols + TCC_CT - 1) / TCC_CT) * nchunks;
    dim3 grid((unsigned)std::max<long>(1, std::min<long>(items, persistent_ctas())));
    LBG_DISPATCH(pi, ({
                   if (commit_tc_warps() == 16) {
                     cudaFuncSetAttribute(k_commit_tc<P, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, TCC_SMEM);
                     k_commit_tc<P, 16><<<grid, TccShape<16>::THREADS, TCC_SMEM, st>>>(W, wdim, Ahat, tcb, cols,
                                                                                      len_ring, chunk, nchunks, partial);
                   } else {
                     cudaFuncSetAttribute(k_commit_tc<P, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, TCC_SMEM);
                     k_commit_tc<P, 12><<<grid, TCC_THREADS, TCC_SMEM, st>>>(W, wdim, Ahat, tcb, cols, len_ring,
                                                                             chunk, nchunks, partial);
                   }
                 }));
  } else {
    dim3 grid((cols + CT - 1) / CT, nchunks);
    size_t smem = commit_smem_bytes();
    LBG_DISPATCH(pi, ({
                   cudaFuncSetAttribute(k_commit<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                   k_commit<P, false><<<grid, 256, smem, st>>>(W, wdim, Ahat, D, cols, len_ring, chunk, partial,
                                                               nullptr);
                 }));
  }
  return cudaGetLastError();
}

cudaError_t launch_commit_finish(int pi, const int32_t* partial, int nchunks, int cols, const DevPrime* D,
                                 int limb, int limbs, int16_t* C, cudaStream_t st) {
  size_t n = (size_t)cols * N162;
  LBG_DISPATCH(pi, (k_commit_finish<P><<<blocks_for(n, 128), 128, 0, st>>>(partial, nchunks, cols, D, limb, limbs, C)));
  return cudaGetLastError();
}

cudaError_t launch_challenge_slots(int pi, const lbg_challenge_d* ch, int r, const DevPrime* D, uint32_t* chat,
                                   cudaStream_t st) {
  size_t n = (size_t)r * N162;
  LBG_DISPATCH(pi, (k_challenge_slots<P><<<blocks_for(n, 128), 128, 0, st>>>(ch, r, D, chat)));
  return cudaGetLastError();
}

size_t fold_smem_bytes() { return LUT_BYTES + (size_t)FJ * N162 * FP * 2 + FJ * N162 * 4; }
int fold_positions_per_cta() { return FP; }
int fold_cols_per_step() { return FJ; }

int fold_blocks_per_sm(int pi) {
  int n = 0;
  size_t smem = fold_smem_bytes();
  cudaError_t e = cudaErrorInvalidValue;
  switch (pi) {
#define LBG_OCC(I)                                                                                      \
  case I:                                                                                               \
    cudaFuncSetAttribute(k_fold<I, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fold<I, false>, 256, smem);                 \
    break;
    LBG_OCC(0) LBG_OCC(1) LBG_OCC(2) LBG_OCC(3) LBG_OCC(4) LBG_OCC(5) LBG_OCC(6)
#undef LBG_OCC
  }
  return (e == cudaSuccess && n > 0) ? n : 1;
}

// The fold's transforms run on the tensor cores (k_fold_tc) unless LBG_FOLD_KERNEL=scalar selects
// the CUDA-core kernel (k_fold) (both exact). The one-pass mode without scratch (vhat null) and the fold
// from the kept transform always run on the CUDA cores.
bool fold_tc_enabled() {
  static const bool on = [] {
    const char* e = getenv("LBG_FOLD_KERNEL");
    return !(e && std::string(e) == "scalar");
  }();
  return on;
}
int fold_tc_positions_per_cta() { return TCF_ROWS; }

// The single prover's fold takes k_fold_gm (the challenge in the multiply's operand) unless
// LBG_FOLD_KERNEL=tc (k_fold_tc) or scalar (k_fold) selects another (all exact).
bool fold_gm_enabled() {
  static const bool on = [] {
    const char* e = getenv("LBG_FOLD_KERNEL");
    return !(e && (std::string(e) == "tc" || std::string(e) == "scalar"));
  }();
  return on;
}
size_t fold_gm_operand_bytes(size_t cols) { return cols * (size_t)TC_B_BYTES; }

cudaError_t launch_fold_gm(int pi, const uint64_t* W, size_t wdim, int cols, int cols_per_split, const uint32_t* chat,
                           const uint8_t* tcb, uint8_t* G, const DevPrime* D, uint32_t* vhat, int16_t* v,
                           cudaStream_t st, int instances, const int* split_inst) {
  if (cols <= 0 || cols_per_split <= 0) return cudaErrorInvalidValue;
  // one instance: splits of at most 512 columns; instances laid out one after another: the caller's
  // splits (split_inst maps each to its instance; each at most 512 columns)
  if (!split_inst) cols_per_split = std::min(cols_per_split, GM_MAX_COLS_PER_SPLIT);
  if (cols_per_split > GM_MAX_COLS_PER_SPLIT) return cudaErrorInvalidValue;
  const int splits = (cols + cols_per_split - 1) / cols_per_split;
  const long items = (long)((wdim + TCF_ROWS - 1) / TCF_ROWS) * splits;
  dim3 grid((unsigned)std::max<long>(1, std::min<long>(items, persistent_ctas())));
  const size_t positions = wdim * (size_t)instances;
  cudaError_t e = cudaMemsetAsync(vhat, 0, positions * N162 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  const size_t nop = (size_t)cols * TC_LEAVES * (TC_KBYTES / 16);
  LBG_DISPATCH(pi, ({
                 k_fold_operand<P><<<blocks_for(nop, 256), 256, 0, st>>>(chat, cols, tcb, G);
                 cudaFuncSetAttribute(k_fold_gm<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, GM_SMEM);
                 k_fold_gm<P><<<grid, GM_THREADS, GM_SMEM, st>>>(W, wdim, cols, cols_per_split, G, vhat, split_inst);
                 k_fold_finish_t<P><<<blocks_for(positions, 4), 216, 0, st>>>(vhat, wdim, positions, D, v);
               }));
  return cudaGetLastError();
}

cudaError_t launch_fold(int pi, const uint64_t* W, size_t wdim, int cols, int cols_per_split, const uint32_t* chat,
                        const DevPrime* D, uint32_t* vhat, int16_t* v, cudaStream_t st, int instances,
                        const int* split_inst, const uint8_t* tcb) {
  if (vhat && tcb && fold_tc_enabled()) {
    int splits = (cols + cols_per_split - 1) / cols_per_split;
    if (splits < 1 || splits > 65535) return cudaErrorInvalidValue;
    const long items = (long)((wdim + TCF_ROWS - 1) / TCF_ROWS) * splits;
    dim3 grid((unsigned)std::max<long>(1, std::min<long>(items, persistent_ctas())));  // persistent, one CTA per SM
    size_t positions = wdim * (size_t)instances;
    cudaError_t e = cudaMemsetAsync(vhat, 0, positions * N162 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    LBG_DISPATCH(pi, ({
                   cudaFuncSetAttribute(k_fold_tc<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, TCF_SMEM);
                   k_fold_tc<P><<<grid, TCF_THREADS, TCF_SMEM, st>>>(W, wdim, cols, cols_per_split, chat, tcb, vhat,
                                                                     split_inst);
                   k_fold_finish_t<P><<<blocks_for(positions, 4), 216, 0, st>>>(vhat, wdim, positions, D, v);
                 }));
    return cudaGetLastError();
  }
  size_t smem = fold_smem_bytes();
  if (!vhat) {  // direct mode: one split, no scratch beyond chat
    dim3 grid(blocks_for(wdim, FP), 1);
    LBG_DISPATCH(pi, ({
                   cudaFuncSetAttribute(k_fold<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                   k_fold<P, true><<<grid, 256, smem, st>>>(W, wdim, cols, cols, chat, D, nullptr, v, nullptr);
                 }));
    return cudaGetLastError();
  }
  int splits = (cols + cols_per_split - 1) / cols_per_split;
  if (splits < 1 || splits > 65535) return cudaErrorInvalidValue;
  dim3 grid(blocks_for(wdim, FP), splits);
  size_t positions = wdim * (size_t)instances;  // instances laid out one after another
  cudaError_t e = cudaMemsetAsync(vhat, 0, positions * N162 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  LBG_DISPATCH(pi, ({
                 cudaFuncSetAttribute(k_fold<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                 k_fold<P, false><<<grid, 256, smem, st>>>(W, wdim, cols, cols_per_split, chat, D, vhat, nullptr,
                                                          split_inst);
                 k_fold_finish<P><<<blocks_for(positions, 4), 216, 0, st>>>(vhat, positions, D, v);
               }));
  return cudaGetLastError();
}

cudaError_t launch_fold_kept(int pi, const uint16_t* keep, size_t wdim, int cols, int cols_per_split,
                             const uint32_t* chat, const DevPrime* D, uint32_t* vhat, int16_t* v, cudaStream_t st,
                             int instances, const int* split_inst) {
  size_t smem = (size_t)FJ * 2 * N162 * 16 * 2;
  if (!vhat) {
    dim3 grid(blocks_for(wdim, FP), 1);
    LBG_DISPATCH(pi, ({
                   cudaFuncSetAttribute(k_fold_kept<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                   k_fold_kept<P, true><<<grid, 256, smem, st>>>(keep, wdim, cols, cols, chat, D, nullptr, v, nullptr);
                 }));
    return cudaGetLastError();
  }
  int splits = (cols + cols_per_split - 1) / cols_per_split;
  if (splits < 1 || splits > 65535) return cudaErrorInvalidValue;
  dim3 grid(blocks_for(wdim, FP), splits);
  cudaError_t e = cudaMemsetAsync(vhat, 0, wdim * (size_t)instances * N162 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  LBG_DISPATCH(pi, ({
                 cudaFuncSetAttribute(k_fold_kept<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                 k_fold_kept<P, false><<<grid, 256, smem, st>>>(keep, wdim, cols, cols_per_split, chat, D, vhat,
                                                                nullptr, split_inst);
               }));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  LBG_DISPATCH(pi, (k_fold_finish<P><<<blocks_for(wdim * instances, 4), 216, 0, st>>>(vhat, wdim * instances, D, v)));
  return cudaGetLastError();
}

cudaError_t launch_fold_commitment(int pi, const int16_t* C, int cols, int limb, int limbs, const uint32_t* chat,
                                   const DevPrime* D, int16_t* out, cudaStream_t st) {
  LBG_DISPATCH(pi, (k_fold_commitment<P><<<dim3((N162 + 31) / 32, 4), 1024, 0, st>>>(C, cols, limb, limbs, chat, D, out)));
  return cudaGetLastError();
}

cudaError_t launch_column_residues(int pi, const int16_t* C, int cols, int limb, int limbs, const DevPrime* D,
                                   uint16_t* res, cudaStream_t st) {
  if (cols <= 0) return cudaSuccess;
  LBG_DISPATCH(pi, (k_column_residues<P><<<cols, 216, 0, st>>>(C, cols, limb, limbs, D, res)));
  return cudaGetLastError();
}

cudaError_t launch_recursion_residues(const uint16_t* res, int cols, size_t polys, uint32_t q, int16_t* out,
                                      cudaStream_t st) {
  const size_t n = 4 * polys * 64;
  if (n == 0) return cudaSuccess;
  k_recursion_residues<<<blocks_for(n, 256), 256, 0, st>>>(res, cols, polys, (int32_t)q, out);
  return cudaGetLastError();
}

cudaError_t launch_left_expansion(const uint64_t* u, int cols, size_t rank, int16_t* out, cudaStream_t st) {
  const size_t n = rank * 64;
  if (n == 0) return cudaSuccess;
  k_left_expansion<<<blocks_for(n, 256), 256, 0, st>>>(u, cols, rank, out);
  return cudaGetLastError();
}

cudaError_t launch_garner(const uint16_t* res, size_t count, int limbs, const GarnerConsts& g, uint16_t* top,
                          uint16_t* digits, cudaStream_t st) {
  k_garner<<<blocks_for(count, 256), 256, 0, st>>>(res, count, limbs, g, top, digits);
  return cudaGetLastError();
}

cudaError_t launch_eq_table(const uint64_t* p, int n, size_t count, uint64_t* eq, cudaStream_t st, int instances) {
  k_eq_table<<<blocks_for(count * instances, 128), 128, 0, st>>>(p, n, count, instances, eq);
  return cudaGetLastError();
}

int row_eval_tile_cols() { return RE_COLS; }

cudaError_t launch_row_eval(const uint64_t* W, size_t wdim, int cols, const uint64_t* eq, uint64_t* u,
                            cudaStream_t st, const int4* tiles, int ntiles) {
  cudaError_t e = cudaMemsetAsync(u, 0, (size_t)cols * 24, st);
  if (e != cudaSuccess) return e;
  if (!tiles) ntiles = (cols + RE_COLS - 1) / RE_COLS;
  int G = (int)(wdim >> 3);
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // enough CTAs for about eight per SM, each with at least 8 groups of rows
  int splits = std::max(1, std::min(G / 8, (8 * sms + ntiles - 1) / ntiles));
  int gps = (G + splits - 1) / splits;
  splits = (G + gps - 1) / gps;
  k_row_eval<<<dim3(ntiles, splits), RE_THREADS, 0, st>>>(W, (int)wdim, cols, eq, tiles, gps,
                                                           (unsigned long long*)u);
  return cudaGetLastError();
}

cudaError_t launch_claim(const uint64_t* u, int cols, const uint64_t* p1, int n, uint64_t* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, 24, st);
  if (e != cudaSuccess) return e;
  k_claim<<<blocks_for(cols, 64), 64, 0, st>>>(u, cols, p1, n, (unsigned long long*)out);
  return cudaGetLastError();
}

cudaError_t launch_claims(const RoundInst* d_inst, const int* col_inst, const uint64_t* u, int total_cols,
                          const uint64_t* p1, int count, uint64_t* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, (size_t)count * 24, st);
  if (e != cudaSuccess) return e;
  k_claims<<<blocks_for(total_cols, 128), 128, 0, st>>>(d_inst, col_inst, u, total_cols, p1,
                                                         (unsigned long long*)out);
  return cudaGetLastError();
}

cudaError_t launch_ntt648(int pi, bool inverse, const uint16_t* in, uint16_t* out, size_t count,
                          const Ntt648Tables* T, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  unsigned grid = (unsigned)((count + NTT_E - 1) / NTT_E);
  // the forward transform of 16-byte aligned buffers takes the persistent kernel: as many CTAs as
  // fit on the SMs at once loop over the groups
  const bool aligned = (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto persistent_grid = [&](const void* kernel) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, 81 * NTT_E, 0) != cudaSuccess || nb < 1) nb = 1;
    return std::min<unsigned>(grid, (unsigned)(sms * nb));
  };
  switch (pi) {
#define LBG_NTT648(P)                                                                                       \
  case P:                                                                                                   \
    if (aligned && !inverse)                                                                                \
      k_ntt648_fwd_p<P><<<persistent_grid((const void*)k_ntt648_fwd_p<P>), 81 * NTT_E, 0, st>>>(in, out, count, T); \
    else if (inverse)                                                                                       \
      k_ntt648_inv<P><<<grid, 81 * NTT_E, 0, st>>>(in, out, count, T);                                     \
    else                                                                                                    \
      k_ntt648_fwd<P><<<grid, 81 * NTT_E, 0, st>>>(in, out, count, T);                                     \
    break;
    LBG_NTT648(1)
    LBG_NTT648(3)
    LBG_NTT648(5)
    LBG_NTT648(6)
#undef LBG_NTT648
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_v_norm(const int16_t* v, size_t len_ring, VerifyFlags* f, cudaStream_t st) {
  k_v_norm<<<blocks_for(len_ring, 8), 256, 0, st>>>(v, len_ring, f);
  return cudaGetLastError();
}

cudaError_t launch_v_limb(int pi, const int16_t* v, size_t len_ring, const DevPrime* D, uint32_t* vhat,
                          const int4* Ahat, int limb, int limbs, const int16_t* fc, VerifyFlags* f, cudaStream_t st,
                          uint32_t* diff) {
  if (len_ring > 0) LBG_DISPATCH(pi, (k_v_transform<P><<<(unsigned)len_ring, 216, 0, st>>>(v, len_ring, D, vhat)));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  LBG_DISPATCH(pi, (k_v_mac<P><<<N162, 256, 0, st>>>(vhat, len_ring, Ahat, D, limb, limbs, fc, f, diff)));
  return cudaGetLastError();
}

cudaError_t launch_bd_columns(int pi, const uint16_t* top, const uint16_t* digits, int cols, int limb,
                              const GarnerConsts& g, int limbs, const DevPrime* D, int16_t* C, cudaStream_t st) {
  if (cols > 0) LBG_DISPATCH(pi, (k_bd_columns<P><<<cols, 216, 0, st>>>(top, digits, cols, limb, g, limbs, D, C)));
  return cudaGetLastError();
}

cudaError_t launch_bd_inverse(int pi, const uint32_t* diff, const DevPrime* D, uint32_t* res, cudaStream_t st) {
  LBG_DISPATCH(pi, (k_bd_inverse<P><<<1, 4, 0, st>>>(diff, D, res)));
  return cudaGetLastError();
}

cudaError_t launch_bd_normsq(const uint32_t* res, int limbs, const GarnerConsts& g, unsigned long long* out,
                             cudaStream_t st) {
  k_bd_normsq<<<1, 1024, 0, st>>>(res, limbs, g, out);
  return cudaGetLastError();
}

cudaError_t launch_v_parity(const int16_t* v, size_t len_ring, uint64_t* W, cudaStream_t st) {
  k_v_parity<<<blocks_for(len_ring * 4, 128), 128, 0, st>>>(v, len_ring, W);
  return cudaGetLastError();
}

cudaError_t launch_fold_binary(const uint64_t* u, const lbg_challenge_d* ch, int r, uint64_t* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, 24, st);
  if (e != cudaSuccess) return e;
  k_fold_binary<<<blocks_for(r, 128), 128, 0, st>>>(u, ch, r, (unsigned long long*)out);
  return cudaGetLastError();
}

cudaError_t launch_xof(const XofRoot& root, size_t nbytes, uint8_t* out, cudaStream_t st) {
  size_t blocks = (nbytes + 63) / 64;
  k_xof_blocks<<<blocks_for(blocks, 128), 128, 0, st>>>(root, nbytes, out);
  return cudaGetLastError();
}

cudaError_t launch_xof_f162(const XofRoot& root, size_t n, uint64_t* W, cudaStream_t st) {
  size_t blocks = (24 * n + 63) / 64;
  k_xof_f162<<<blocks_for(blocks, 128), 128, 0, st>>>(root, n, W);
  return cudaGetLastError();
}

cudaError_t launch_xof_lifted(const XofRoot& root, size_t n, uint64_t* W, cudaStream_t st) {
  size_t blocks = (n + 3) / 4;
  k_xof_lifted<<<blocks_for(blocks, 128), 128, 0, st>>>(root, n, W);
  return cudaGetLastError();
}

cudaError_t launch_mask_f162(uint64_t* W, size_t n, cudaStream_t st) {
  k_mask_f162<<<blocks_for(n, 256), 256, 0, st>>>(W, n);
  return cudaGetLastError();
}

cudaError_t launch_lift_b128(const uint64_t* b, size_t n, uint64_t* W, cudaStream_t st) {
  k_lift_b128<<<blocks_for(n, 256), 256, 0, st>>>(b, n, W);
  return cudaGetLastError();
}

}  // namespace lbg
