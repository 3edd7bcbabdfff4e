// Batched rounds: many independent witnesses under one key, every stage one launch over all of
// them, stages replayed as CUDA graphs, grid schedule autotuned per batch shape.
//
// All instances share the public parameters' key, so they share its column length (wdim F162)
// and moduli; they differ in their column counts (2^column_log_len_i). Instance i's columns follow
// instance i-1's in one device witness buffer, which makes the batched commit the single-instance
// commit kernel over the concatenated columns (a column's commitment depends on that column and
// the key only, crates/pcs/src/key.rs:174-191), and the batched fold the single-instance fold with
// every column split mapped to its instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "error.h"
#include "handles.h"
#include "launch.h"
#include "ring_tables.h"
#include "switch.h"
#include "transcript.h"
#include "transcript_dev.h"

using namespace lbg;

namespace {
int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}
}  // namespace

#define LBG_BCU(x)                                                                      \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) return fail(LBG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct lbg_batch {
  const lbg_pp* pp = nullptr;
  int count = 0;
  std::vector<uint32_t> col_log;
  std::vector<size_t> col_off;  // first column of each instance, plus the total at the end
  size_t total_cols = 0;
  size_t wdim = 0, len_ring = 0;
  int min_col_log = 0;
  size_t cap_cols = 0, cap_instances = 0;
  cudaStream_t stream = nullptr;
  uint64_t* d_w = nullptr;        // [total_cols * wdim][3]
  int* d_col_inst = nullptr;      // [total_cols]
  int4* d_row_tiles = nullptr;    // row-evaluation tiles: (first column, columns, instance)
  int n_row_tiles = 0;
  int* d_split_inst = nullptr;    // [total_cols] (at most one split per column)
  int chunk = 0, nchunks = 0, fold_per = 0;
  int32_t* d_partial = nullptr;   // [max_chunks][total_cols][162][4]
  int max_chunks = 0;
  int16_t* d_C = nullptr;         // [total_cols][4][limbs][162]
  uint16_t* d_keep = nullptr;     // the base limb's kept transform [cap_cols][162][wdim] (allocated on demand)
  bool keep = false;              // the commit keeps it and the fold reads it
  uint16_t* d_res = nullptr;      // [limbs][total_cols*648]
  uint16_t* d_top = nullptr;
  uint16_t* d_digits = nullptr;
  uint64_t* d_p0 = nullptr;       // [count][row_log][3]
  uint64_t* d_p1 = nullptr;       // [count][32][3]
  uint64_t* d_eq = nullptr;       // [count][wdim][3]
  uint64_t* d_u = nullptr;        // [total_cols][3]
  uint64_t* d_claim = nullptr;    // [count][3]
  lbg_challenge_d* d_ch = nullptr;
  uint32_t* d_chat = nullptr;     // [total_cols][162]
  uint32_t* d_vhat = nullptr;     // [count][wdim][162]
  uint8_t* d_gm = nullptr;        // the fold's per-column tensor-core operands (k_fold_gm)
  int16_t* d_v = nullptr;         // [count][len_ring][648]
  bool graphs = false;
  int sm_cap = 0;                 // CTAs of the persistent commit and fold launches (0: one per SM)
  int commit_warps = 0;           // the tensor-core commit's compute warps (0: the default; autotuned)
  cudaGraphExec_t g_commit = nullptr, g_fold = nullptr, g_round = nullptr;
  uint64_t launches = 0;
  // the round on the device: per-instance transcripts, planned once per layout and domain
  bool plan_ok = false;
  std::string plan_domain;
  AbsorbPlan ab_commit, ab_u;
  SamplerTables sampler;
  HasherState* d_prefix = nullptr;  // [cap_instances]: each transcript up to the commitment's bytes
  HasherState* d_states = nullptr;  // [cap_instances]: the transcripts during the round
  RoundInst* d_inst = nullptr;      // [cap_instances]
  uint32_t* d_oldcv = nullptr;      // [cap_instances][8]
  uint8_t* d_stage = nullptr;
  size_t stage_cap = 0;
  uint32_t* d_cvs = nullptr;
  size_t cvs_cap = 0;
  uint8_t* d_packed = nullptr;      // bit-dropped commitments as absorbed
  size_t packed_cap = 0;
  std::vector<uint64_t> packed_off, packed_len;
  PackDropped pack{};
  // switch instances: lifted B128 traces opened through the cross-field switch
  std::vector<uint8_t> sw_flag;     // [count]
  std::vector<SwInst> sw_h;         // host copies of the device table, in instance order
  SwInst* d_sw_inst = nullptr;
  size_t sw_inst_cap = 0;
  SwSmall* d_sw_small = nullptr;
  size_t sw_small_cap = 0;
  uint8_t* d_sw_scratch = nullptr;
  size_t sw_scratch_cap = 0;
  uint64_t* d_sw_r = nullptr;       // the statements' r_hi
  size_t sw_r_cap = 0;
};

static void free_graphs(lbg_batch* b) {
  if (b->g_commit) cudaGraphExecDestroy(b->g_commit);
  if (b->g_fold) cudaGraphExecDestroy(b->g_fold);
  if (b->g_round) cudaGraphExecDestroy(b->g_round);
  b->g_commit = b->g_fold = b->g_round = nullptr;
}

// The device work of each stage, enqueued on the batch's stream (also what the graphs capture).
// Batches of at most 32768 columns fold with the challenges in the tensor-core operand (k_fold_gm:
// 67.5 KB of operand a column, 2.2 GB at the limit); wider ones weight the transforms on the CUDA
// cores (k_fold_tc).
static bool batch_fold_gm(size_t max_cols) { return fold_gm_enabled() && max_cols <= 32768; }

// The batch's cap on the persistent kernels' CTAs, for the launches enqueued in its scope.
struct CapScope {
  explicit CapScope(int ctas, int warps = 0) {
    set_persistent_cap(ctas);
    set_commit_warps(warps);
  }
  ~CapScope() {
    set_persistent_cap(0);
    set_commit_warps(0);
  }
};

static cudaError_t enqueue_commit(lbg_batch* b) {
  CapScope cap(b->sm_cap, b->commit_warps);
  const lbg_pp* pp = b->pp;
  int L = pp->limbs, cols = (int)b->total_cols;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < L && e == cudaSuccess; k++) {
    e = launch_commit(pp->pidx[k], b->d_w, b->wdim, pp->d_Ahat + (size_t)k * pp->len_ring * N162 * 2, pp->d_prime[k],
                      cols, (int)b->len_ring, b->chunk, b->nchunks, b->d_partial, b->stream,
                      k == 0 && b->keep ? b->d_keep : nullptr, pp->d_tcb[k]);
    if (e == cudaSuccess)
      e = launch_commit_finish(pp->pidx[k], b->d_partial, b->nchunks, cols, pp->d_prime[k], k, L, b->d_C, b->stream);
  }
  b->launches += 2 * L;
  if (e == cudaSuccess && pp->params.opening == LBG_OPENING_BIT_DROPPED) {
    size_t count = b->total_cols * N648;
    for (int k = 0; k < L && e == cudaSuccess; k++)
      e = launch_column_residues(pp->pidx[k], b->d_C, cols, k, L, pp->d_prime[k], b->d_res + (size_t)k * count,
                                 b->stream);
    GarnerConsts g;
    std::memset(&g, 0, sizeof(g));
    for (int k = 0; k < L; k++) {
      g.q[k] = pp->primes[k];
      for (int m = 0; m < k; m++) g.inv[k][m] = (uint32_t)inv_mod(pp->primes[m], pp->primes[k]);
    }
    g.dropped_bits = pp->params.dropped_bits;
    if (e == cudaSuccess) e = launch_garner(b->d_res, count, L, g, b->d_top, b->d_digits, b->stream);
    b->launches += L + 1;
  }
  return e;
}

static cudaError_t enqueue_fold(lbg_batch* b) {
  CapScope cap(b->sm_cap);
  const lbg_pp* pp = b->pp;
  cudaError_t e = launch_challenge_slots(pp->pidx[0], b->d_ch, (int)b->total_cols, pp->d_prime[0], b->d_chat, b->stream);
  if (e == cudaSuccess && b->keep)
    e = launch_fold_kept(pp->pidx[0], b->d_keep, b->wdim, (int)b->total_cols, b->fold_per, b->d_chat,
                         pp->d_prime[0], b->d_vhat, b->d_v, b->stream, b->count, b->d_split_inst);
  else if (e == cudaSuccess && b->d_gm)
    e = launch_fold_gm(pp->pidx[0], b->d_w, b->wdim, (int)b->total_cols, b->fold_per, b->d_chat, pp->d_tcb[0],
                       b->d_gm, pp->d_prime[0], b->d_vhat, b->d_v, b->stream, b->count, b->d_split_inst);
  else if (e == cudaSuccess)
    e = launch_fold(pp->pidx[0], b->d_w, b->wdim, (int)b->total_cols, b->fold_per, b->d_chat, pp->d_prime[0],
                    b->d_vhat, b->d_v, b->stream, b->count, b->d_split_inst, pp->d_tcb[0]);
  b->launches += (b->d_gm && !b->keep) ? 4 : 3;
  return e;
}

// The split -> instance map for fold splits of `per` columns (per divides every column count).
static int upload_splits(lbg_batch* b, int per) {
  std::vector<int> inst(b->total_cols / per);
  for (int i = 0; i < b->count; i++)
    for (size_t c = b->col_off[i]; c < b->col_off[i + 1]; c += per) inst[c / per] = i;
  LBG_BCU(cudaMemcpyAsync(b->d_split_inst, inst.data(), inst.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  b->fold_per = per;
  return LBG_OK;
}

static void set_chunks(lbg_batch* b, int nch) {
  int step = commit_ring_per_step();
  int chunk = (int)((b->len_ring + nch - 1) / nch);
  chunk = (chunk + step - 1) / step * step;
  b->chunk = chunk;
  b->nchunks = (int)((b->len_ring + chunk - 1) / chunk);
}

// Time one enqueue (median of three) on the batch's stream.
template <class F>
static float time_stage(lbg_batch* b, F enqueue) {
  cudaEvent_t a, c;
  cudaEventCreate(&a);
  cudaEventCreate(&c);
  std::vector<float> ts;
  enqueue(b);  // warm
  for (int r = 0; r < 3; r++) {
    cudaEventRecord(a, b->stream);
    enqueue(b);
    cudaEventRecord(c, b->stream);
    cudaEventSynchronize(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, c);
    ts.push_back(ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(c);
  std::sort(ts.begin(), ts.end());
  return ts[1];
}

// ---------------------------------------------------------------------------------------------
// the whole round on the device
// ---------------------------------------------------------------------------------------------
static cudaError_t grow(void** p, size_t* cap, size_t bytes) {
  if (bytes <= *cap) return cudaSuccess;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) *cap = bytes;
  return e;
}

static void le64(uint64_t x, uint8_t* b) {
  for (int i = 0; i < 8; i++) b[i] = (uint8_t)(x >> (8 * i));
}

static bool is_switch(const lbg_batch* b, int i) { return !b->sw_flag.empty() && b->sw_flag[i]; }

// Each instance's transcript up to the commitment's own bytes (host, once per layout and domain),
// the byte layout of the two device absorbs (the commitment; the row values with their framing)
// and the derivation counters. The transcript steps are those of derive_evaluation_point and
// FoldingChallenges::derive (crates/pcs/src/scheme/verifier.rs:41-100,
// crates/pcs/src/scheme/commitment.rs:217-229); a switch instance's are those of a B128 trace
// opened through the switch (crates/pcs/examples/two_fields.rs:176-194): the tagged commitment
// (Commitment::to_bytes), the switch's own steps, then FoldingChallenges::derive.
static int plan_round(lbg_batch* b, const uint8_t* domain, size_t domain_len) {
  const lbg_pp* pp = b->pp;
  int L = pp->limbs;
  bool dropped = pp->params.opening == LBG_OPENING_BIT_DROPPED;
  uint32_t row_log = pp->params.witness_log_len - pp->params.column_log_len;
  RoundShape base;
  base.limbs = (uint32_t)L;
  base.dropped_bits = dropped ? pp->params.dropped_bits : 0;
  for (int k = 0; k < 8; k++) base.primes[k] = k < L ? pp->primes[k] : 0;
  std::memcpy(base.matrix_seed, pp->seed, 32);
  // bit-dropped commitments as the transcript reads them (crates/pcs/src/wire/mod.rs:386-397)
  b->packed_off.assign(1, 0);
  b->packed_len.clear();
  if (dropped) {
    PackDropped pk{};
    pk.limbs = (uint32_t)L;
    pk.top_bits = top_bits(pp->primes[0], pp->params.dropped_bits);
    pk.bits_per = pk.top_bits;
    for (int k = 1; k < L; k++) {
      pk.residue_bits[k] = residue_bits(pp->primes[k]);
      pk.bits_per += pk.residue_bits[k];
    }
    b->pack = pk;
    for (int i = 0; i < b->count; i++) {
      uint64_t count = (uint64_t)(b->col_off[i + 1] - b->col_off[i]) * N648;
      uint64_t bytes = (count * pk.bits_per + 7) / 8;
      b->packed_len.push_back(bytes);
      b->packed_off.push_back(b->packed_off.back() + (bytes + 15) / 16 * 16);
    }
    LBG_BCU(grow((void**)&b->d_packed, &b->packed_cap, b->packed_off.back()));
  }
  b->ab_commit.clear();
  b->ab_u.clear();
  std::vector<HasherState> pre(b->count);
  std::vector<RoundInst> ri(b->count);
  for (int i = 0; i < b->count; i++) {
    RoundShape s = base;
    s.column_log_len = b->col_log[i];
    s.witness_log_len = row_log + b->col_log[i];
    bool sw = is_switch(b, i);
    uint32_t l = row_log + b->col_log[i];
    Transcript t(domain, domain_len);
    if (!sw) absorb_commitment_header(s, t);
    t.state().save(pre[i]);
    uint64_t len0 = absorbed_len(pre[i]);
    uint64_t cols = b->col_off[i + 1] - b->col_off[i];
    AbsorbSource sc;
    std::memset(&sc, 0, sizeof(sc));
    // Commitment::to_bytes (crates/pcs/src/wire/mod.rs:307-333) as absorb_bytes frames it: the
    // length, the form's tag, the column count (u32), then the body
    auto tagged = [&](uint8_t tag, uint64_t body) {
      le64(5 + body, sc.prefix);
      sc.prefix[8] = tag;
      for (int k = 0; k < 4; k++) sc.prefix[9 + k] = (uint8_t)(cols >> (8 * k));
      sc.prefix_len = 13;
    };
    if (!dropped) {
      if (sw) {
        tagged(0, cols * 4 * L * N162 * 2);  // the matrix column by column, i16 little-endian
      } else {
        // absorb_elements per column: le64(4), then the column's 4 x limbs x 162 i16, little-endian
        le64(4, sc.hdr);
        sc.hdr_len = 8;
      }
      sc.rows = (uint32_t)cols;
      sc.row_bytes = (uint32_t)(4 * L * N162 * 2);
      sc.row_stride = sc.row_bytes;
      sc.data = (const uint8_t*)(b->d_C + b->col_off[i] * 4 * L * N162);
    } else {
      if (sw) {
        tagged(2, b->packed_len[i]);
      } else {
        le64(b->packed_len[i], sc.prefix);
        sc.prefix_len = 8;
      }
      sc.rows = 1;
      sc.row_bytes = (uint32_t)b->packed_len[i];
      sc.row_stride = 0;
      sc.data = b->d_packed + b->packed_off[i];
    }
    plan_absorb(b->ab_commit, b->d_states + i, len0, sc);
    // absorb_bytes("labinius/row-evaluation"), absorb_bytes(u as 24-byte F162)
    AbsorbSource su;
    std::memset(&su, 0, sizeof(su));
    le64(23, su.prefix);
    std::memcpy(su.prefix + 8, "labinius/row-evaluation", 23);
    le64(24 * cols, su.prefix + 31);
    su.prefix_len = 39;
    su.rows = 1;
    su.row_bytes = (uint32_t)(24 * cols);
    su.data = (const uint8_t*)(b->d_u + 3 * b->col_off[i]);
    uint64_t sw_bytes = sw ? sw_transcript_bytes(l, 0) : 0;
    plan_absorb(b->ab_u, b->d_states + i, len0 + sc.length() + sw_bytes, su);
    ri[i].st = b->d_states + i;
    ri[i].point_counter = t.counter();
    // the switch derives the batch, then one challenge per round
    ri[i].chal_counter = t.counter() + (sw ? 1 + l : 1);
    ri[i].row_log = row_log;
    ri[i].col_log = b->col_log[i];
    ri[i].col_off = (uint32_t)b->col_off[i];
    ri[i].pad_ = 0;
  }
  LBG_BCU(cudaMemcpyAsync(b->d_prefix, pre.data(), pre.size() * sizeof(HasherState), cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(cudaMemcpyAsync(b->d_inst, ri.data(), ri.size() * sizeof(RoundInst), cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(upload_absorb(b->ab_commit));
  LBG_BCU(upload_absorb(b->ab_u));
  LBG_BCU(grow((void**)&b->d_stage, &b->stage_cap, std::max(b->ab_commit.stage_bytes, b->ab_u.stage_bytes)));
  LBG_BCU(grow((void**)&b->d_cvs, &b->cvs_cap, 32 * std::max(b->ab_commit.cv_slots, b->ab_u.cv_slots)));
  LBG_BCU(sampler_tables(pp->device, b->sampler));
  b->plan_domain.assign((const char*)domain, domain_len);
  b->plan_ok = true;
  if (b->g_round) {
    cudaGraphExecDestroy(b->g_round);
    b->g_round = nullptr;
  }
  return LBG_OK;
}

static cudaError_t enqueue_round(lbg_batch* b) {
  const lbg_pp* pp = b->pp;
  int row_log = (int)(pp->params.witness_log_len - pp->params.column_log_len);
  int cols = (int)b->total_cols;
  cudaError_t e = cudaMemcpyAsync(b->d_states, b->d_prefix, (size_t)b->count * sizeof(HasherState),
                                  cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = enqueue_commit(b);
  if (e == cudaSuccess && pp->params.opening == LBG_OPENING_BIT_DROPPED) {
    uint64_t stride = (uint64_t)b->total_cols * N648;
    for (int i = 0; i < b->count && e == cudaSuccess; i++) {
      uint64_t o = (uint64_t)b->col_off[i] * N648;
      e = launch_pack_dropped(b->d_top + o, b->d_digits + o, (uint64_t)(b->col_off[i + 1] - b->col_off[i]) * N648,
                              stride, b->pack, b->d_packed + b->packed_off[i], b->packed_len[i], b->stream);
    }
    b->launches += b->count;
  }
  if (e == cudaSuccess) e = launch_absorb(b->ab_commit, b->d_stage, b->d_cvs, b->d_oldcv, b->stream);
  if (e == cudaSuccess) e = launch_point(b->d_inst, b->count, (uint32_t)row_log, b->d_p0, b->d_p1, b->stream);
  // switch instances: their evaluation point is where the switch's sumcheck ends
  if (e == cudaSuccess && !b->sw_h.empty())
    e = enqueue_switch(b->d_sw_inst, b->sw_h.data(), (int)b->sw_h.size(), b->stream, &b->launches);
  if (e == cudaSuccess) e = launch_eq_table(b->d_p0, row_log, b->wdim, b->d_eq, b->stream, b->count);
  if (e == cudaSuccess) e = launch_row_eval(b->d_w, b->wdim, cols, b->d_eq, b->d_u, b->stream, b->d_row_tiles, b->n_row_tiles);
  if (e == cudaSuccess) e = launch_claims(b->d_inst, b->d_col_inst, b->d_u, cols, b->d_p1, b->count, b->d_claim, b->stream);
  if (e == cudaSuccess) e = launch_absorb(b->ab_u, b->d_stage, b->d_cvs, b->d_oldcv, b->stream);
  if (e == cudaSuccess) e = launch_challenges(b->d_inst, b->d_col_inst, cols, b->sampler, b->d_ch, b->stream);
  if (e == cudaSuccess) e = enqueue_fold(b);
  b->launches += 11;
  return e;
}

extern "C" {

void lbg_batch_free(lbg_batch* b) {
  if (!b) return;
  cudaSetDevice(b->pp->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_graphs(b);
  void* ptrs[] = {b->d_w, b->d_col_inst, b->d_row_tiles, b->d_split_inst, b->d_partial, b->d_C, b->d_res, b->d_top, b->d_digits,
                  b->d_p0, b->d_p1, b->d_eq, b->d_u, b->d_claim, b->d_ch, b->d_chat, b->d_vhat, b->d_v,
                  b->d_prefix, b->d_states, b->d_inst, b->d_oldcv, b->d_stage, b->d_cvs, b->d_packed, b->d_keep,
                  b->d_sw_inst, b->d_sw_small, b->d_sw_scratch, b->d_sw_r, b->d_gm};
  for (void* p : ptrs) cudaFree(p);
  b->ab_commit.release();
  b->ab_u.release();
  if (b->stream) cudaStreamDestroy(b->stream);
  const lbg_pp* pp = b->pp;
  delete b;
  lbg_pp_release(pp);
}

// The device bytes lbg_batch_new_capacity allocates for an arena of this size (the buffers below,
// in the same order); the kept transform, the switch workspace and the packed bit-dropped bytes
// are allocated later, on use.
size_t lbg_batch_arena_bytes(const lbg_pp* pp, size_t max_cols, size_t max_instances) {
  if (!pp) return 0;
  const size_t L = (size_t)pp->limbs, C = max_cols, I = max_instances, wdim = pp->wdim;
  const size_t count648 = C * N648;
  size_t chunks = (pp->len_ring + commit_ring_per_step() - 1) / commit_ring_per_step();
  if (chunks > 64) chunks = 64;
  return C * wdim * 24 + C * sizeof(int) + C * sizeof(int4) + C * sizeof(int) + chunks * C * N162 * 16 +
         C * 4 * L * N162 * 2 + L * count648 * 2 + count648 * 2 + (L > 1 ? L - 1 : 1) * count648 * 2 + I * 32 * 24 * 2 +
         I * wdim * 24 + C * 24 + I * 24 + C * sizeof(lbg_challenge_d) + C * N162 * 4 + I * wdim * N162 * 4 +
         I * pp->len_ring * N648 * 2 + 2 * I * sizeof(HasherState) + I * sizeof(RoundInst) + I * 32 +
         (batch_fold_gm(C) ? fold_gm_operand_bytes(C) : 0);
}

// The batch's stream at the device's greatest (high != 0) or default priority: when both are
// waiting for SMs, the CTAs of a high-priority stream's launches are scheduled first. The stream is
// replaced (after the old one drains) and the graphs captured on it are dropped, so their next
// capture takes the new priority.
int lbg_batch_set_priority(lbg_batch* b, int high) {
  if (!b) return fail(LBG_ERR_INVALID, "null argument");
  LBG_BCU(cudaSetDevice(b->pp->device));
  int least = 0, greatest = 0;
  LBG_BCU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  cudaStream_t st = nullptr;
  LBG_BCU(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high ? greatest : 0));
  cudaStreamSynchronize(b->stream);
  free_graphs(b);
  cudaStreamDestroy(b->stream);
  b->stream = st;
  return LBG_OK;
}

// At most `ctas` CTAs (one per SM) for the batch's persistent commit and fold launches (0: every SM),
// so that another slot's launches find SMs free while this batch runs. Drops captured graphs.
int lbg_batch_set_sm_limit(lbg_batch* b, int ctas) {
  if (!b || ctas < 0) return fail(LBG_ERR_INVALID, "null argument or negative limit");
  if (b->sm_cap != ctas) {
    LBG_BCU(cudaSetDevice(b->pp->device));
    cudaStreamSynchronize(b->stream);
    free_graphs(b);
    b->sm_cap = ctas;
  }
  return LBG_OK;
}

// An arena of `max_cols` columns and `max_instances` instances: the device buffers are sized once;
// lbg_batch_assign lays out a set of instances inside it without allocating.
int lbg_batch_new_capacity(const lbg_pp* pp, size_t max_cols, size_t max_instances, lbg_batch** out) {
  if (!pp || !out || max_cols == 0 || max_instances == 0) return fail(LBG_ERR_INVALID, "null argument or empty batch");
  *out = nullptr;
  if (pp->params.opening == LBG_OPENING_RECURSIVE)
    return fail(LBG_ERR_UNSUPPORTED, "batched rounds cover the Clear and bit-dropped openings");
  if (max_instances > 65536) return fail(LBG_ERR_INVALID, "at most 65536 instances");
  if (max_cols > ((size_t)1 << 30) / pp->wdim) return fail(LBG_ERR_PARAMS, "batch too large");
  lbg_batch* b = new lbg_batch();
  b->pp = pp;
  lbg_pp_retain(pp);  // released when the batch goes
  b->wdim = pp->wdim;
  b->len_ring = pp->len_ring;
  b->cap_cols = max_cols;
  b->cap_instances = max_instances;
  auto bail = [&](int code) {
    lbg_batch_free(b);
    return code;
  };
  if (cudaSetDevice(pp->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(LBG_ERR_CUDA, "stream"));
  int L = pp->limbs;
  size_t C = max_cols, I = max_instances, n = C * b->wdim, count648 = C * N648;
  b->max_chunks = (int)((b->len_ring + commit_ring_per_step() - 1) / commit_ring_per_step());
  if (b->max_chunks > 64) b->max_chunks = 64;
  bool ok = cudaMalloc((void**)&b->d_w, n * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_col_inst, C * sizeof(int)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_row_tiles, C * sizeof(int4)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_split_inst, C * sizeof(int)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_partial, (size_t)b->max_chunks * C * N162 * 16) == cudaSuccess &&
            cudaMalloc((void**)&b->d_C, C * 4 * L * N162 * 2) == cudaSuccess &&
            cudaMalloc((void**)&b->d_res, (size_t)L * count648 * 2) == cudaSuccess &&
            cudaMalloc((void**)&b->d_top, count648 * 2) == cudaSuccess &&
            cudaMalloc((void**)&b->d_digits, (size_t)(L > 1 ? L - 1 : 1) * count648 * 2) == cudaSuccess &&
            cudaMalloc((void**)&b->d_p0, I * 32 * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_p1, I * 32 * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_eq, I * b->wdim * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_u, C * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_claim, I * 24) == cudaSuccess &&
            cudaMalloc((void**)&b->d_ch, C * sizeof(lbg_challenge_d)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_chat, C * N162 * 4) == cudaSuccess &&
            cudaMalloc((void**)&b->d_vhat, I * b->wdim * N162 * 4) == cudaSuccess &&
            cudaMalloc((void**)&b->d_v, I * b->len_ring * N648 * 2) == cudaSuccess &&
            cudaMalloc((void**)&b->d_prefix, I * sizeof(HasherState)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_states, I * sizeof(HasherState)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_inst, I * sizeof(RoundInst)) == cudaSuccess &&
            cudaMalloc((void**)&b->d_oldcv, I * 32) == cudaSuccess &&
            (!batch_fold_gm(C) || cudaMalloc((void**)&b->d_gm, fold_gm_operand_bytes(C)) == cudaSuccess);
  if (!ok) {
    cudaGetLastError();
    return bail(fail(LBG_ERR_OOM, "batch: device allocation failed"));
  }
  if (cudaMemsetAsync(b->d_w, 0, n * 24, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->d_ch, 0, C * sizeof(lbg_challenge_d), b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return bail(fail(LBG_ERR_CUDA, "batch init"));
  *out = b;
  return LBG_OK;
}

// Lay out `count` instances (instance i: 2^column_log_lens[i] columns) in the arena; the model
// schedule is set, the CUDA graphs (if any) dropped.
int lbg_batch_assign(lbg_batch* b, const uint32_t* column_log_lens, size_t count) {
  if (!b || !column_log_lens || count == 0) return fail(LBG_ERR_INVALID, "null argument or empty batch");
  if (count > b->cap_instances) return fail(LBG_ERR_INVALID, "more instances than the batch holds");
  const lbg_pp* pp = b->pp;
  uint32_t row_log = pp->params.witness_log_len - pp->params.column_log_len;
  std::vector<uint32_t> cl(column_log_lens, column_log_lens + count);
  std::vector<size_t> off{0};
  int minc = 31;
  for (size_t i = 0; i < count; i++) {
    if (cl[i] < 1 || cl[i] + row_log > 30)
      return fail(LBG_ERR_PARAMS, "instance " + std::to_string(i) + ": column_log_len out of range");
    minc = std::min(minc, (int)cl[i]);
    off.push_back(off.back() + ((size_t)1 << cl[i]));
  }
  if (off.back() > b->cap_cols) return fail(LBG_ERR_INVALID, "more columns than the batch holds");
  LBG_BCU(cudaSetDevice(pp->device));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  if (b->graphs) {
    free_graphs(b);
    b->graphs = false;
  }
  b->plan_ok = false;
  b->sw_flag.clear();
  b->sw_h.clear();
  b->count = (int)count;
  b->col_log = cl;
  b->col_off = off;
  b->total_cols = off.back();
  b->min_col_log = minc;
  std::vector<int> ci(b->total_cols);
  for (int i = 0; i < b->count; i++)
    for (size_t c = off[i]; c < off[i + 1]; c++) ci[c] = i;
  LBG_BCU(cudaMemcpyAsync(b->d_col_inst, ci.data(), ci.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  std::vector<int4> rtiles;
  int tc = row_eval_tile_cols();
  for (int i = 0; i < b->count; i++)
    for (size_t c = off[i]; c < off[i + 1]; c += tc)
      rtiles.push_back(make_int4((int)c, (int)std::min<size_t>(tc, off[i + 1] - c), i, 0));
  LBG_BCU(cudaMemcpyAsync(b->d_row_tiles, rtiles.data(), rtiles.size() * sizeof(int4), cudaMemcpyHostToDevice,
                          b->stream));
  b->n_row_tiles = (int)rtiles.size();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pp->device);
  long tiles = (long)((b->total_cols + commit_cols_per_cta() - 1) / commit_cols_per_cta());
  int want = (int)std::max<long>(1, (2L * sms * commit_blocks_per_sm(pp->pidx[0]) + tiles - 1) / tiles);
  set_chunks(b, std::min(want, b->max_chunks));
  return upload_splits(b, std::min(16, 1 << b->min_col_log));
}

int lbg_batch_new(const lbg_pp* pp, const uint32_t* column_log_lens, size_t count, lbg_batch** out) {
  if (!pp || !column_log_lens || !out || count == 0) return fail(LBG_ERR_INVALID, "null argument or empty batch");
  *out = nullptr;
  uint32_t row_log = pp->params.witness_log_len - pp->params.column_log_len;
  size_t cols = 0;
  for (size_t i = 0; i < count; i++) {
    if (column_log_lens[i] < 1 || column_log_lens[i] + row_log > 30)
      return fail(LBG_ERR_PARAMS, "instance " + std::to_string(i) + ": column_log_len out of range");
    cols += (size_t)1 << column_log_lens[i];
  }
  lbg_batch* b = nullptr;
  int rc = lbg_batch_new_capacity(pp, cols, count, &b);
  if (rc) return rc;
  rc = lbg_batch_assign(b, column_log_lens, count);
  if (rc) {
    lbg_batch_free(b);
    return rc;
  }
  *out = b;
  return LBG_OK;
}

size_t lbg_batch_columns(const lbg_batch* b) { return b ? b->total_cols : 0; }

// The keyed BLAKE3 root of a one-block message (the XOF kernels compute its output blocks).
static XofRoot keyed_root(const uint8_t* key, const char* label) {
  XofRoot root;
  for (int w = 0; w < 8; w++)
    root.cv[w] = (uint32_t)key[4 * w] | ((uint32_t)key[4 * w + 1] << 8) | ((uint32_t)key[4 * w + 2] << 16) |
                 ((uint32_t)key[4 * w + 3] << 24);
  uint8_t msg[64] = {0};
  size_t len = std::strlen(label);
  std::memcpy(msg, label, len);
  for (int w = 0; w < 16; w++)
    root.m[w] = (uint32_t)msg[4 * w] | ((uint32_t)msg[4 * w + 1] << 8) | ((uint32_t)msg[4 * w + 2] << 16) |
                ((uint32_t)msg[4 * w + 3] << 24);
  root.block_len = (uint32_t)len;
  root.flags = 16 | 1 | 2 | 8;  // keyed hash, chunk start, chunk end, root
  return root;
}

// Witnesses of every instance from 32-byte seeds: kind 0 is Witness::random (keyed BLAKE3 XOF of
// "labinius/witness", crates/pcs/src/scheme/witness.rs:66-87); kind 1 is a B128 trace (keyed XOF
// of "labinius/b128-trace", 16 bytes per element) lifted bit for bit (Witness::lifted,
// crates/pcs/src/scheme/witness.rs:45-52). `kinds` may be null (all kind 0).
int lbg_batch_witness_generate(lbg_batch* b, const uint8_t* seeds, const uint8_t* kinds) {
  if (!b || !seeds) return fail(LBG_ERR_INVALID, "null argument");
  LBG_BCU(cudaSetDevice(b->pp->device));
  for (int i = 0; i < b->count; i++) {
    size_t n = (b->col_off[i + 1] - b->col_off[i]) * b->wdim;
    uint64_t* dst = b->d_w + b->col_off[i] * b->wdim * 3;
    if (kinds && kinds[i] == 1) {
      LBG_BCU(launch_xof_lifted(keyed_root(seeds + 32 * i, "labinius/b128-trace"), n, dst, b->stream));
    } else {
      LBG_BCU(launch_xof_f162(keyed_root(seeds + 32 * i, "labinius/witness"), n, dst, b->stream));
    }
  }
  LBG_BCU(cudaStreamSynchronize(b->stream));
  return LBG_OK;
}

int lbg_batch_witness_random(lbg_batch* b, const uint8_t* seeds) { return lbg_batch_witness_generate(b, seeds, nullptr); }

int lbg_batch_witness_upload(lbg_batch* b, size_t instance, const uint64_t* f162, size_t n) {
  if (!b || !f162) return fail(LBG_ERR_INVALID, "null argument");
  if (instance >= (size_t)b->count) return fail(LBG_ERR_INVALID, "instance out of range");
  if (n != (b->col_off[instance + 1] - b->col_off[instance]) * b->wdim)
    return fail(LBG_ERR_WITNESS, "the witness is not witness_len() elements");
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaMemcpyAsync(b->d_w + b->col_off[instance] * b->wdim * 3, f162, n * 24, cudaMemcpyHostToDevice,
                          b->stream));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  return LBG_OK;
}

int lbg_batch_witness_download(const lbg_batch* b, size_t instance, uint64_t* out, size_t n) {
  if (!b || !out) return fail(LBG_ERR_INVALID, "null argument");
  if (instance >= (size_t)b->count) return fail(LBG_ERR_INVALID, "instance out of range");
  if (n != (b->col_off[instance + 1] - b->col_off[instance]) * b->wdim) return fail(LBG_ERR_INVALID, "length mismatch");
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaMemcpy(out, b->d_w + b->col_off[instance] * b->wdim * 3, n * 24, cudaMemcpyDeviceToHost));
  return LBG_OK;
}

// CUDA graphs of the two device stages; rebuilt after the autotuner changes the schedule.
int lbg_batch_use_graphs(lbg_batch* b, int enable) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  free_graphs(b);
  b->graphs = false;
  if (!enable) return LBG_OK;
  cudaGraph_t g = nullptr;
  uint64_t before = b->launches;
  LBG_BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = enqueue_commit(b);
  cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) return fail(LBG_ERR_CUDA, "graph capture (commit)");
  e = cudaGraphInstantiate(&b->g_commit, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, "graph instantiate (commit)");
  LBG_BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  e = enqueue_fold(b);
  e2 = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) return fail(LBG_ERR_CUDA, "graph capture (fold)");
  e = cudaGraphInstantiate(&b->g_fold, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, "graph instantiate (fold)");
  b->launches = before;  // capture launched nothing
  b->graphs = true;
  return LBG_OK;
}

// The kept transform on or off (allocated on first use: 324 B per F162 of the arena); the
// captured graphs are rebuilt.
static int set_keep(lbg_batch* b, bool on) {
  if (on && !b->d_keep) {
    if (cudaMalloc((void**)&b->d_keep, b->cap_cols * b->wdim * N162 * 2) != cudaSuccess) {
      cudaGetLastError();
      b->d_keep = nullptr;
      return fail(LBG_ERR_OOM, "kept transform: device allocation failed");
    }
  }
  if (b->keep == on) return LBG_OK;
  bool had = b->graphs;
  if (had) lbg_batch_use_graphs(b, 0);
  b->keep = on;
  if (had) return lbg_batch_use_graphs(b, 1);
  return LBG_OK;
}

int lbg_batch_set_kept_transform(lbg_batch* b, int enable) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  return set_keep(b, enable != 0);
}

// The autotuner: time candidate schedules of both stages on this batch's shape and keep the
// fastest (commit: ring-element chunks per column tile; fold: columns per split; whether the
// fold reads the commit's kept transform).
int lbg_batch_autotune(lbg_batch* b, uint32_t* chunks_out, uint32_t* fold_cols_out) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  LBG_BCU(cudaSetDevice(b->pp->device));
  bool had = b->graphs;
  if (had) lbg_batch_use_graphs(b, 0);
  uint64_t launches = b->launches;
  std::vector<int> cand;
  for (int c = 1; c <= b->max_chunks; c *= 2) cand.push_back(c);
  for (int c = 3; c <= b->max_chunks; c *= 2) cand.push_back(c);
  float best = -1;
  int best_c = b->nchunks;
  for (int c : cand) {
    set_chunks(b, c);
    float t = time_stage(b, enqueue_commit);
    if (best < 0 || t < best) {
      best = t;
      best_c = c;
    }
  }
  set_chunks(b, best_c);
  // the commit's CTA shape: 12 compute warps and a producer warp, or 16 compute warps
  best = -1;
  int best_w = 12;
  for (int w : {12, 16}) {
    b->commit_warps = w;
    float t = time_stage(b, enqueue_commit);
    if (best < 0 || t < best) {
      best = t;
      best_w = w;
    }
  }
  b->commit_warps = best_w;
  best = -1;
  int best_p = b->fold_per;
  for (int per = 8; per <= std::min(256, 1 << b->min_col_log); per *= 2) {
    if (upload_splits(b, per)) return LBG_ERR_CUDA;
    float t = time_stage(b, enqueue_fold);
    if (best < 0 || t < best) {
      best = t;
      best_p = per;
    }
  }
  if (1 << b->min_col_log < 8) best_p = 1 << b->min_col_log;
  int rc = upload_splits(b, best_p);
  if (rc) return rc;
  {
    auto both = [](lbg_batch* x) {
      cudaError_t e = enqueue_commit(x);
      return e == cudaSuccess ? enqueue_fold(x) : e;
    };
    b->keep = false;
    float t_off = time_stage(b, both);
    float t_on = -1;
    if (b->d_keep || cudaMalloc((void**)&b->d_keep, b->cap_cols * b->wdim * N162 * 2) == cudaSuccess) {
      b->keep = true;
      t_on = time_stage(b, both);
    } else {
      cudaGetLastError();
      b->d_keep = nullptr;
    }
    b->keep = t_on >= 0 && t_on < t_off;
  }
  b->launches = launches;
  LBG_BCU(cudaStreamSynchronize(b->stream));
  if (chunks_out) *chunks_out = (uint32_t)b->nchunks;
  if (fold_cols_out) *fold_cols_out = (uint32_t)b->fold_per;
  if (had) return lbg_batch_use_graphs(b, 1);
  return LBG_OK;
}

int lbg_batch_schedule(const lbg_batch* b, uint32_t* commit_warps, int* kept_transform) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  if (commit_warps) *commit_warps = (uint32_t)(b->commit_warps ? b->commit_warps : 12);
  if (kept_transform) *kept_transform = b->keep ? 1 : 0;
  return LBG_OK;
}

int lbg_batch_commit(lbg_batch* b, int16_t* matrix_out, uint16_t* top_out, uint16_t* digits_out) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  const lbg_pp* pp = b->pp;
  LBG_BCU(cudaSetDevice(pp->device));
  if (b->graphs) {
    LBG_BCU(cudaGraphLaunch(b->g_commit, b->stream));
    b->launches += 2 * pp->limbs + (pp->params.opening == LBG_OPENING_BIT_DROPPED ? pp->limbs + 1 : 0);
  } else {
    LBG_BCU(enqueue_commit(b));
  }
  size_t C = b->total_cols, count = C * N648;
  int L = pp->limbs;
  if (matrix_out) LBG_BCU(cudaMemcpyAsync(matrix_out, b->d_C, C * 4 * L * N162 * 2, cudaMemcpyDeviceToHost, b->stream));
  if (top_out) LBG_BCU(cudaMemcpyAsync(top_out, b->d_top, count * 2, cudaMemcpyDeviceToHost, b->stream));
  if (digits_out && L > 1)
    LBG_BCU(cudaMemcpyAsync(digits_out, b->d_digits, (size_t)(L - 1) * count * 2, cudaMemcpyDeviceToHost, b->stream));
  if (matrix_out || top_out || digits_out) LBG_BCU(cudaStreamSynchronize(b->stream));
  return LBG_OK;
}

int lbg_batch_row_evaluate(lbg_batch* b, const uint64_t* p0, uint64_t* u_out) {
  if (!b || !p0 || !u_out) return fail(LBG_ERR_INVALID, "null argument");
  int row_log = (int)(b->pp->params.witness_log_len - b->pp->params.column_log_len);
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaMemcpyAsync(b->d_p0, p0, (size_t)b->count * row_log * 24, cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(launch_eq_table(b->d_p0, row_log, b->wdim, b->d_eq, b->stream, b->count));
  LBG_BCU(launch_row_eval(b->d_w, b->wdim, (int)b->total_cols, b->d_eq, b->d_u, b->stream, b->d_row_tiles, b->n_row_tiles));
  b->launches += 2;
  LBG_BCU(cudaMemcpyAsync(u_out, b->d_u, b->total_cols * 24, cudaMemcpyDeviceToHost, b->stream));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  return LBG_OK;
}

// claims: p1 of instance i is column_log_len_i F162 at p1 + 3 * sum_{l<i} column_log_len_l.
int lbg_batch_mle_evaluate(lbg_batch* b, const uint64_t* p0, const uint64_t* p1, uint64_t* out) {
  if (!b || !p0 || !p1 || !out) return fail(LBG_ERR_INVALID, "null argument");
  int row_log = (int)(b->pp->params.witness_log_len - b->pp->params.column_log_len);
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaMemcpyAsync(b->d_p0, p0, (size_t)b->count * row_log * 24, cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(launch_eq_table(b->d_p0, row_log, b->wdim, b->d_eq, b->stream, b->count));
  LBG_BCU(launch_row_eval(b->d_w, b->wdim, (int)b->total_cols, b->d_eq, b->d_u, b->stream, b->d_row_tiles, b->n_row_tiles));
  size_t off = 0;
  for (int i = 0; i < b->count; i++) {
    int cl = (int)b->col_log[i];
    LBG_BCU(cudaMemcpyAsync(b->d_p1 + 3 * 32 * i, p1 + 3 * off, cl * 24, cudaMemcpyHostToDevice, b->stream));
    LBG_BCU(launch_claim(b->d_u + 3 * b->col_off[i], 1 << cl, b->d_p1 + 3 * 32 * i, cl, b->d_claim + 3 * i, b->stream));
    off += cl;
  }
  b->launches += 2 + b->count;
  LBG_BCU(cudaMemcpyAsync(out, b->d_claim, (size_t)b->count * 24, cudaMemcpyDeviceToHost, b->stream));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  return LBG_OK;
}

int lbg_batch_fold(lbg_batch* b, const lbg_challenge* challenges, size_t r, int16_t* v_out) {
  if (!b || !challenges) return fail(LBG_ERR_INVALID, "null argument");
  if (r != b->total_cols) return fail(LBG_ERR_INVALID, "one challenge per column");
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaMemcpyAsync(b->d_ch, challenges, r * sizeof(lbg_challenge), cudaMemcpyHostToDevice, b->stream));
  if (b->graphs) {
    LBG_BCU(cudaGraphLaunch(b->g_fold, b->stream));
    b->launches += (b->d_gm && !b->keep) ? 4 : 3;
  } else {
    LBG_BCU(enqueue_fold(b));
  }
  if (v_out) {
    LBG_BCU(cudaMemcpyAsync(v_out, b->d_v, (size_t)b->count * b->len_ring * N648 * 2, cudaMemcpyDeviceToHost,
                            b->stream));
    LBG_BCU(cudaStreamSynchronize(b->stream));
  }
  return LBG_OK;
}

int lbg_batch_round(lbg_batch* b, const uint8_t* domain, size_t domain_len, const lbg_batch_outputs* out) {
  if (!b || (!domain && domain_len)) return fail(LBG_ERR_INVALID, "null argument");
  if (b->count == 0) return fail(LBG_ERR_INVALID, "no instances assigned");
  const lbg_pp* pp = b->pp;
  LBG_BCU(cudaSetDevice(pp->device));
  std::string dom((const char*)domain, domain_len);
  if (!b->plan_ok || b->plan_domain != dom) {
    LBG_BCU(cudaStreamSynchronize(b->stream));
    int rc = plan_round(b, domain, domain_len);
    if (rc) return rc;
  }
  uint64_t per_round = 11 + 2 * pp->limbs + ((b->d_gm && !b->keep) ? 4 : 3) +
                       (pp->params.opening == LBG_OPENING_BIT_DROPPED ? pp->limbs + 1 + b->count : 0);
  per_round += sw_launches(b->sw_h.data(), (int)b->sw_h.size());
  if (b->graphs) {
    if (!b->g_round) {
      cudaGraph_t g = nullptr;
      uint64_t before = b->launches;
      LBG_BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue_round(b);
      cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
      b->launches = before;
      if (e != cudaSuccess || e2 != cudaSuccess) return fail(LBG_ERR_CUDA, "graph capture (round)");
      e = cudaGraphInstantiate(&b->g_round, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(LBG_ERR_CUDA, "graph instantiate (round)");
    }
    LBG_BCU(cudaGraphLaunch(b->g_round, b->stream));
    b->launches += per_round;
  } else {
    LBG_BCU(enqueue_round(b));
  }
  size_t C = b->total_cols, count = C * N648;
  int L = pp->limbs;
  int row_log = (int)(pp->params.witness_log_len - pp->params.column_log_len);
  std::vector<lbg_challenge> ch(C);
  std::vector<uint64_t> p1(out && out->p1 ? (size_t)b->count * 32 * 3 : 0);
  cudaStream_t st = b->stream;
  LBG_BCU(cudaMemcpyAsync(ch.data(), b->d_ch, C * sizeof(lbg_challenge), cudaMemcpyDeviceToHost, st));
  if (out) {
    if (out->matrix) LBG_BCU(cudaMemcpyAsync(out->matrix, b->d_C, C * 4 * L * N162 * 2, cudaMemcpyDeviceToHost, st));
    if (out->top) LBG_BCU(cudaMemcpyAsync(out->top, b->d_top, count * 2, cudaMemcpyDeviceToHost, st));
    if (out->digits && L > 1)
      LBG_BCU(cudaMemcpyAsync(out->digits, b->d_digits, (size_t)(L - 1) * count * 2, cudaMemcpyDeviceToHost, st));
    if (out->p0)
      LBG_BCU(cudaMemcpyAsync(out->p0, b->d_p0, (size_t)b->count * row_log * 24, cudaMemcpyDeviceToHost, st));
    if (out->p1) LBG_BCU(cudaMemcpyAsync(p1.data(), b->d_p1, p1.size() * 8, cudaMemcpyDeviceToHost, st));
    if (out->mle) LBG_BCU(cudaMemcpyAsync(out->mle, b->d_claim, (size_t)b->count * 24, cudaMemcpyDeviceToHost, st));
    if (out->u) LBG_BCU(cudaMemcpyAsync(out->u, b->d_u, C * 24, cudaMemcpyDeviceToHost, st));
    if (out->v)
      LBG_BCU(cudaMemcpyAsync(out->v, b->d_v, (size_t)b->count * b->len_ring * N648 * 2, cudaMemcpyDeviceToHost, st));
  }
  LBG_BCU(cudaStreamSynchronize(st));
  for (size_t j = 0; j < C; j++)
    if (ch[j].weight == 0) return fail(LBG_ERR_CUDA, "the device sampler found no challenge for column " + std::to_string(j));
  if (out && out->challenges) std::memcpy(out->challenges, ch.data(), C * sizeof(lbg_challenge));
  if (out && out->p1) {
    size_t o = 0;
    for (int i = 0; i < b->count; i++) {
      std::memcpy(out->p1 + o, p1.data() + (size_t)i * 32 * 3, b->col_log[i] * 24);
      o += 3 * b->col_log[i];
    }
  }
  return LBG_OK;
}

int lbg_batch_set_switch(lbg_batch* b, const uint8_t* flags, const uint64_t* r_hi, const uint64_t* claims) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  if (b->count == 0) return fail(LBG_ERR_INVALID, "no instances assigned");
  const lbg_pp* pp = b->pp;
  LBG_BCU(cudaSetDevice(pp->device));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  b->sw_flag.clear();
  b->sw_h.clear();
  b->plan_ok = false;
  if (b->g_round) {
    cudaGraphExecDestroy(b->g_round);
    b->g_round = nullptr;
  }
  if (!flags) return LBG_OK;
  uint32_t row_log = pp->params.witness_log_len - pp->params.column_log_len;
  std::vector<int> list;
  size_t scratch = 0, rwords = 0;
  for (int i = 0; i < b->count; i++) {
    if (!flags[i]) continue;
    uint32_t l = row_log + b->col_log[i];
    if (l > 32) return fail(LBG_ERR_PARAMS, "instance " + std::to_string(i) + ": a switch over more than 2^32 words");
    list.push_back(i);
    scratch += sw_scratch_bytes(l);
    rwords += 2 * (size_t)l;
  }
  if (list.empty()) return LBG_OK;
  if (!r_hi) return fail(LBG_ERR_INVALID, "switch instances need their r_hi");
  size_t n = list.size();
  LBG_BCU(grow((void**)&b->d_sw_inst, &b->sw_inst_cap, n * sizeof(SwInst)));
  LBG_BCU(grow((void**)&b->d_sw_small, &b->sw_small_cap, n * sizeof(SwSmall)));
  LBG_BCU(grow((void**)&b->d_sw_scratch, &b->sw_scratch_cap, scratch));
  LBG_BCU(grow((void**)&b->d_sw_r, &b->sw_r_cap, rwords * 8));
  LBG_BCU(cudaMemcpyAsync(b->d_sw_r, r_hi, rwords * 8, cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(cudaMemsetAsync(b->d_sw_small, 0, n * sizeof(SwSmall), b->stream));
  if (claims)
    LBG_BCU(cudaMemcpy2DAsync(&b->d_sw_small[0].claim[0], sizeof(SwSmall), claims, 16, 16, n, cudaMemcpyHostToDevice,
                              b->stream));
  std::vector<SwInst> hs(n);
  size_t roff = 0, soff = 0;
  for (size_t k = 0; k < n; k++) {
    int i = list[k];
    SwInst& h = hs[k];
    std::memset(&h, 0, sizeof(h));
    h.l = row_log + b->col_log[i];
    h.w = b->d_w + b->col_off[i] * b->wdim * 3;
    h.r_hi = b->d_sw_r + roff;
    h.s = b->d_sw_small + k;
    h.st = b->d_states + i;
    h.counter0 = 0;  // the instance's transcript derives nothing before the switch
    h.p0 = b->d_p0 + 3 * (size_t)row_log * i;
    h.p1 = b->d_p1 + 3 * 32 * (size_t)i;
    h.row_log = row_log;
    h.col_log = b->col_log[i];
    h.claim_given = claims ? 1 : 0;
    sw_layout(h, b->d_sw_scratch + soff);
    roff += 2 * (size_t)h.l;
    soff += sw_scratch_bytes(h.l);
  }
  LBG_BCU(cudaMemcpyAsync(b->d_sw_inst, hs.data(), n * sizeof(SwInst), cudaMemcpyHostToDevice, b->stream));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  b->sw_flag.assign(flags, flags + b->count);
  b->sw_h = hs;
  return LBG_OK;
}

int lbg_batch_switch_outputs(const lbg_batch* b, uint64_t* partials, uint64_t* rounds, uint64_t* opened,
                             uint64_t* claims) {
  if (!b) return fail(LBG_ERR_INVALID, "null batch");
  size_t n = b->sw_h.size();
  if (n == 0) return LBG_OK;
  LBG_BCU(cudaSetDevice(b->pp->device));
  LBG_BCU(cudaStreamSynchronize(b->stream));
  std::vector<SwSmall> hs(n);
  LBG_BCU(cudaMemcpy(hs.data(), b->d_sw_small, n * sizeof(SwSmall), cudaMemcpyDeviceToHost));
  size_t ro = 0;
  for (size_t k = 0; k < n; k++) {
    const SwSmall& o = hs[k];
    if (o.status != 1) return fail(LBG_ERR_INVALID, "no switch has run since the statements were set");
    uint32_t l = b->sw_h[k].l;
    if (partials) std::memcpy(partials + 256 * k, o.v, 128 * 16);
    if (rounds) std::memcpy(rounds + ro, o.rounds, (size_t)l * 48);
    if (opened) std::memcpy(opened + 3 * k, o.opened, 24);
    if (claims) std::memcpy(claims + 2 * k, o.claim, 16);
    ro += 6 * (size_t)l;
  }
  return LBG_OK;
}

void* lbg_batch_stream(const lbg_batch* b) { return b ? (void*)b->stream : nullptr; }
uint64_t lbg_batch_launch_count(const lbg_batch* b) { return b ? b->launches : 0; }

}  // extern "C"
