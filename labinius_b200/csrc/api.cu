// The C ABI of include/labinius_gpu.h: handles, device buffers, streams, and the per-call
// drivers that chain the kernels of kernels.cu.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "prime_structs.h"
#include "error.h"
#include "handles.h"
#include "launch.h"
#include "ring_tables.h"
#include "transcript.h"
#include "upload.h"

using namespace lbg;

// The fold's per-column tensor-core operands take 67.5 KB a column (276 MB at 4096 columns); wider
// witnesses fold with k_fold_tc instead.
constexpr size_t LBG_FOLD_GM_MAX_COLUMNS = 4096;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace

namespace lbg {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace lbg

#define LBG_CU(x)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) return fail(LBG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define LBG_ALLOC(ptr, bytes)                                                           \
  do {                                                                                  \
    cudaError_t e_ = cudaMalloc((void**)&(ptr), (bytes) ? (bytes) : 16);                \
    if (e_ != cudaSuccess) {                                                            \
      cudaGetLastError();                                                               \
      return fail(LBG_ERR_OOM, std::string("cudaMalloc ") + std::to_string(bytes) + ": " + cudaGetErrorString(e_)); \
    }                                                                                   \
  } while (0)

// Released witness buffers are kept (a few per process) and handed to the next witness of the
// same size, so a prover that commits new witnesses repeatedly does not pay cudaMalloc/cudaFree of
// the whole witness every round (tens of ms for 100 MB), the device-side counterpart of the
// reference's recycled workspace (crates/pcs/src/scheme/prover.rs:12-20).
namespace {
struct CachedBuf {
  int device;
  size_t bytes;
  uint64_t* p;
};
std::mutex g_cache_mu;
std::vector<CachedBuf> g_cache;
constexpr size_t CACHE_ENTRIES = 4;
}  // namespace

static uint64_t* witness_buf_get(int device, size_t bytes) {
  {
    std::lock_guard<std::mutex> g(g_cache_mu);
    for (size_t i = 0; i < g_cache.size(); i++)
      if (g_cache[i].device == device && g_cache[i].bytes == bytes) {
        uint64_t* p = g_cache[i].p;
        g_cache.erase(g_cache.begin() + i);
        return p;
      }
  }
  uint64_t* p = nullptr;
  if (cudaMalloc((void**)&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    // the cache may hold the memory this allocation needs: release it and retry once
    std::vector<CachedBuf> drop;
    {
      std::lock_guard<std::mutex> g(g_cache_mu);
      drop.swap(g_cache);
    }
    for (auto& c : drop) {
      cudaSetDevice(c.device);
      cudaFree(c.p);
    }
    cudaSetDevice(device);
    if (cudaMalloc((void**)&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  return p;
}

static void witness_buf_put(int device, size_t bytes, uint64_t* p) {
  // no kernel of any stream may still read the buffer when it is handed out again
  cudaSetDevice(device);
  cudaDeviceSynchronize();
  std::lock_guard<std::mutex> g(g_cache_mu);
  if (g_cache.size() < CACHE_ENTRIES) {
    g_cache.push_back({device, bytes, p});
    return;
  }
  cudaFree(p);
}

static void witness_release(lbg_witness* w) {
  if (w && w->refs.fetch_sub(1) == 1) {
    witness_buf_put(w->device, w->n * 24, w->d);
    delete w;
  }
}
void lbg_witness_release_internal(lbg_witness* w) { witness_release(w); }

extern "C" {

const char* lbg_last_error(void) { return g_err.c_str(); }
int lbg_version(void) { return 1; }

// crates/pcs/src/scheme/params.rs:172-203, plus what this path supports.
int lbg_params_check(const lbg_params* p) {
  if (!p) return fail(LBG_ERR_INVALID, "null params");
  if (p->column_log_len > p->witness_log_len) return fail(LBG_ERR_PARAMS, "column_log_len exceeds witness_log_len");
  if (p->column_log_len < 1) return fail(LBG_ERR_PARAMS, "column_log_len must be at least 1");
  if (p->witness_log_len - p->column_log_len < 7) return fail(LBG_ERR_PARAMS, "a column must hold at least 2^7 F162 elements");
  if (p->n_moduli < 1 || p->n_moduli > 7) return fail(LBG_ERR_PARAMS, "between 1 and 7 moduli");
  for (uint32_t i = 0; i < p->n_moduli; i++) {
    if (prime_index(p->moduli[i]) < 0) return fail(LBG_ERR_PARAMS, "unsupported modulus " + std::to_string(p->moduli[i]));
    for (uint32_t j = 0; j < i; j++)
      if (p->moduli[j] == p->moduli[i])
        return fail(LBG_ERR_PARAMS, j == 0 ? "the base modulus is listed again as an extra one" : "a modulus is listed twice");
  }
  if (p->opening == LBG_OPENING_BIT_DROPPED && (p->dropped_bits < 1 || p->dropped_bits > 14))
    return fail(LBG_ERR_PARAMS, "dropped bits out of range");
  if (p->opening > LBG_OPENING_RECURSIVE) return fail(LBG_ERR_PARAMS, "unknown opening mode");
  if (p->witness_log_len > 30) return fail(LBG_ERR_PARAMS, "witness too large");
  return LBG_OK;
}

// After a synchronisation: a tensor-core kernel whose bounded wait ran out reports a timeout.
static cudaError_t tc_checked(cudaError_t e) {
  if (e == cudaSuccess && tc_timeout_take() == 1) return cudaErrorLaunchTimeout;
  return e;
}

static int upload_prime(lbg_pp* pp, int k) {
  const PrimeTables& T = prime_tables(pp->primes[k]);
  HotPrime h;
  std::memcpy(h.tw, T.tw, sizeof(h.tw));
  h.omega = T.omega;
  h.omega_s = T.omega_s;
  LBG_CU(upload_hot(pp->pidx[k], h));
  DevPrime* D = new DevPrime();
  std::memcpy(D->lut, T.lut, sizeof(D->lut));
  std::memcpy(D->pow3_to_leaf, T.pow3_to_leaf, sizeof(D->pow3_to_leaf));
  std::memcpy(D->leaf_to_pow3, T.leaf_to_pow3, sizeof(D->leaf_to_pow3));
  std::memcpy(D->theta_leaf, T.theta_leaf, sizeof(D->theta_leaf));
  std::memcpy(D->key_rows, T.key_rows, sizeof(D->key_rows));
  std::memcpy(D->key_D, T.key_D, sizeof(D->key_D));
  uint64_t q = T.q;
  for (int L = 1; L <= 4; L++) {
    int cnt = 2;
    for (int l = 1; l < L; l++) cnt *= 3;
    for (int kk = 0; kk < cnt; kk++) {
      uint64_t zi = inv_mod(T.z_level[L][kk], q);
      D->zinv3[L][kk] = (uint32_t)(zi * T.inv3 % q);
      D->zinv3sq[L][kk] = (uint32_t)(zi * zi % q * T.inv3 % q);
      D->zfwd[L][kk] = T.z_level[L][kk];
    }
  }
  D->omega = T.omega;
  D->inv3 = T.inv3;
  D->zeta6 = T.zeta6;
  D->det0 = T.det0;
  std::memcpy(D->chal, T.chal_table.data(), sizeof(D->chal));
  cudaError_t e = cudaMalloc((void**)&pp->d_prime[k], sizeof(DevPrime));
  if (e == cudaSuccess) e = upload_sync(pp->d_prime[k], D, sizeof(DevPrime));
  delete D;
  if (e == cudaSuccess) {
    // the transform as the tensor-core operand, followed by the same T[m][v] as plain u16 rows
    // (TC_T16_BYTES: row v, m = 0..175, zero past 161) for the fold's operand builder
    std::vector<uint8_t> tcb(TC_B_BYTES + TC_T16_BYTES, 0);
    tc_transform_operand(T, tcb.data());
    uint16_t* t16 = reinterpret_cast<uint16_t*>(tcb.data() + TC_B_BYTES);
    for (int v = 0; v < N162; v++) {
      uint64_t x = 1;
      for (int m = 0; m < N162; m++) {
        t16[v * TC_LEAVES + m] = (uint16_t)x;
        x = x * T.theta_leaf[v] % T.q;
      }
    }
    e = cudaMalloc((void**)&pp->d_tcb[k], tcb.size());
    if (e == cudaSuccess) e = upload_sync(pp->d_tcb[k], tcb.data(), tcb.size());
  }
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("prime tables: ") + cudaGetErrorString(e));
  return LBG_OK;
}

void lbg_pp_retain(const lbg_pp* pp) { const_cast<lbg_pp*>(pp)->refs.fetch_add(1); }

static void pp_destroy(lbg_pp* pp);
void lbg_pp_release(const lbg_pp* pp) {
  lbg_pp* p = const_cast<lbg_pp*>(pp);
  if (p && p->refs.fetch_sub(1) == 1) pp_destroy(p);
}

// The caller's reference; the parameters go once the provers and batches made from them are freed.
void lbg_public_parameters_free(lbg_pp* pp) { lbg_pp_release(pp); }

static void pp_destroy(lbg_pp* pp) {
  cudaSetDevice(pp->device);
  if (pp->stream) cudaStreamSynchronize(pp->stream);
  cudaFree(pp->d_A);
  cudaFree(pp->d_Ahat);
  for (int k = 0; k < 7; k++) {
    cudaFree(pp->d_prime[k]);
    cudaFree(pp->d_tcb[k]);
  }
  cudaFree(pp->d_jumps);
  cudaFree(pp->d_eq);
  cudaFree(pp->d_p);
  cudaFree(pp->d_u);
  cudaFree(pp->d_out);
  cudaFree(pp->d_C);
  cudaFree(pp->d_ch);
  cudaFree(pp->d_chat);
  cudaFree(pp->d_fc);
  cudaFree(pp->d_wire);
  cudaFree(pp->d_lift);
  cudaFree(pp->d_vws);
  lbg_switch_release(pp);
  if (pp->stream) cudaStreamDestroy(pp->stream);
  delete pp;
}

int lbg_public_parameters_from_seed(const lbg_params* p, const uint8_t matrix_seed[32], lbg_pp** out) {
  if (!out || !matrix_seed) return fail(LBG_ERR_INVALID, "null argument");
  *out = nullptr;
  int rc = lbg_params_check(p);
  if (rc) return rc;
  lbg_pp* pp = new lbg_pp();
  pp->params = *p;
  pp->limbs = (int)p->n_moduli;
  for (int k = 0; k < pp->limbs; k++) {
    pp->primes[k] = p->moduli[k];
    pp->pidx[k] = prime_index(p->moduli[k]);
  }
  pp->cols = (size_t)1 << p->column_log_len;
  pp->wdim = (size_t)1 << (p->witness_log_len - p->column_log_len);
  pp->len_ring = pp->wdim / 4;
  pp->n = (size_t)1 << p->witness_log_len;
  std::memcpy(pp->seed, matrix_seed, 32);
  // crates/pcs/src/scheme/params.rs:321-322
  Blake3 h;
  h.update(matrix_seed, 32);
  uint8_t d[8];
  h.finalize(0, d, 8);
  uint64_t s = 0;
  for (int i = 7; i >= 0; i--) s = (s << 8) | d[i];
  pp->key_seed = s;

  auto bail = [&](int code) {
    lbg_public_parameters_free(pp);
    return code;
  };
  if (cudaGetDevice(&pp->device) != cudaSuccess) return bail(fail(LBG_ERR_CUDA, "no CUDA device"));
  if (cudaStreamCreateWithFlags(&pp->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(LBG_ERR_CUDA, "stream"));
  for (int k = 0; k < pp->limbs; k++)
    if ((rc = upload_prime(pp, k))) return bail(rc);
  const std::vector<uint64_t>& J = xorshift_jumps();
  size_t a_elems = (size_t)pp->limbs * pp->len_ring * N648;
  size_t ahat_elems = (size_t)pp->limbs * pp->len_ring * N162 * 2;
  if (cudaMalloc((void**)&pp->d_jumps, J.size() * 8) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_A, a_elems * 2) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_Ahat, ahat_elems * sizeof(int4)) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_eq, pp->wdim * 24) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_p, 64 * 24) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_u, pp->cols * 24) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_out, 64) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_C, pp->cols * 4 * pp->limbs * N162 * 2) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_ch, pp->cols * sizeof(lbg_challenge_d)) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_chat, pp->cols * N162 * 4) != cudaSuccess ||
      cudaMalloc((void**)&pp->d_fc, 4 * pp->limbs * N162 * 2) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(LBG_ERR_OOM, "public parameters: device allocation failed"));
  }
  if (cudaMemcpyAsync(pp->d_jumps, J.data(), J.size() * 8, cudaMemcpyHostToDevice, pp->stream) != cudaSuccess)
    return bail(fail(LBG_ERR_CUDA, "jump tables"));
  for (int k = 0; k < pp->limbs; k++) {
    // crates/pcs/src/key.rs:68 and crates/pcs/src/rng.rs:6-8
    uint64_t seed_k = pp->key_seed ^ (0x9E3779B9ull * (uint64_t)(k + 1));
    uint64_t state0 = (seed_k * 0x9E3779B97F4A7C15ull) | 1;
    int16_t* Ak = pp->d_A + (size_t)k * pp->len_ring * N648;
    if (launch_key_expand(pp->d_jumps, state0, pp->primes[k], (int)(pp->len_ring / 32), Ak, pp->stream) != cudaSuccess ||
        launch_key_components(pp->pidx[k], Ak, pp->d_prime[k], (int)pp->len_ring,
                              pp->d_Ahat + (size_t)k * pp->len_ring * N162 * 2, pp->stream) != cudaSuccess)
      return bail(fail(LBG_ERR_CUDA, std::string("key expansion: ") + cudaGetErrorString(cudaGetLastError())));
  }
  cudaError_t e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) return bail(fail(LBG_ERR_CUDA, std::string("key expansion: ") + cudaGetErrorString(e)));
  *out = pp;
  return LBG_OK;
}

int lbg_key_download(const lbg_pp* pp, int16_t* out) {
  if (!pp || !out) return fail(LBG_ERR_INVALID, "null argument");
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpy(out, pp->d_A, (size_t)pp->limbs * pp->len_ring * N648 * 2, cudaMemcpyDeviceToHost));
  return LBG_OK;
}

size_t lbg_pp_columns(const lbg_pp* pp) { return pp ? pp->cols : 0; }
size_t lbg_pp_len_ring(const lbg_pp* pp) { return pp ? pp->len_ring : 0; }
size_t lbg_pp_witness_len(const lbg_pp* pp) { return pp ? pp->n : 0; }
uint32_t lbg_pp_limbs(const lbg_pp* pp) { return pp ? (uint32_t)pp->limbs : 0; }

// ---------------------------------------------------------------------------------------------
// witnesses
// ---------------------------------------------------------------------------------------------
static int witness_alloc(const lbg_pp* pp, size_t n, lbg_witness** out) {
  lbg_witness* w = new lbg_witness();
  w->n = n;
  w->device = pp->device;
  w->d = witness_buf_get(pp->device, n * 24);
  if (!w->d) {
    delete w;
    return fail(LBG_ERR_OOM, "witness: device allocation failed");
  }
  *out = w;
  return LBG_OK;
}

int lbg_witness_from_host(const lbg_pp* pp, const uint64_t* f162, size_t n, lbg_witness** out) {
  if (!pp || !f162 || !out) return fail(LBG_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n != pp->n) return fail(LBG_ERR_WITNESS, "the witness is not witness_len() elements");
  LBG_CU(cudaSetDevice(pp->device));
  lbg_witness* w;
  int rc = witness_alloc(pp, n, &w);
  if (rc) return rc;
  if (upload_sync(w->d, f162, n * 24) != cudaSuccess) {
    witness_release(w);
    return fail(LBG_ERR_CUDA, "witness upload");
  }
  *out = w;
  return LBG_OK;
}

int lbg_witness_lifted(const lbg_pp* pp, const uint64_t* b128, size_t n, lbg_witness** out) {
  if (!pp || !b128 || !out) return fail(LBG_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n != pp->n) return fail(LBG_ERR_WITNESS, "the witness is not witness_len() elements");
  LBG_CU(cudaSetDevice(pp->device));
  lbg_witness* w;
  int rc = witness_alloc(pp, n, &w);
  if (rc) return rc;
  uint64_t* tmp = nullptr;
  cudaError_t e = cudaMalloc((void**)&tmp, n * 16);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, b128, n * 16, cudaMemcpyHostToDevice, pp->stream);
  if (e == cudaSuccess) e = launch_lift_b128(tmp, n, w->d, pp->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(pp->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) {
    witness_release(w);
    return fail(LBG_ERR_CUDA, std::string("lifted witness: ") + cudaGetErrorString(e));
  }
  *out = w;
  return LBG_OK;
}

int lbg_witness_random(const lbg_pp* pp, const uint8_t seed[32], lbg_witness** out) {
  if (!pp || !seed || !out) return fail(LBG_ERR_INVALID, "null argument");
  *out = nullptr;
  LBG_CU(cudaSetDevice(pp->device));
  lbg_witness* w;
  int rc = witness_alloc(pp, pp->n, &w);
  if (rc) return rc;
  // keyed BLAKE3 of "labinius/witness": one chunk, one block, so the XOF is the root node's
  // output blocks.
  XofRoot root;
  for (int i = 0; i < 8; i++)
    root.cv[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                 ((uint32_t)seed[4 * i + 3] << 24);
  uint8_t msg[64] = {0};
  std::memcpy(msg, "labinius/witness", 16);
  for (int i = 0; i < 16; i++)
    root.m[i] = (uint32_t)msg[4 * i] | ((uint32_t)msg[4 * i + 1] << 8) | ((uint32_t)msg[4 * i + 2] << 16) |
                ((uint32_t)msg[4 * i + 3] << 24);
  root.block_len = 16;
  root.flags = 16 | 1 | 2 | 8;  // keyed hash, chunk start, chunk end, root
  cudaError_t e = launch_xof_f162(root, pp->n, w->d, pp->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) {
    witness_release(w);
    return fail(LBG_ERR_CUDA, std::string("random witness: ") + cudaGetErrorString(e));
  }
  *out = w;
  return LBG_OK;
}

int lbg_witness_download(const lbg_witness* w, uint64_t* out, size_t n) {
  if (!w || !out) return fail(LBG_ERR_INVALID, "null argument");
  if (n != w->n) return fail(LBG_ERR_INVALID, "length mismatch");
  LBG_CU(cudaSetDevice(w->device));
  LBG_CU(cudaMemcpy(out, w->d, n * 24, cudaMemcpyDeviceToHost));
  return LBG_OK;
}

void lbg_witness_free(lbg_witness* w) { witness_release(w); }

// ---------------------------------------------------------------------------------------------
// prover
// ---------------------------------------------------------------------------------------------
// The commit's grid over `cols` columns: column tiles x ring-element chunks. A wave of the commit
// kernel is (SMs x resident CTAs) CTAs and its length is proportional to the chunk, so pick the
// chunk count that minimises waves x chunk (ties: fewer chunks, fewer partial sums), with at most
// max_partial chunk partials (chunks x cols) where the buffer is shared.
static void commit_chunking(const lbg_pp* pp, int cols, long max_partial, int* chunk_out, int* nchunks_out) {
  int col_tiles = (cols + commit_cols_per_cta() - 1) / commit_cols_per_cta();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pp->device);
  int slots = sms * commit_blocks_per_sm(pp->pidx[0]);
  int step = commit_ring_per_step();
  long best_cost = -1;
  int max_chunks = (int)((pp->len_ring + step - 1) / step);
  for (int nch = 1; nch <= max_chunks; nch++) {
    int chunk = (int)((pp->len_ring + nch - 1) / nch);
    chunk = (chunk + step - 1) / step * step;
    int nact = (int)((pp->len_ring + chunk - 1) / chunk);
    if ((long)nact * cols > max_partial) break;
    long total = (long)col_tiles * nact;
    long waves = (total + slots - 1) / slots;
    // the tensor-core kernel is persistent (its items run back to back on one CTA per SM): an item
    // costs its chunk plus about two ring elements, a chunk of partial sums about one
    long cost = commit_tc_enabled() ? waves * (chunk + 2) + nact : waves * chunk;
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      *chunk_out = chunk;
      *nchunks_out = nact;
    }
  }
}

static void free_bufs(OpeningBufs* b) {
  if (!b) return;
  cudaFree(b->d_C);
  cudaFree(b->d_top);
  cudaFree(b->d_digits);
  cudaFree(b->d_keep);
  delete b;
}

static void prover_destroy(lbg_prover* pr);
static void prover_release(lbg_prover* pr) {
  if (pr && pr->refs.fetch_sub(1) == 1) prover_destroy(pr);
}

// The caller's reference; the prover goes once its openings are freed or folded.
void lbg_prover_free(lbg_prover* pr) { prover_release(pr); }

static void prover_destroy(lbg_prover* pr) {
  const lbg_pp* pp = pr->pp;
  cudaSetDevice(pr->pp->device);
  if (pr->stream) cudaStreamSynchronize(pr->stream);
  if (pr->copy_stream) {
    cudaStreamSynchronize(pr->copy_stream);
    cudaStreamDestroy(pr->copy_stream);
  }
  for (auto e : pr->group_events) cudaEventDestroy(e);
  for (auto sl : pr->limb_streams) {
    cudaStreamSynchronize(sl);
    cudaStreamDestroy(sl);
  }
  for (auto e : pr->limb_done) cudaEventDestroy(e);
  for (auto* d : pr->limb_partial) cudaFree(d);
  for (int s = 0; s < lbg_prover::STAGES; s++) {
    if (pr->stage_copied[s]) cudaEventDestroy(pr->stage_copied[s]);
    if (pr->stage[s]) cudaFreeHost(pr->stage[s]);
  }
  delete pr->copy_pool;
  cudaFree(pr->d_partial);
  cudaFree(pr->d_vhat);
  cudaFree(pr->d_ch);
  cudaFree(pr->d_chat);
  cudaFree(pr->d_v);
  cudaFree(pr->d_wire);
  cudaFree(pr->d_rec);
  cudaFree(pr->d_gm);
  cudaFree(pr->d_res);
  for (auto* b : pr->spare) free_bufs(b);
  for (auto& m : pr->marks) {
    cudaEventDestroy(m.a);
    cudaEventDestroy(m.b);
  }
  for (auto e : pr->event_pool) cudaEventDestroy(e);
  if (pr->stream) cudaStreamDestroy(pr->stream);
  delete pr;
  lbg_pp_release(pp);
}

// The kept transform of an opening, when the prover keeps it and the device has the room
// (otherwise the fold transforms the witness again).
static void attach_keep(const lbg_prover* pr, OpeningBufs* b) {
  if (!pr->keep) {
    cudaFree(b->d_keep);
    b->d_keep = nullptr;
  } else if (!b->d_keep && cudaMalloc((void**)&b->d_keep, pr->pp->n * N162 * 2) != cudaSuccess) {
    cudaGetLastError();
    b->d_keep = nullptr;
  }
}

static int get_bufs(lbg_prover* pr, OpeningBufs** out) {
  {
    std::lock_guard<std::mutex> g(pr->mu);
    if (!pr->spare.empty()) {
      *out = pr->spare.back();
      pr->spare.pop_back();
      attach_keep(pr, *out);
      return LBG_OK;
    }
  }
  const lbg_pp* pp = pr->pp;
  OpeningBufs* b = new OpeningBufs();
  size_t count = pp->cols * N648;
  if (cudaMalloc((void**)&b->d_C, pp->cols * 4 * pp->limbs * N162 * 2) != cudaSuccess ||
      cudaMalloc((void**)&b->d_top, count * 2) != cudaSuccess ||
      cudaMalloc((void**)&b->d_digits, (pp->limbs > 1 ? pp->limbs - 1 : 1) * count * 2) != cudaSuccess) {
    cudaGetLastError();
    free_bufs(b);
    return fail(LBG_ERR_OOM, "opening: device allocation failed");
  }
  attach_keep(pr, b);
  *out = b;
  return LBG_OK;
}

int lbg_prover_set_kept_transform(lbg_prover* pr, int enable) {
  if (!pr) return fail(LBG_ERR_INVALID, "null prover");
  LBG_CU(cudaSetDevice(pr->pp->device));
  LBG_CU(cudaStreamSynchronize(pr->stream));
  std::lock_guard<std::mutex> g(pr->mu);
  pr->keep = enable != 0;
  for (OpeningBufs* b : pr->spare) attach_keep(pr, b);
  return LBG_OK;
}

int lbg_prover_new(const lbg_pp* pp, lbg_prover** out) {
  if (!pp || !out) return fail(LBG_ERR_INVALID, "null argument");
  *out = nullptr;
  LBG_CU(cudaSetDevice(pp->device));
  lbg_prover* pr = new lbg_prover();
  pr->pp = pp;
  lbg_pp_retain(pp);  // released when the prover goes
  auto bail = [&](int code) {
    lbg_prover_free(pr);
    return code;
  };
  if (cudaStreamCreateWithFlags(&pr->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(LBG_ERR_CUDA, "stream"));
  // Grid: column tiles x ring-element chunks. A wave of the commit kernel is (SMs x resident CTAs)
  // CTAs and its length is proportional to the chunk, so pick the chunk count that minimises
  // waves x chunk (ties: fewer chunks, fewer partial sums).
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pp->device);
  commit_chunking(pp, (int)pp->cols, 1 << 30, &pr->chunk, &pr->nchunks);
  // the fold: position tiles x column splits, chosen the same way (the tensor-core kernel: 128
  // positions per work item, one CTA per SM, one column a step)
  {
    const bool ftc = fold_tc_enabled();
    const int fpos = ftc ? fold_tc_positions_per_cta() : fold_positions_per_cta();
    int tiles = (int)((pp->wdim + fpos - 1) / fpos);
    int fslots = sms * (ftc ? 1 : fold_blocks_per_sm(pp->pidx[0]));
    int fstep = ftc ? 1 : fold_cols_per_step();
    long best = -1;
    int max_splits = (int)((pp->cols + fstep - 1) / fstep);
    for (int ns = 1; ns <= max_splits; ns++) {
      int per = (int)((pp->cols + ns - 1) / ns);
      per = (per + fstep - 1) / fstep * fstep;
      int nact = (int)((pp->cols + per - 1) / per);
      long total = (long)tiles * nact;
      // the tensor-core kernel runs its items back to back: an item costs its columns plus about
      // two more (its sums added into vhat)
      long cost = ((total + fslots - 1) / fslots) * (per + (ftc ? 2 : 0));
      if (best < 0 || cost < best) {
        best = cost;
        pr->fold_cols_per_split = per;
      }
    }
  }
  size_t count = pp->cols * N648;
  if (cudaMalloc((void**)&pr->d_partial, (size_t)pr->nchunks * pp->cols * N162 * 16) != cudaSuccess ||
      cudaMalloc((void**)&pr->d_vhat, pp->wdim * N162 * 4) != cudaSuccess ||
      cudaMalloc((void**)&pr->d_ch, pp->cols * sizeof(lbg_challenge_d)) != cudaSuccess ||
      cudaMalloc((void**)&pr->d_chat, pp->cols * N162 * 4) != cudaSuccess ||
      cudaMalloc((void**)&pr->d_v, pp->len_ring * N648 * 2) != cudaSuccess ||
      cudaMalloc((void**)&pr->d_res, (size_t)pp->limbs * count * 2) != cudaSuccess ||
      (fold_gm_enabled() && pp->cols <= LBG_FOLD_GM_MAX_COLUMNS &&
       cudaMalloc((void**)&pr->d_gm, fold_gm_operand_bytes(pp->cols)) != cudaSuccess)) {
    cudaGetLastError();
    return bail(fail(LBG_ERR_OOM, "prover workspace: device allocation failed"));
  }
  // warm-up: one commitment and one fold of a zero witness (crates/pcs/src/scheme/prover.rs:31-53)
  lbg_witness* zw = nullptr;
  int rc = witness_alloc(pp, pp->n, &zw);
  if (rc) return bail(rc);
  if (cudaMemsetAsync(zw->d, 0, pp->n * 24, pr->stream) != cudaSuccess) {
    witness_release(zw);
    return bail(fail(LBG_ERR_CUDA, "warm-up"));
  }
  lbg_opening* op = nullptr;
  rc = lbg_commit(pr, zw, nullptr, nullptr, nullptr, &op);
  witness_release(zw);
  if (rc) return bail(rc);
  std::vector<lbg_challenge> zero(pp->cols);
  std::memset(zero.data(), 0, zero.size() * sizeof(lbg_challenge));
  rc = lbg_fold(pr, op, zero.data(), pp->cols, nullptr);
  if (rc) return bail(rc);
  if (cudaStreamSynchronize(pr->stream) != cudaSuccess) return bail(fail(LBG_ERR_CUDA, "warm-up sync"));
  *out = pr;
  return LBG_OK;
}

void* lbg_prover_stream(const lbg_prover* pr) { return pr ? (void*)pr->stream : nullptr; }

int lbg_prover_profile(lbg_prover* pr, int enable) {
  if (!pr) return fail(LBG_ERR_INVALID, "null prover");
  LBG_CU(cudaSetDevice(pr->pp->device));
  LBG_CU(cudaStreamSynchronize(pr->stream));
  for (auto& m : pr->marks) {
    pr->event_pool.push_back(m.a);
    pr->event_pool.push_back(m.b);
  }
  pr->marks.clear();
  pr->profiling = enable != 0;
  return LBG_OK;
}

int lbg_prover_kernel_stats(lbg_prover* pr, const char* kernel, uint64_t* launches, double* total_ms) {
  if (!pr || !kernel) return fail(LBG_ERR_INVALID, "null argument");
  LBG_CU(cudaSetDevice(pr->pp->device));
  LBG_CU(cudaStreamSynchronize(pr->stream));
  uint64_t n = 0;
  double ms = 0;
  for (auto& m : pr->marks) {
    if (std::strcmp(m.name, kernel) != 0) continue;
    float t = 0;
    LBG_CU(cudaEventElapsedTime(&t, m.a, m.b));
    n++;
    ms += t;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return LBG_OK;
}

uint64_t lbg_prover_launch_count(const lbg_prover* pr) { return pr ? pr->launches : 0; }
int lbg_prover_sync(lbg_prover* pr) {
  if (!pr) return fail(LBG_ERR_INVALID, "null prover");
  LBG_CU(cudaStreamSynchronize(pr->stream));
  return LBG_OK;
}

// ---------------------------------------------------------------------------------------------
// commit
// ---------------------------------------------------------------------------------------------
int lbg_commit(lbg_prover* pr, const lbg_witness* w, int16_t* matrix_out, uint16_t* top_out,
               uint16_t* digits_out, lbg_opening** opening_out) {
  if (!pr || !w) return fail(LBG_ERR_INVALID, "null argument");
  const lbg_pp* pp = pr->pp;
  if (w->n != pp->n) return fail(LBG_ERR_INVALID, "the witness was built for other parameters");
  LBG_CU(cudaSetDevice(pp->device));
  OpeningBufs* b = nullptr;
  int rc = get_bufs(pr, &b);
  if (rc) return rc;
  cudaStream_t st = pr->stream;
  int cols = (int)pp->cols, L = pp->limbs;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < L && e == cudaSuccess; k++) {
    {
      KernelScope ks(pr, "commit");
      e = launch_commit(pp->pidx[k], w->d, pp->wdim, pp->d_Ahat + (size_t)k * pp->len_ring * N162 * 2,
                        pp->d_prime[k], cols, (int)pp->len_ring, pr->chunk, pr->nchunks, pr->d_partial, st,
                        k == 0 ? b->d_keep : nullptr, pp->d_tcb[k]);
    }
    if (e == cudaSuccess) {
      KernelScope ks(pr, "commit_finish");
      e = launch_commit_finish(pp->pidx[k], pr->d_partial, pr->nchunks, cols, pp->d_prime[k], k, L, b->d_C, st);
    }
  }
  bool bd = pp->params.opening == LBG_OPENING_BIT_DROPPED;
  size_t count = pp->cols * N648;
  if (bd && e == cudaSuccess) {
    for (int k = 0; k < L && e == cudaSuccess; k++) {
      KernelScope ks(pr, "column_residues");
      e = launch_column_residues(pp->pidx[k], b->d_C, cols, k, L, pp->d_prime[k], pr->d_res + (size_t)k * count, st);
    }
    if (e == cudaSuccess) {
      GarnerConsts g;
      std::memset(&g, 0, sizeof(g));
      for (int k = 0; k < L; k++) {
        g.q[k] = pp->primes[k];
        for (int m = 0; m < k; m++) g.inv[k][m] = (uint32_t)inv_mod(pp->primes[m], pp->primes[k]);
      }
      g.dropped_bits = pp->params.dropped_bits;
      KernelScope ks(pr, "garner");
      e = launch_garner(pr->d_res, count, L, g, b->d_top, b->d_digits, st);
    }
  }
  if (e == cudaSuccess && matrix_out && !bd)
    e = cudaMemcpyAsync(matrix_out, b->d_C, pp->cols * 4 * L * N162 * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && bd && top_out) e = cudaMemcpyAsync(top_out, b->d_top, count * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && bd && digits_out && L > 1)
    e = cudaMemcpyAsync(digits_out, b->d_digits, (size_t)(L - 1) * count * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && (matrix_out || top_out || digits_out)) e = tc_checked(cudaStreamSynchronize(st));
  if (e != cudaSuccess) {
    std::lock_guard<std::mutex> g(pr->mu);
    pr->spare.push_back(b);
    return fail(LBG_ERR_CUDA, std::string("commit: ") + cudaGetErrorString(e));
  }
  lbg_opening* op = new lbg_opening();
  op->pr = pr;
  pr->refs.fetch_add(1);
  op->w = const_cast<lbg_witness*>(w);
  op->w->refs.fetch_add(1);
  op->bufs = b;
  if (opening_out)
    *opening_out = op;
  else
    lbg_opening_free(op);
  return LBG_OK;
}

// Whether host memory `p` is pageable (not page-locked or registered with CUDA).
static bool host_pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// The staging ring of lbg_commit_host for pageable witnesses: STAGES page-locked buffers of at
// least `bytes`, their copy events, and the host copy threads. Waits for any copy still reading
// the buffers (a previous call's) before they are handed out again.
static int stage_ready(lbg_prover* pr, size_t bytes) {
  for (int s = 0; s < lbg_prover::STAGES; s++)
    if (pr->stage_copied[s]) LBG_CU(cudaEventSynchronize(pr->stage_copied[s]));
  if (pr->stage_bytes < bytes) {
    for (int s = 0; s < lbg_prover::STAGES; s++) {
      if (pr->stage[s]) cudaFreeHost(pr->stage[s]);
      pr->stage[s] = nullptr;
    }
    pr->stage_bytes = 0;
    for (int s = 0; s < lbg_prover::STAGES; s++)
      if (cudaHostAlloc(&pr->stage[s], bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        for (int t = 0; t <= s; t++) {
          if (pr->stage[t]) cudaFreeHost(pr->stage[t]);
          pr->stage[t] = nullptr;
        }
        return fail(LBG_ERR_OOM, "page-locked staging buffers");
      }
    pr->stage_bytes = bytes;
  }
  for (int s = 0; s < lbg_prover::STAGES; s++)
    if (!pr->stage_copied[s] && cudaEventCreateWithFlags(&pr->stage_copied[s], cudaEventDisableTiming) != cudaSuccess)
      return fail(LBG_ERR_CUDA, "event");
  if (!pr->copy_pool) {
    unsigned hc = std::thread::hardware_concurrency();
    // half the host's threads (8 of 16 on the bench host: 14 copied the witness 1.2x slower)
    int workers = hc >= 16 ? 7 : hc >= 4 ? (int)hc / 2 - 1 : 0;
    pr->copy_pool = new lbg::CopyPool(workers);
  }
  return LBG_OK;
}

// Witness::from_elements + Prover::commit with the upload pipelined against the commit: the
// witness arrives in column groups on the prover's copy stream, and every limb's commit of a
// group starts on the compute stream as soon as that group has landed. Page-locked host memory is
// copied to the device directly; pageable memory (a Rust Vec, a numpy array) passes group by
// group through a ring of page-locked staging buffers, each filled by several host threads while
// the device copies the previous group out and commits the ones before. The results are those of
// lbg_witness_from_host + lbg_commit.
int lbg_commit_host(lbg_prover* pr, const uint64_t* f162, size_t n, int16_t* matrix_out, uint16_t* top_out,
                    uint16_t* digits_out, lbg_witness** w_out, lbg_opening** opening_out) {
  if (!pr || !f162 || !w_out) return fail(LBG_ERR_INVALID, "null argument");
  *w_out = nullptr;
  if (opening_out) *opening_out = nullptr;
  const lbg_pp* pp = pr->pp;
  if (n != pp->n) return fail(LBG_ERR_WITNESS, "the witness is not witness_len() elements");
  LBG_CU(cudaSetDevice(pp->device));
  const int cols = (int)pp->cols, L = pp->limbs;
  // column groups of at least 64 columns, at most 8; the first one split in two halves, so that the
  // commit starts after half a group's copy
  int ngroups = 1;
  while (ngroups < 8 && cols / (2 * ngroups) >= 64) ngroups *= 2;
  const int gc = cols / ngroups;
  std::vector<int> gstart, gcols;  // the groups' first columns and widths
  if (ngroups > 1) {
    gstart = {0, gc / 2};
    gcols = {gc / 2, gc / 2};
  } else {
    gstart = {0};
    gcols = {gc};
  }
  for (int g = 1; g < ngroups; g++) {
    gstart.push_back(g * gc);
    gcols.push_back(gc);
  }
  const int groups = (int)gstart.size();
  // the chunking of each group width
  int chunk = pr->chunk, nch = pr->nchunks, chunk_h = pr->chunk, nch_h = pr->nchunks;
  if (ngroups > 1) {
    commit_chunking(pp, gc, (long)pr->nchunks * cols, &chunk, &nch);
    commit_chunking(pp, gc / 2, (long)pr->nchunks * cols, &chunk_h, &nch_h);
  }
  if (!pr->copy_stream && cudaStreamCreateWithFlags(&pr->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(LBG_ERR_CUDA, "copy stream");
  while ((int)pr->group_events.size() < groups) {
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail(LBG_ERR_CUDA, "event");
    pr->group_events.push_back(ev);
  }
  // a limb's stream, event and partials are made together and kept only when all three exist, so
  // the three lists always have the same length
  while ((int)pr->limb_streams.size() < L - 1) {
    cudaStream_t sl = nullptr;
    cudaEvent_t ev = nullptr;
    int32_t* part = nullptr;
    if (cudaStreamCreateWithFlags(&sl, cudaStreamNonBlocking) != cudaSuccess) return fail(LBG_ERR_CUDA, "limb stream");
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaStreamDestroy(sl);
      return fail(LBG_ERR_CUDA, "event");
    }
    if (cudaMalloc((void**)&part, (size_t)pr->nchunks * pp->cols * N162 * 16) != cudaSuccess) {
      cudaEventDestroy(ev);
      cudaStreamDestroy(sl);
      return fail(LBG_ERR_OOM, "limb partials");
    }
    pr->limb_streams.push_back(sl);
    pr->limb_done.push_back(ev);
    pr->limb_partial.push_back(part);
  }
  if (pr->limb_done.size() != pr->limb_streams.size() || pr->limb_partial.size() != pr->limb_streams.size())
    return fail(LBG_ERR_INVALID, "limb streams, events and partials out of step");
  lbg_witness* w;
  int rc = witness_alloc(pp, n, &w);
  if (rc) return rc;
  OpeningBufs* b = nullptr;
  rc = get_bufs(pr, &b);
  if (rc) {
    witness_release(w);
    return rc;
  }
  cudaStream_t st = pr->stream, cp = pr->copy_stream;
  const size_t per_col = pp->wdim * 3;  // u64 words of a column
  const size_t group_bytes = (size_t)gc * per_col * 8;  // the widest group's
  const bool pageable = host_pageable(f162);
  if (pageable) {
    rc = stage_ready(pr, group_bytes);
    if (rc) {
      std::lock_guard<std::mutex> g(pr->mu);
      pr->spare.push_back(b);
      witness_release(w);
      return rc;
    }
  }
  cudaError_t e = cudaSuccess;
  for (int g = 0; g < groups && e == cudaSuccess; g++) {
    const size_t c0 = (size_t)gstart[g];
    const int gw = gcols[g];
    const int gch = gw == gc ? chunk : chunk_h, gnch = gw == gc ? nch : nch_h;
    const size_t gbytes = (size_t)gw * per_col * 8;
    if (pageable) {
      // stage g % STAGES is free once the device copy of group g - STAGES out of it has finished
      const int s = g % lbg_prover::STAGES;
      e = cudaEventSynchronize(pr->stage_copied[s]);
      if (e != cudaSuccess) break;
      pr->copy_pool->copy(pr->stage[s], f162 + c0 * per_col, gbytes);
      e = cudaMemcpyAsync(w->d + c0 * per_col, pr->stage[s], gbytes, cudaMemcpyHostToDevice, cp);
      if (e == cudaSuccess) e = cudaEventRecord(pr->stage_copied[s], cp);
    } else {
      e = cudaMemcpyAsync(w->d + c0 * per_col, f162 + c0 * per_col, gbytes, cudaMemcpyHostToDevice, cp);
    }
    if (e == cudaSuccess) e = cudaEventRecord(pr->group_events[g], cp);
    for (int k = 0; k < L && e == cudaSuccess; k++) {
      // limb 0 on the prover's stream (bracketed for the profile), limb k >= 1 on its own
      cudaStream_t sk = k == 0 ? st : pr->limb_streams[k - 1];
      int32_t* part = k == 0 ? pr->d_partial : pr->limb_partial[k - 1];
      e = cudaStreamWaitEvent(sk, pr->group_events[g], 0);
      if (e != cudaSuccess) break;
      if (k == 0) {
        KernelScope ks(pr, "commit");
        e = launch_commit(pp->pidx[k], w->d + c0 * per_col, pp->wdim, pp->d_Ahat + (size_t)k * pp->len_ring * N162 * 2,
                          pp->d_prime[k], gw, (int)pp->len_ring, gch, gnch, part, sk,
                          b->d_keep ? b->d_keep + c0 * pp->wdim * N162 : nullptr, pp->d_tcb[k]);
      } else {
        pr->launches += 1;
        e = launch_commit(pp->pidx[k], w->d + c0 * per_col, pp->wdim, pp->d_Ahat + (size_t)k * pp->len_ring * N162 * 2,
                          pp->d_prime[k], gw, (int)pp->len_ring, gch, gnch, part, sk, nullptr, pp->d_tcb[k]);
      }
      if (e != cudaSuccess) break;
      if (k == 0) {
        KernelScope ks(pr, "commit_finish");
        e = launch_commit_finish(pp->pidx[k], part, gnch, gw, pp->d_prime[k], k, L, b->d_C + c0 * 4 * L * N162, sk);
      } else {
        pr->launches += 1;
        e = launch_commit_finish(pp->pidx[k], part, gnch, gw, pp->d_prime[k], k, L, b->d_C + c0 * 4 * L * N162, sk);
      }
    }
  }
  // the prover's stream goes on once every limb stream has finished its groups
  for (int k = 1; k < L && e == cudaSuccess; k++) {
    e = cudaEventRecord(pr->limb_done[k - 1], pr->limb_streams[k - 1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, pr->limb_done[k - 1], 0);
  }
  bool bd = pp->params.opening == LBG_OPENING_BIT_DROPPED;
  size_t count = pp->cols * N648;
  if (bd && e == cudaSuccess) {
    for (int k = 0; k < L && e == cudaSuccess; k++) {
      KernelScope ks(pr, "column_residues");
      e = launch_column_residues(pp->pidx[k], b->d_C, cols, k, L, pp->d_prime[k], pr->d_res + (size_t)k * count, st);
    }
    if (e == cudaSuccess) {
      GarnerConsts gcs;
      std::memset(&gcs, 0, sizeof(gcs));
      for (int k = 0; k < L; k++) {
        gcs.q[k] = pp->primes[k];
        for (int m = 0; m < k; m++) gcs.inv[k][m] = (uint32_t)inv_mod(pp->primes[m], pp->primes[k]);
      }
      gcs.dropped_bits = pp->params.dropped_bits;
      KernelScope ks(pr, "garner");
      e = launch_garner(pr->d_res, count, L, gcs, b->d_top, b->d_digits, st);
    }
  }
  if (e == cudaSuccess && matrix_out && !bd)
    e = cudaMemcpyAsync(matrix_out, b->d_C, pp->cols * 4 * L * N162 * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && bd && top_out) e = cudaMemcpyAsync(top_out, b->d_top, count * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && bd && digits_out && L > 1)
    e = cudaMemcpyAsync(digits_out, b->d_digits, (size_t)(L - 1) * count * 2, cudaMemcpyDeviceToHost, st);
  // the witness is complete once the compute stream has passed every group's event
  if (e == cudaSuccess) e = tc_checked(cudaStreamSynchronize(st));
  if (e != cudaSuccess) {
    cudaStreamSynchronize(cp);
    for (auto sl : pr->limb_streams) cudaStreamSynchronize(sl);
    {
      std::lock_guard<std::mutex> g(pr->mu);
      pr->spare.push_back(b);
    }
    witness_release(w);
    return fail(LBG_ERR_CUDA, std::string("commit: ") + cudaGetErrorString(e));
  }
  lbg_opening* op = new lbg_opening();
  op->pr = pr;
  pr->refs.fetch_add(1);
  op->w = w;
  w->refs.fetch_add(1);
  op->bufs = b;
  if (opening_out)
    *opening_out = op;
  else
    lbg_opening_free(op);
  *w_out = w;
  return LBG_OK;
}

int lbg_device_memory(const lbg_pp* pp, size_t* free_bytes, size_t* total_bytes) {
  if (!pp || !free_bytes || !total_bytes) return fail(LBG_ERR_INVALID, "null argument");
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemGetInfo(free_bytes, total_bytes));
  return LBG_OK;
}

int lbg_opening_matrix(const lbg_opening* op, int16_t* matrix_out) {
  if (!op || !matrix_out) return fail(LBG_ERR_INVALID, "null argument");
  const lbg_pp* pp = op->pr->pp;
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpyAsync(matrix_out, op->bufs->d_C, pp->cols * 4 * pp->limbs * N162 * 2, cudaMemcpyDeviceToHost,
                         op->pr->stream));
  LBG_CU(cudaStreamSynchronize(op->pr->stream));
  return LBG_OK;
}

int lbg_opening_dropped(const lbg_opening* op, uint16_t* top_out, uint16_t* digits_out) {
  if (!op) return fail(LBG_ERR_INVALID, "null argument");
  const lbg_pp* pp = op->pr->pp;
  if (pp->params.opening != LBG_OPENING_BIT_DROPPED) return fail(LBG_ERR_INVALID, "this commitment is not bit-dropped");
  size_t count = pp->cols * N648;
  LBG_CU(cudaSetDevice(pp->device));
  if (top_out) LBG_CU(cudaMemcpyAsync(top_out, op->bufs->d_top, count * 2, cudaMemcpyDeviceToHost, op->pr->stream));
  if (digits_out && pp->limbs > 1)
    LBG_CU(cudaMemcpyAsync(digits_out, op->bufs->d_digits, (size_t)(pp->limbs - 1) * count * 2,
                           cudaMemcpyDeviceToHost, op->pr->stream));
  LBG_CU(cudaStreamSynchronize(op->pr->stream));
  return LBG_OK;
}

// Grows a device buffer to at least `bytes` (contents not kept).
static int grow(void** buf, size_t* cap, size_t bytes) {
  if (*cap >= bytes) return LBG_OK;
  cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  if (cudaMalloc(buf, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(LBG_ERR_OOM, "device buffer");
  }
  *cap = bytes;
  return LBG_OK;
}

// recursion::limbs::residues (crates/pcs/src/recursion/limbs.rs:379-398) of the opening's commitment,
// computed on the device from where the commit left it: per limb, the columns' coefficients
// (k_column_residues), then the four component vectors of chunked, signed, centred coefficients.
int lbg_opening_residues(const lbg_opening* op, size_t polys, int16_t* out) {
  if (!op || !out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_prover* pr = op->pr;
  const lbg_pp* pp = pr->pp;
  if (pp->params.opening == LBG_OPENING_BIT_DROPPED)
    return fail(LBG_ERR_INVALID, "a bit-dropped commitment keeps no matrix to take residues of");
  const int cols = (int)pp->cols, L = pp->limbs;
  if (polys < (size_t)3 * cols) return fail(LBG_ERR_INVALID, "fewer polynomials than 3 x columns");
  LBG_CU(cudaSetDevice(pp->device));
  std::lock_guard<std::mutex> g(pr->mu);
  const size_t per_limb = 4 * polys * 64;
  int rc = grow((void**)&pr->d_rec, &pr->rec_cap, (size_t)L * per_limb * 2);
  if (rc) return rc;
  const size_t count = pp->cols * N648;
  cudaStream_t st = pr->stream;
  for (int k = 0; k < L; k++) {
    LBG_CU(launch_column_residues(pp->pidx[k], op->bufs->d_C, cols, k, L, pp->d_prime[k], pr->d_res + (size_t)k * count,
                                  st));
    LBG_CU(launch_recursion_residues(pr->d_res + (size_t)k * count, cols, polys, pp->primes[k],
                                     pr->d_rec + (size_t)k * per_limb, st));
  }
  pr->launches += 2 * L;
  LBG_CU(cudaMemcpyAsync(out, pr->d_rec, (size_t)L * per_limb * 2, cudaMemcpyDeviceToHost, st));
  LBG_CU(cudaStreamSynchronize(st));
  return LBG_OK;
}

// Prover::commit_left_expansion's vector u (crates/pcs/src/scheme/prover.rs:95-115) on the device.
int lbg_left_expansion(const lbg_pp* pp_c, const uint64_t* row_values, size_t cols, size_t rank, int16_t* out) {
  if (!pp_c || !row_values || !out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (cols != pp->cols) return fail(LBG_ERR_INVALID, "the row evaluation does not match the parameters");
  if (rank < 3 * cols) return fail(LBG_ERR_INVALID, "fewer polynomials than 3 x columns");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  int rc = grow((void**)&pp->d_lift, &pp->lift_cap, rank * 64 * 2);
  if (rc) return rc;
  LBG_CU(cudaMemcpyAsync(pp->d_u, row_values, cols * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_left_expansion(pp->d_u, (int)cols, rank, pp->d_lift, pp->stream));
  LBG_CU(cudaMemcpyAsync(out, pp->d_lift, rank * 64 * 2, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return LBG_OK;
}

void lbg_opening_free(lbg_opening* op) {
  if (!op) return;
  lbg_prover* pr = op->pr;
  {
    std::lock_guard<std::mutex> g(pr->mu);
    pr->spare.push_back(op->bufs);
  }
  // the last reference frees the witness with cudaFree, which waits for the device first
  cudaSetDevice(pr->pp->device);
  witness_release(op->w);
  delete op;
  prover_release(pr);
}

// ---------------------------------------------------------------------------------------------
// evaluation
// ---------------------------------------------------------------------------------------------
int lbg_row_evaluate(const lbg_pp* pp_c, const lbg_witness* w, const uint64_t* p0, size_t p0_len, uint64_t* u_out) {
  if (!pp_c || !w || !p0 || !u_out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (p0_len != (size_t)(pp->params.witness_log_len - pp->params.column_log_len) || w->n != pp->n)
    return fail(LBG_ERR_INVALID, "the evaluation point does not match the witness");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpyAsync(pp->d_p, p0, p0_len * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_eq_table(pp->d_p, (int)p0_len, pp->wdim, pp->d_eq, pp->stream));
  LBG_CU(launch_row_eval(w->d, pp->wdim, (int)pp->cols, pp->d_eq, pp->d_u, pp->stream));
  LBG_CU(cudaMemcpyAsync(u_out, pp->d_u, pp->cols * 24, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return LBG_OK;
}

int lbg_mle_evaluate(const lbg_pp* pp_c, const lbg_witness* w, const uint64_t* p0, size_t p0_len, const uint64_t* p1,
                     size_t p1_len, uint64_t out[3]) {
  if (!pp_c || !w || !p0 || !p1 || !out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (p0_len != (size_t)(pp->params.witness_log_len - pp->params.column_log_len) ||
      p1_len != (size_t)pp->params.column_log_len || w->n != pp->n)
    return fail(LBG_ERR_INVALID, "the evaluation point does not match the witness");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpyAsync(pp->d_p, p0, p0_len * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(cudaMemcpyAsync(pp->d_p + 3 * 32, p1, p1_len * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_eq_table(pp->d_p, (int)p0_len, pp->wdim, pp->d_eq, pp->stream));
  LBG_CU(launch_row_eval(w->d, pp->wdim, (int)pp->cols, pp->d_eq, pp->d_u, pp->stream));
  LBG_CU(launch_claim(pp->d_u, (int)pp->cols, pp->d_p + 3 * 32, (int)p1_len, pp->d_out, pp->stream));
  LBG_CU(cudaMemcpyAsync(out, pp->d_out, 24, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return LBG_OK;
}

// ---------------------------------------------------------------------------------------------
// fold
// ---------------------------------------------------------------------------------------------
int lbg_fold(lbg_prover* pr, lbg_opening* op, const lbg_challenge* challenges, size_t r, int16_t* v_out) {
  if (!pr || !op) return fail(LBG_ERR_INVALID, "null argument");
  const lbg_pp* pp = pr->pp;
  int rc = LBG_OK;
  if (op->pr != pr) rc = fail(LBG_ERR_INVALID, "the opening belongs to another prover");
  else if (!challenges || r != pp->cols) rc = fail(LBG_ERR_INVALID, "one challenge per column");
  if (rc) {
    lbg_opening_free(op);
    return rc;
  }
  cudaSetDevice(pp->device);
  cudaStream_t st = pr->stream;
  cudaError_t e = cudaMemcpyAsync(pr->d_ch, challenges, r * sizeof(lbg_challenge), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    KernelScope ks(pr, "challenge_slots");
    e = launch_challenge_slots(pp->pidx[0], pr->d_ch, (int)r, pp->d_prime[0], pr->d_chat, st);
  }
  if (e == cudaSuccess) {
    // k_fold_operand + k_fold_gm + k_fold_finish_t, or k_fold_tc (k_fold, k_fold_kept) + the finish
    KernelScope ks(pr, "fold", (pr->d_gm && !op->bufs->d_keep) ? 3 : 2);
    if (op->bufs->d_keep)
      e = launch_fold_kept(pp->pidx[0], op->bufs->d_keep, pp->wdim, (int)pp->cols, pr->fold_cols_per_split,
                           pr->d_chat, pp->d_prime[0], pr->d_vhat, pr->d_v, st);
    else if (pr->d_gm)
      e = launch_fold_gm(pp->pidx[0], op->w->d, pp->wdim, (int)pp->cols, pr->fold_cols_per_split, pr->d_chat,
                         pp->d_tcb[0], pr->d_gm, pp->d_prime[0], pr->d_vhat, pr->d_v, st);
    else
      e = launch_fold(pp->pidx[0], op->w->d, pp->wdim, (int)pp->cols, pr->fold_cols_per_split, pr->d_chat,
                      pp->d_prime[0], pr->d_vhat, pr->d_v, st, 1, nullptr, pp->d_tcb[0]);
  }
  if (e == cudaSuccess && v_out) e = cudaMemcpyAsync(v_out, pr->d_v, pp->len_ring * N648 * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && v_out) e = cudaStreamSynchronize(st);
  lbg_opening_free(op);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("fold: ") + cudaGetErrorString(e));
  return LBG_OK;
}

int lbg_prover_folded(const lbg_prover* pr, int16_t* v_out) {
  if (!pr || !v_out) return fail(LBG_ERR_INVALID, "null argument");
  LBG_CU(cudaSetDevice(pr->pp->device));
  LBG_CU(cudaMemcpyAsync(v_out, pr->d_v, pr->pp->len_ring * N648 * 2, cudaMemcpyDeviceToHost, pr->stream));
  LBG_CU(cudaStreamSynchronize(pr->stream));
  return LBG_OK;
}

int lbg_fold_commitment(const lbg_pp* pp_c, const int16_t* matrix, size_t columns, const lbg_challenge* challenges,
                        size_t r, int16_t* out) {
  if (!pp_c || !matrix || !challenges || !out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (columns != pp->cols || r != columns) return fail(LBG_ERR_INVALID, "one challenge per column");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  int L = pp->limbs;
  LBG_CU(cudaMemcpyAsync(pp->d_C, matrix, pp->cols * 4 * L * N162 * 2, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(cudaMemcpyAsync(pp->d_ch, challenges, r * sizeof(lbg_challenge), cudaMemcpyHostToDevice, pp->stream));
  for (int k = 0; k < L; k++) {
    LBG_CU(launch_challenge_slots(pp->pidx[k], pp->d_ch, (int)r, pp->d_prime[k], pp->d_chat, pp->stream));
    LBG_CU(launch_fold_commitment(pp->pidx[k], pp->d_C, (int)pp->cols, k, L, pp->d_chat, pp->d_prime[k], pp->d_fc,
                                  pp->stream));
  }
  LBG_CU(cudaMemcpyAsync(out, pp->d_fc, 4 * L * N162 * 2, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return LBG_OK;
}

// ---------------------------------------------------------------------------------------------
// verifier
// ---------------------------------------------------------------------------------------------
int lbg_fold_row_evaluation(const lbg_pp* pp_c, const uint64_t* u, const lbg_challenge* challenges, size_t r,
                            uint64_t out[3]) {
  if (!pp_c || !u || !challenges || !out) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  if (r != pp->cols) return fail(LBG_ERR_INVALID, "one challenge per column");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpyAsync(pp->d_u, u, r * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(cudaMemcpyAsync(pp->d_ch, challenges, r * sizeof(lbg_challenge), cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_fold_binary(pp->d_u, pp->d_ch, (int)r, pp->d_out, pp->stream));
  LBG_CU(cudaMemcpyAsync(out, pp->d_out, 24, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return LBG_OK;
}

int lbg_verify_evaluation(const lbg_pp* pp_c, const uint64_t* p1, size_t p1_len, const uint64_t claimed[3],
                          const uint64_t* u, size_t r, int* accepted) {
  if (!pp_c || !p1 || !claimed || !u || !accepted) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  *accepted = 0;
  if (r != pp->cols || p1_len != (size_t)pp->params.column_log_len) return LBG_OK;  // Rejected
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  LBG_CU(cudaMemcpyAsync(pp->d_u, u, r * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(cudaMemcpyAsync(pp->d_p + 3 * 32, p1, p1_len * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_claim(pp->d_u, (int)r, pp->d_p + 3 * 32, (int)p1_len, pp->d_out, pp->stream));
  uint64_t t[3];
  LBG_CU(cudaMemcpyAsync(t, pp->d_out, 24, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  *accepted = t[0] == claimed[0] && t[1] == claimed[1] && t[2] == claimed[2];
  return LBG_OK;
}

// Verifier::verify_folded_opening (crates/pcs/src/scheme/verifier.rs:178-231), Opening::Clear: v
// centred within the base modulus and its squared norm within fold_cap (params.rs:259-265), A v
// equal to the folded commitment on every limb, and eq(p0) . (v mod 2) equal to the folded row
// value. Device scratch is allocated per call (a verifier's call, not the prover's hot path).
// The verifier's device scratch: one buffer kept in the parameters (grown on use, under pp->mu) and
// carved per call, so that a verification allocates and frees nothing once it has run.
extern "C++" {
struct Carve {
  uint8_t* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t bytes) {
    T* p = reinterpret_cast<T*>(base + off);
    off += (bytes + 255) & ~(size_t)255;
    return p;
  }
};
static size_t carve_size(std::initializer_list<size_t> parts) {
  size_t n = 0;
  for (size_t b : parts) n += (b + 255) & ~(size_t)255;
  return n;
}
}  // extern "C++"

int lbg_verify_folded_opening(const lbg_pp* pp_c, const int16_t* folded_commitment, const int16_t* v,
                              const uint64_t* p0, size_t p0_len, const uint64_t folded_row_value[3],
                              int* accepted) {
  if (!pp_c || !folded_commitment || !v || !p0 || !folded_row_value || !accepted)
    return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  *accepted = 0;
  if (pp->params.opening != LBG_OPENING_CLEAR)
    return fail(LBG_ERR_INVALID, "bit-dropped parameters: the check is lbg_verify_folded_opening_bd");
  if (4 * pp->len_ring != ((size_t)1 << p0_len) || p0_len != (size_t)(pp->params.witness_log_len - pp->params.column_log_len))
    return LBG_OK;  // Rejected, as binary_check's length test
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  cudaStream_t st = pp->stream;
  size_t L = pp->len_ring, nv = L * N648, fcn = 4 * (size_t)pp->limbs * N162;
  int rc = grow((void**)&pp->d_vws, &pp->vws_cap,
                carve_size({nv * 2, fcn * 2, nv * 4, 4 * L * 24, sizeof(VerifyFlags)}));
  if (rc) return rc;
  Carve cv{pp->d_vws};
  int16_t* d_v = cv.take<int16_t>(nv * 2);
  int16_t* d_fc = cv.take<int16_t>(fcn * 2);
  uint32_t* d_vhat = cv.take<uint32_t>(nv * 4);
  uint64_t* d_bits = cv.take<uint64_t>(4 * L * 24);
  VerifyFlags* d_f = cv.take<VerifyFlags>(sizeof(VerifyFlags));
  auto release = [] {};
  cudaError_t e = cudaMemcpyAsync(d_v, v, nv * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_fc, folded_commitment, fcn * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_f, 0, sizeof(VerifyFlags), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pp->d_p, p0, p0_len * 24, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_v_norm(d_v, L, d_f, st);
  for (int k = 0; k < pp->limbs && e == cudaSuccess; k++)
    e = launch_v_limb(pp->pidx[k], d_v, L, pp->d_prime[k], d_vhat, pp->d_Ahat + (size_t)k * L * N162 * 2, k,
                      pp->limbs, d_fc, d_f, st);
  if (e == cudaSuccess) e = launch_v_parity(d_v, L, d_bits, st);
  if (e == cudaSuccess) e = launch_eq_table(pp->d_p, (int)p0_len, 4 * L, pp->d_eq, st);
  if (e == cudaSuccess) e = launch_row_eval(d_bits, 4 * L, 1, pp->d_eq, pp->d_out, st);
  VerifyFlags f;
  uint64_t ub[3];
  if (e == cudaSuccess) e = cudaMemcpyAsync(&f, d_f, sizeof(f), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ub, pp->d_out, 24, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("verify: ") + cudaGetErrorString(e));
  int half = (int)(pp->primes[0] - 1) / 2;
  double cap = std::ceil(108.0 * (double)(pp->n / 4 * N648));  // recursion::FOLD_CAP * (witness_len / 4) * N
  bool ok = !f.wrapped && f.worst <= half && (double)f.normsq <= cap && !f.mismatch && ub[0] == folded_row_value[0] &&
            ub[1] == folded_row_value[1] && ub[2] == folded_row_value[2];
  *accepted = ok ? 1 : 0;
  return LBG_OK;
}

// Verifier::verify_opening, bit-dropped arm (crates/pcs/src/scheme/verifier.rs:232-276): the norm
// checks of the Clear arm, the bit-dropped residual (crates/pcs/src/bd/residual.rs:66-130) against
// bd_cap (crates/pcs/src/bd/mod.rs:72-75), and the binary check.
int lbg_verify_folded_opening_bd(const lbg_pp* pp_c, const uint16_t* top, const uint16_t* digits,
                                 const lbg_challenge* challenges, size_t r, const int16_t* v, const uint64_t* p0,
                                 size_t p0_len, const uint64_t folded_row_value[3], int* accepted,
                                 uint64_t residual_out[2]) {
  if (!pp_c || !top || !challenges || !v || !p0 || !folded_row_value || !accepted)
    return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  *accepted = 0;
  if (pp->params.opening != LBG_OPENING_BIT_DROPPED) return fail(LBG_ERR_INVALID, "the parameters are not bit-dropped");
  int L = pp->limbs;
  if (L > 1 && !digits) return fail(LBG_ERR_INVALID, "null argument");
  if (r != pp->cols) return LBG_OK;  // Rejected: the residual's shape test
  if (4 * pp->len_ring != ((size_t)1 << p0_len) || p0_len != (size_t)(pp->params.witness_log_len - pp->params.column_log_len))
    return LBG_OK;  // Rejected, as binary_check's length test
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  cudaStream_t st = pp->stream;
  size_t Lr = pp->len_ring, nv = Lr * N648, count = pp->cols * N648;
  const size_t ndig = (size_t)(L > 1 ? L - 1 : 1) * count * 2;
  int rc = grow((void**)&pp->d_vws, &pp->vws_cap,
                carve_size({nv * 2, count * 2, ndig, nv * 4, 4 * N162 * 4, (size_t)L * N648 * 4, 4 * Lr * 24, 16,
                            sizeof(VerifyFlags)}));
  if (rc) return rc;
  Carve cv{pp->d_vws};
  int16_t* d_v = cv.take<int16_t>(nv * 2);
  uint16_t* d_top = cv.take<uint16_t>(count * 2);
  uint16_t* d_digits = cv.take<uint16_t>(ndig);
  uint32_t* d_vhat = cv.take<uint32_t>(nv * 4);
  uint32_t* d_diff = cv.take<uint32_t>(4 * N162 * 4);
  uint32_t* d_res = cv.take<uint32_t>((size_t)L * N648 * 4);
  uint64_t* d_bits = cv.take<uint64_t>(4 * Lr * 24);
  unsigned long long* d_ns = cv.take<unsigned long long>(16);
  VerifyFlags* d_f = cv.take<VerifyFlags>(sizeof(VerifyFlags));
  auto release = [] {};
  GarnerConsts gc;
  std::memset(&gc, 0, sizeof(gc));
  for (int k = 0; k < L; k++) {
    gc.q[k] = pp->primes[k];
    for (int m = 0; m < k; m++) gc.inv[k][m] = (uint32_t)inv_mod(pp->primes[m], pp->primes[k]);
  }
  gc.dropped_bits = pp->params.dropped_bits;
  cudaError_t e = cudaMemcpyAsync(d_v, v, nv * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_top, top, count * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && L > 1)
    e = cudaMemcpyAsync(d_digits, digits, (size_t)(L - 1) * count * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pp->d_ch, challenges, r * sizeof(lbg_challenge), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_f, 0, sizeof(VerifyFlags), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pp->d_p, p0, p0_len * 24, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_v_norm(d_v, Lr, d_f, st);
  for (int k = 0; k < L && e == cudaSuccess; k++)
    e = launch_bd_columns(pp->pidx[k], d_top, d_digits, (int)pp->cols, k, gc, L, pp->d_prime[k], pp->d_C, st);
  for (int k = 0; k < L && e == cudaSuccess; k++) {
    e = launch_challenge_slots(pp->pidx[k], pp->d_ch, (int)r, pp->d_prime[k], pp->d_chat, st);
    if (e == cudaSuccess)
      e = launch_fold_commitment(pp->pidx[k], pp->d_C, (int)pp->cols, k, L, pp->d_chat, pp->d_prime[k], pp->d_fc, st);
  }
  for (int k = 0; k < L && e == cudaSuccess; k++) {
    e = launch_v_limb(pp->pidx[k], d_v, Lr, pp->d_prime[k], d_vhat, pp->d_Ahat + (size_t)k * Lr * N162 * 2, k, L,
                      pp->d_fc, d_f, st, d_diff);
    if (e == cudaSuccess) e = launch_bd_inverse(pp->pidx[k], d_diff, pp->d_prime[k], d_res + (size_t)k * N648, st);
  }
  if (e == cudaSuccess) e = launch_bd_normsq(d_res, L, gc, d_ns, st);
  if (e == cudaSuccess) e = launch_v_parity(d_v, Lr, d_bits, st);
  if (e == cudaSuccess) e = launch_eq_table(pp->d_p, (int)p0_len, 4 * Lr, pp->d_eq, st);
  if (e == cudaSuccess) e = launch_row_eval(d_bits, 4 * Lr, 1, pp->d_eq, pp->d_out, st);
  VerifyFlags f;
  uint64_t ub[3], ns[2];
  if (e == cudaSuccess) e = cudaMemcpyAsync(&f, d_f, sizeof(f), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ub, pp->d_out, 24, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ns, d_ns, 16, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("verify: ") + cudaGetErrorString(e));
  if (residual_out) {
    residual_out[0] = ns[0];
    residual_out[1] = ns[1];
  }
  int half = (int)(pp->primes[0] - 1) / 2;
  double cap = std::ceil(108.0 * (double)(pp->n / 4 * N648));  // recursion::FOLD_CAP * (witness_len / 4) * N
  double spread = (double)((1ull << (2 * pp->params.dropped_bits)) - 1) / 12.0;
  uint64_t bd_cap = (uint64_t)std::ceil(4.0 * (double)(N648 * pp->cols * 28) * spread);  // bd::cap
  bool ok = !f.wrapped && f.worst <= half && (double)f.normsq <= cap && ns[1] == 0 && ns[0] <= bd_cap &&
            ub[0] == folded_row_value[0] && ub[1] == folded_row_value[1] && ub[2] == folded_row_value[2];
  *accepted = ok ? 1 : 0;
  return LBG_OK;
}

// ---------------------------------------------------------------------------------------------
// transcript (host)
// ---------------------------------------------------------------------------------------------
lbg_transcript* lbg_transcript_new(const uint8_t* domain, size_t len) { return new lbg_transcript(domain, len); }
lbg_transcript* lbg_transcript_clone(const lbg_transcript* t) { return t ? new lbg_transcript(*t) : nullptr; }
void lbg_transcript_free(lbg_transcript* t) { delete t; }
void lbg_transcript_absorb_bytes(lbg_transcript* t, const uint8_t* b, size_t len) { t->t.absorb_bytes(b, len); }
void lbg_transcript_absorb_u64(lbg_transcript* t, uint64_t x) { t->t.absorb_u64(x); }
void lbg_transcript_fill(lbg_transcript* t, const char* label, uint8_t* out, size_t n) { t->t.fill(label, out, n); }

int lbg_sample_short_challenge(lbg_transcript* t, uint32_t weight, double bound, lbg_challenge* out, uint64_t* attempts) {
  if (!t || !out) return fail(LBG_ERR_INVALID, "null argument");
  if (weight > 32 || weight > 162) return fail(LBG_ERR_INVALID, "weight exceeds MAX_WEIGHT = 32");
  Challenge c = sample_short_challenge(t->t, weight, bound, attempts);
  std::memcpy(out, &c, sizeof(c));
  return LBG_OK;
}

static RoundShape shape_of_params(const lbg_params* p, const uint8_t* seed) {
  RoundShape s;
  s.witness_log_len = p->witness_log_len;
  s.column_log_len = p->column_log_len;
  s.limbs = p->n_moduli;
  s.dropped_bits = p->opening == LBG_OPENING_BIT_DROPPED ? p->dropped_bits : 0;
  for (int k = 0; k < 8; k++) s.primes[k] = k < (int)p->n_moduli ? p->moduli[k] : 0;
  if (seed)
    std::memcpy(s.matrix_seed, seed, 32);
  else
    std::memset(s.matrix_seed, 0, 32);
  return s;
}
static RoundShape shape_of(const lbg_pp* pp) { return shape_of_params(&pp->params, pp->seed); }

static int derive_point(const RoundShape& s, lbg_transcript* t, const int16_t* matrix, const uint16_t* top,
                        const uint16_t* digits, uint64_t* p0_out, uint64_t* p1_out) {
  if (s.dropped_bits == 0 && !matrix) return fail(LBG_ERR_INVALID, "a Clear commitment needs its matrix");
  if (s.dropped_bits > 0 && (!top || (!digits && s.limbs > 1)))
    return fail(LBG_ERR_INVALID, "a bit-dropped commitment needs its digits");
  derive_evaluation_point(s, t->t, matrix, top, digits, p0_out, p1_out);
  return LBG_OK;
}

// The recursive opening's transcript absorbs LaBRADOR commitments (T_y for the evaluation point,
// T_u for the folding challenges: crates/pcs/src/scheme/verifier.rs), which the host's LaBRADOR
// bridge makes; the library's transcript steps cover the Clear and bit-dropped rounds only.
static int refuse_recursive(uint32_t opening) {
  return opening == LBG_OPENING_RECURSIVE
             ? fail(LBG_ERR_UNSUPPORTED, "the recursive round absorbs LaBRADOR commitments made on the host")
             : LBG_OK;
}

int lbg_params_derive_evaluation_point(const lbg_params* p, const uint8_t matrix_seed[32], lbg_transcript* t,
                                       const int16_t* matrix, const uint16_t* top, const uint16_t* digits,
                                       uint64_t* p0_out, uint64_t* p1_out) {
  if (!p || !matrix_seed || !t || !p0_out || !p1_out) return fail(LBG_ERR_INVALID, "null argument");
  int rc = lbg_params_check(p);
  if (!rc) rc = refuse_recursive(p->opening);
  if (rc) return rc;
  return derive_point(shape_of_params(p, matrix_seed), t, matrix, top, digits, p0_out, p1_out);
}

int lbg_params_derive_folding_challenges(const lbg_params* p, lbg_transcript* t, const uint64_t* u,
                                         lbg_challenge* out) {
  if (!p || !t || !u || !out) return fail(LBG_ERR_INVALID, "null argument");
  int rc = lbg_params_check(p);
  if (!rc) rc = refuse_recursive(p->opening);
  if (rc) return rc;
  derive_folding_challenges(shape_of_params(p, nullptr), t->t, u, (Challenge*)out);
  return LBG_OK;
}

size_t lbg_params_pack_dropped(const lbg_params* p, const uint16_t* top, const uint16_t* digits, uint8_t* out,
                               size_t cap) {
  if (!p || !top || lbg_params_check(p) != LBG_OK || p->opening != LBG_OPENING_BIT_DROPPED) return 0;
  std::vector<uint8_t> b = pack_dropped(shape_of_params(p, nullptr), top, digits);
  if (out && cap >= b.size()) std::memcpy(out, b.data(), b.size());
  return b.size();
}

int lbg_derive_evaluation_point(const lbg_pp* pp, lbg_transcript* t, const int16_t* matrix, const uint16_t* top,
                                const uint16_t* digits, uint64_t* p0_out, uint64_t* p1_out) {
  if (!pp || !t || !p0_out || !p1_out) return fail(LBG_ERR_INVALID, "null argument");
  if (int rc = refuse_recursive(pp->params.opening)) return rc;
  return derive_point(shape_of(pp), t, matrix, top, digits, p0_out, p1_out);
}

int lbg_derive_folding_challenges(const lbg_pp* pp, lbg_transcript* t, const uint64_t* u, lbg_challenge* out) {
  if (!pp || !t || !u || !out) return fail(LBG_ERR_INVALID, "null argument");
  if (int rc = refuse_recursive(pp->params.opening)) return rc;
  derive_folding_challenges(shape_of(pp), t->t, u, (Challenge*)out);
  return LBG_OK;
}

size_t lbg_pack_dropped(const lbg_pp* pp, const uint16_t* top, const uint16_t* digits, uint8_t* out, size_t cap) {
  if (!pp || !top) return 0;
  std::vector<uint8_t> b = pack_dropped(shape_of(pp), top, digits);
  if (out && cap >= b.size()) std::memcpy(out, b.data(), b.size());
  return b.size();
}

}  // extern "C"
