// lbg_fold_static: the fold for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc at the moment they fold: a prover embedded
// in a runtime that owns all device memory through its own arena, or one that replays its steps
// inside a stream it must not disturb with allocator calls. For them this file provides one entry
// point that allocates no device memory: the fold's scratch (the challenges' slot values, and for
// short columns the per-position sums) lives in file-scope static device arrays of fixed size, and
// so do the per-prime tables the fold reads.
// The caller passes the witness, the challenges and the output in device memory it owns.
//
// Limits and behaviour, for the caller:
//  * the witness, the challenges and the output are device pointers the caller owns;
//  * at most LBG_FOLD_STATIC_MAX_COLUMNS challenges (columns); larger requests are rejected;
//  * every GPU that loads the library holds the arrays below until the process exits;
//  * the first call on a device sets that device up (symbol addresses, table upload) and
//    synchronises; make that first call before any stream capture;
//  * all calls share the one scratch array: two calls whose work overlaps on the GPU race.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/labinius_gpu.h"
#include "error.h"
#include "launch.h"
#include "prime_structs.h"
#include "ring_tables.h"
#include "upload.h"

using namespace lbg;

namespace {

constexpr size_t MAX_COLUMNS = LBG_FOLD_STATIC_MAX_COLUMNS;
constexpr size_t SCRATCH_BYTES = MAX_COLUMNS * N162 * sizeof(uint32_t);  // 648 KiB of slot values
// Positions (ring elements of one column) up to which the columns may be split over several CTAs,
// each adding its columns' share into the per-position sums below. Longer columns already give
// every SM a CTA of their own and fold in one pass; the split pays only below this length.
constexpr size_t SPLIT_MAX_POSITIONS = 4096;
constexpr size_t SUMS_BYTES = SPLIT_MAX_POSITIONS * N162 * sizeof(uint32_t);  // 2.53 MiB

// The scratch: the challenges' slot values c_j(-theta^v), shared by every call on the device.
static __device__ __align__(256) uint8_t g_fold_scratch[SCRATCH_BYTES];
// The per-position sums of a split fold, shared by every call on the device like the slot values.
static __device__ __align__(256) uint32_t g_fold_sums[SUMS_BYTES / sizeof(uint32_t)];
// The fold's read-only per-prime tables, one slot per supported prime.
static __device__ __align__(256) DevPrime g_fold_tables[7];

struct DeviceState {
  bool ready = false;
  uint8_t* scratch = nullptr;
  uint32_t* sums = nullptr;
  DevPrime* tables = nullptr;
  int sms = 0;
  bool uploaded[7] = {false, false, false, false, false, false, false};
  int blocks_per_sm[7] = {0, 0, 0, 0, 0, 0, 0};
};
constexpr int MAX_DEVICES = 64;
DeviceState g_state[MAX_DEVICES];
std::mutex g_mu;
int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

void fill_tables(const PrimeTables& T, DevPrime* D) {
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
    for (int k = 0; k < cnt; k++) {
      uint64_t zi = inv_mod(T.z_level[L][k], q);
      D->zinv3[L][k] = (uint32_t)(zi * T.inv3 % q);
      D->zinv3sq[L][k] = (uint32_t)(zi * zi % q * T.inv3 % q);
    }
  }
  D->omega = T.omega;
  D->inv3 = T.inv3;
  D->zeta6 = T.zeta6;
  D->det0 = T.det0;
  std::memcpy(D->chal, T.chal_table.data(), sizeof(D->chal));
}

// Once per device (with that device current): the symbol addresses, then per prime its tables.
int setup(int dev, int pi, uint32_t q, DeviceState** out) {
  std::lock_guard<std::mutex> g(g_mu);
  DeviceState& S = g_state[dev];
  if (!S.ready) {
    cudaError_t e = cudaGetSymbolAddress((void**)&S.scratch, g_fold_scratch);
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void**)&S.sums, g_fold_sums);
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("cudaGetSymbolAddress(sums): ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void**)&S.tables, g_fold_tables);
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("cudaGetSymbolAddress(tables): ") + cudaGetErrorString(e));
    e = cudaDeviceGetAttribute(&S.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("SM count: ") + cudaGetErrorString(e));
    S.ready = true;
  }
  if (!S.uploaded[pi]) {
    const PrimeTables& T = prime_tables(q);
    static DevPrime staging;  // host copy, filled under the lock
    fill_tables(T, &staging);
    cudaError_t e = upload_sync(S.tables + pi, &staging, sizeof(DevPrime));
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
    HotPrime h;
    std::memcpy(h.tw, T.tw, sizeof(h.tw));
    h.omega = T.omega;
    h.omega_s = T.omega_s;
    e = upload_hot(pi, h);
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("twiddle upload: ") + cudaGetErrorString(e));
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("set-up: ") + cudaGetErrorString(e));
    S.blocks_per_sm[pi] = std::max(1, fold_blocks_per_sm(pi));
    S.uploaded[pi] = true;
  }
  *out = &S;
  return LBG_OK;
}

// Columns per split for a fold of `wdim` positions: the split count whose waves of CTAs (position
// tiles x splits over the SMs' resident slots) cost the fewest column steps. 0 keeps one pass.
int static_cols_per_split(const DeviceState& S, int pi, size_t wdim, int cols) {
  if (wdim > SPLIT_MAX_POSITIONS) return 0;
  const long tiles = (long)((wdim + fold_positions_per_cta() - 1) / fold_positions_per_cta());
  const long slots = (long)S.sms * S.blocks_per_sm[pi];
  const int step = fold_cols_per_step();
  long best = -1;
  int best_per = cols;
  for (int ns = 1; ns <= (cols + step - 1) / step; ns++) {
    int per = (cols + ns - 1) / ns;
    per = (per + step - 1) / step * step;
    long items = tiles * ((cols + per - 1) / per);
    long cost = (items + slots - 1) / slots * per;
    if (best < 0 || cost < best) {
      best = cost;
      best_per = per;
    }
  }
  return best_per < cols ? best_per : 0;
}

}  // namespace

extern "C" {

int lbg_fold_static(uint32_t base_prime, uint32_t witness_log_len, uint32_t column_log_len,
                    const uint64_t* d_witness, const lbg_challenge* d_challenges, size_t r, int16_t* d_v_out,
                    void* stream) {
  if (!d_witness || !d_challenges || !d_v_out) return fail(LBG_ERR_INVALID, "null argument");
  int pi = prime_index(base_prime);
  if (pi < 0) return fail(LBG_ERR_PARAMS, "unsupported base modulus " + std::to_string(base_prime));
  if (column_log_len < 1 || column_log_len > witness_log_len || witness_log_len - column_log_len < 7 ||
      witness_log_len > 30)
    return fail(LBG_ERR_PARAMS, "invalid shape");
  size_t cols = (size_t)1 << column_log_len;
  if (r != cols) return fail(LBG_ERR_INVALID, "one challenge per column");
  if (cols > MAX_COLUMNS)
    return fail(LBG_ERR_INVALID, "lbg_fold_static handles at most " + std::to_string(MAX_COLUMNS) +
                                     " columns (its scratch is a fixed static array); got " + std::to_string(cols));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(LBG_ERR_INVALID, "device index out of range");
  DeviceState* S = nullptr;
  int rc = setup(dev, pi, base_prime, &S);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  size_t wdim = (size_t)1 << (witness_log_len - column_log_len);
  uint32_t* d_chat = (uint32_t*)S->scratch;
  // every slot value of the r challenges is rewritten by the first launch, so nothing needs clearing
  e = launch_challenge_slots(pi, (const lbg_challenge_d*)d_challenges, (int)r, S->tables + pi, d_chat, st);
  // short columns leave SMs idle in one pass: split the columns, each split adding into the static sums
  const int per = static_cols_per_split(*S, pi, wdim, (int)cols);
  if (e == cudaSuccess)
    e = launch_fold(pi, d_witness, wdim, (int)cols, per ? per : (int)cols, d_chat, S->tables + pi,
                    per ? S->sums : nullptr, d_v_out, st);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("lbg_fold_static: ") + cudaGetErrorString(e));
  return LBG_OK;
}

}  // extern "C"
