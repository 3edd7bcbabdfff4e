// The library's handle types, shared by the C-ABI translation units (api.cu, batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "copy_pool.h"
#include "launch.h"
#include "prime_structs.h"
#include "transcript.h"

using lbg::DevPrime;
using lbg::lbg_challenge_d;
using lbg::Transcript;

struct lbg_pp {
  // references: the caller's, and one per prover and batch made from it, so that the handles may be
  // freed in any order (a garbage collector finalizes a cycle in no fixed order)
  std::atomic<int> refs{1};
  lbg_params params;
  int limbs = 0;
  uint32_t primes[7];
  int pidx[7];
  size_t cols = 0, wdim = 0, len_ring = 0, n = 0;
  uint8_t seed[32];
  uint64_t key_seed = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  int16_t* d_A = nullptr;     // [limbs][len_ring][648]
  int4* d_Ahat = nullptr;     // [limbs][len_ring][162][2]
  DevPrime* d_prime[7] = {nullptr};
  uint8_t* d_tcb[7] = {nullptr};  // per limb: the transform as a tensor-core operand (TC_B_BYTES)
  uint64_t* d_jumps = nullptr;
  std::mutex mu;              // guards the scratch below (Witness::row_evaluate takes &self)
  uint64_t* d_eq = nullptr;   // [wdim][3]
  uint64_t* d_p = nullptr;    // point coordinates
  uint64_t* d_u = nullptr;    // [cols][3]
  uint64_t* d_out = nullptr;  // [3]
  int16_t* d_C = nullptr;     // fold_commitment input [cols][4][limbs][162]
  lbg_challenge_d* d_ch = nullptr;
  uint32_t* d_chat = nullptr;  // [cols][162]
  int16_t* d_fc = nullptr;     // [4][limbs][162]
  uint8_t* d_sw = nullptr;     // the switch prover's workspace (lbg_switch_prove), allocated on first use
  uint8_t* d_wire = nullptr;   // lbg_row_evaluate_packed's bytes (grown on use)
  size_t wire_cap = 0;
  int16_t* d_lift = nullptr;   // lbg_left_expansion's vector (grown on use)
  size_t lift_cap = 0;
  uint8_t* d_vws = nullptr;    // the verifier's scratch (grown on use, carved per call)
  size_t vws_cap = 0;
};

// Frees the switch prover's workspace of pp (switch.cu).
void lbg_switch_release(lbg_pp* pp);
// A reference to pp taken by a prover or batch, and its release (the last one frees pp).
extern "C" void lbg_pp_retain(const lbg_pp* pp);
extern "C" void lbg_pp_release(const lbg_pp* pp);

struct lbg_witness {
  std::atomic<int> refs{1};
  uint64_t* d = nullptr;
  size_t n = 0;
  int device = 0;
};

struct OpeningBufs;

struct lbg_prover {
  std::atomic<int> refs{1};  // the caller's, and one per live opening
  const lbg_pp* pp = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;        // lbg_commit_host's uploads (created on first use)
  std::vector<cudaEvent_t> group_events;     // one per column group of lbg_commit_host
  // lbg_commit_host commits limb k >= 1 on its own stream with its own chunk partials, so the
  // limbs' launches of a column group overlap (created on first use)
  std::vector<cudaStream_t> limb_streams;
  std::vector<cudaEvent_t> limb_done;
  std::vector<int32_t*> limb_partial;
  // lbg_commit_host from pageable host memory: the column groups pass through a ring of
  // page-locked staging buffers, filled by a few host threads (created on first use)
  static constexpr int STAGES = 3;
  void* stage[STAGES] = {nullptr, nullptr, nullptr};
  size_t stage_bytes = 0;
  cudaEvent_t stage_copied[STAGES] = {nullptr, nullptr, nullptr};  // the device copy out of stage s
  lbg::CopyPool* copy_pool = nullptr;
  int chunk = 0, nchunks = 0;
  int fold_cols_per_split = 0;
  int32_t* d_partial = nullptr;
  uint32_t* d_vhat = nullptr;  // [wdim][162]
  lbg_challenge_d* d_ch = nullptr;
  uint32_t* d_chat = nullptr;
  int16_t* d_v = nullptr;     // [len_ring][648]
  uint8_t* d_wire = nullptr;  // lbg_opening_pack_commitment's bytes (grown on use)
  size_t wire_cap = 0;
  uint16_t* d_res = nullptr;  // [limbs][cols*648]
  uint8_t* d_gm = nullptr;    // the fold's per-column tensor-core operands (LBG_FOLD_KERNEL=gm)
  int16_t* d_rec = nullptr;   // lbg_opening_residues' vectors (grown on use)
  size_t rec_cap = 0;
  std::mutex mu;
  std::vector<struct OpeningBufs*> spare;
  // the fold reads the commit's kept transform (the reference's AuxData, crates/pcs/src/key.rs:275-326)
  // instead of transforming the witness again; 324 B of device memory per F162 and opening. Off by
  // default: at 2^22 the commit's extra 1.36 GB of stores cost more than the fold saves.
  bool keep = false;
  // kernel accounting
  uint64_t launches = 0;
  bool profiling = false;
  struct Mark {
    const char* name;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> event_pool;
};

// Brackets one launch of the prover with events when profiling is on, and counts it.
struct KernelScope {
  lbg_prover* pr;
  const char* name;
  cudaEvent_t a = nullptr, b = nullptr;
  static cudaEvent_t take(lbg_prover* pr) {
    if (!pr->event_pool.empty()) {
      cudaEvent_t e = pr->event_pool.back();
      pr->event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  KernelScope(lbg_prover* p, const char* n, int kernels = 1) : pr(p), name(n) {
    pr->launches += kernels;
    if (pr->profiling) {
      a = take(pr);
      b = take(pr);
      cudaEventRecord(a, pr->stream);
    }
  }
  ~KernelScope() {
    if (a) {
      cudaEventRecord(b, pr->stream);
      pr->marks.push_back({name, a, b});
    }
  }
};

struct OpeningBufs {
  int16_t* d_C = nullptr;       // [cols][4][limbs][162]
  uint16_t* d_top = nullptr;    // [cols*648]
  uint16_t* d_digits = nullptr; // [limbs-1][cols*648]
  uint16_t* d_keep = nullptr;   // the base limb's transform [cols][162][wdim] (kept-transform mode)
};

struct lbg_opening {
  lbg_prover* pr = nullptr;
  lbg_witness* w = nullptr;
  OpeningBufs* bufs = nullptr;
};

struct lbg_transcript {
  Transcript t;
  explicit lbg_transcript(const uint8_t* d, size_t n) : t(d, n) {}
};


void lbg_witness_release_internal(lbg_witness* w);
