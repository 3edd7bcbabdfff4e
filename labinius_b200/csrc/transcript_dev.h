// The Fiat-Shamir transcript of a round on the device: absorbing the commitment and the row
// values into per-instance BLAKE3 hasher states, the evaluation point and the folding challenges
// drawn from them, all in stream order with the rest of the round (no host round trip between
// commit and fold). The byte stream, the hasher states and the sampler are the host transcript's
// (transcript.h), so the two agree bit for bit.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "hasher_state.h"
#include "launch.h"

namespace lbg {

// Bytes appended to one hasher: `prefix` (known on the host when the round is planned), then
// `rows` rows, each `hdr_len` header bytes followed by `row_bytes` bytes read from
// data + r * row_stride (device memory).
struct AbsorbSource {
  uint8_t prefix[48];
  uint32_t prefix_len;
  uint8_t hdr[8];
  uint32_t hdr_len;
  uint32_t rows;
  uint32_t row_bytes;
  uint64_t row_stride;
  const uint8_t* data;
  uint64_t length() const { return prefix_len + (uint64_t)rows * (hdr_len + row_bytes); }
};

// One hasher's share of a planned absorb. Chunks t0 .. t1-1 complete during it (chunk t0 was the
// open chunk before it); chunk t1 is the open chunk after it.
struct AbsorbJob {
  HasherState* st;
  AbsorbSource src;
  uint64_t stage_off;  // staging bytes of chunk t0's first byte (1024-aligned)
  uint64_t stage_len;  // (t1 - t0) * 1024 + c1
  uint64_t t0, t1;
  uint32_t ob, obl;    // compressed blocks and buffered bytes of chunk t0 before the absorb
  uint32_t c1;         // bytes of chunk t1 after the absorb (1..1024)
  uint32_t entry_off;  // first entry of the job in the chunk kernel (t1 - t0 + 1 entries)
  uint64_t level_off;  // first chaining-value slot of the job's subtree levels
};

// An absorb over several hashers at once (one job each), with its tables on the device.
struct AbsorbPlan {
  std::vector<AbsorbJob> jobs;
  std::vector<int> entry_job;  // chunk-kernel entry -> job
  std::vector<uint64_t> stage_word_off;  // per job: first 16-byte staging word, plus the total
  uint64_t stage_bytes = 0, cv_slots = 0;
  AbsorbJob* d_jobs = nullptr;
  int* d_entry_job = nullptr;
  uint64_t* d_stage_word_off = nullptr;
  void clear();
  void release();
};

// Add a job: the hasher at d_state (device) has absorbed `old_len` bytes (old_len >= 1) and
// takes the bytes of `src` next.
void plan_absorb(AbsorbPlan& p, HasherState* d_state, uint64_t old_len, const AbsorbSource& src);
// Copy the plan's tables to the device (once per plan).
cudaError_t upload_absorb(AbsorbPlan& p);
// The absorb (staging, chunk chaining values, subtree merge) on `st`. Scratch: stage_bytes bytes,
// cv_slots * 32 bytes, 32 bytes per job.
cudaError_t launch_absorb(const AbsorbPlan& p, uint8_t* d_stage, uint32_t* d_cvs, uint32_t* d_oldcv, cudaStream_t st);

// Per instance of a round on the device.
struct RoundInst {
  const HasherState* st;     // the instance's transcript hasher
  uint64_t point_counter;    // derivation counter of the evaluation point
  uint64_t chal_counter;     // derivation counter of the first folding challenge
  uint32_t row_log, col_log;
  uint32_t col_off;          // first column of the instance in the batch
  uint32_t pad_;
};

// The evaluation point of every instance: p0 (row_log F162) at p0 + 3 * row_log * i, p1
// (col_log F162) at p1 + 3 * 32 * i (crates/pcs/src/scheme/verifier.rs:86-100).
cudaError_t launch_point(const RoundInst* d_inst, int count, uint32_t row_log, uint64_t* p0, uint64_t* p1,
                         cudaStream_t st);
// One folding challenge per column, sampled from its instance's hasher
// (crates/pcs/src/scheme/commitment.rs:217-229, crates/pcs/src/challenge.rs:517-533).
struct SamplerTables {
  const double* re;  // [162][81]
  const double* im;
  uint32_t signs_key[8];
  double bound_sq;
  uint32_t weight;
};
// The sampler's tables on `device` (uploaded once per device), weight 28, bound 12
// (crates/pcs/src/challenge.rs:517-533 as called by FoldingChallenges::derive).
cudaError_t sampler_tables(int device, SamplerTables& out);
cudaError_t launch_challenges(const RoundInst* d_inst, const int* col_inst, int total_cols, SamplerTables tab,
                              lbg_challenge_d* out, cudaStream_t st);
// mle claims of every instance at once: out[i] = sum_j eq(p1_i, j) u_{col_off_i + j}.
cudaError_t launch_claims(const RoundInst* d_inst, const int* col_inst, const uint64_t* u, int total_cols,
                          const uint64_t* p1, int count, uint64_t* out, cudaStream_t st);
// Bit-dropped commitment bytes (crates/pcs/src/wire/mod.rs:386-397): element e's top value then
// its digits, LSB first, at bit e * bits_per.
struct PackDropped {
  uint32_t top_bits;
  uint32_t residue_bits[8];
  uint32_t limbs;
  uint32_t bits_per;
};
cudaError_t launch_pack_dropped(const uint16_t* top, const uint16_t* digits, uint64_t count, uint64_t digit_stride,
                                PackDropped pk, uint8_t* out, uint64_t nbytes, cudaStream_t st);

}  // namespace lbg
