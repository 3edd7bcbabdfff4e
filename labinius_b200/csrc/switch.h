// The cross-field switch prover on the device, shared by the single-instance entry point
// (lbg_switch_prove) and the batched round (lbg_batch_round with switch instances).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "hasher_state.h"

namespace lbg {

// The small per-instance values of a switch: one device block per instance.
struct SwSmall {
  // the pass over the trace: three 128 x 128 GF(2) matrices, row k as 4 words (bit m of word
  // m / 32): sum_j bit_k(t_j) bit_m(eq_j) over j >= n/2, over j < n/2, and over the pairs
  // (j, j + n/2) with t_j + t_j+n/2 and eq_j + eq_j+n/2
  uint32_t mat[3][128][4];
  uint64_t v[128][2];         // the partial evaluations
  uint64_t msg[8];            // the running round's message (e0, einf): XOR accumulators
  uint64_t claim[2];          // the B128 claim: given, or the trace's value at r_hi
  uint64_t rp[8][3];          // the 7 batch coordinates
  uint64_t rr[32][3];         // the round challenges
  uint64_t rounds[32][6];     // the round messages
  uint64_t rtab[41 * 16][3];  // the running round's products by its challenge r: (t x^(4i)) r at 16 i + t
  uint64_t psi[32 * 16][3];   // psi by nibble: the XOR of batch[4c + b] over the set bits b of t at 16 c + t
  uint64_t rpsi[32 * 16][3];  // the same times round 0's challenge
  uint64_t opened[3];
  uint32_t status;            // 0 once the instance's switch has run
  uint32_t pad_;
};

// One switch instance: its trace (the words of a lifted witness), its statement, its device
// scratch, its transcript, and where its evaluation point goes.
struct SwInst {
  const uint64_t* w;     // the lifted witness, F162 [n][3]: trace word j is w[3j], w[3j+1]
  const uint64_t* r_hi;  // [l][2]
  const uint64_t* r_lo;  // [nlo][2] for a bit-level statement
  uint64_t* e_hi;        // [2^lh][2]
  uint64_t* e_lo;        // [2^ll][2]
  uint64_t* eq;          // [n][2]
  uint64_t* a;           // [max(n/2, 1)][3]
  uint64_t* p;           // [max(n/2, 1)][3]
  SwSmall* s;
  HasherState* st;       // the instance's transcript hasher
  uint64_t counter0;     // its derivation counter when the switch starts
  uint64_t* p0;          // the evaluation point, p0 [row_log][3] and p1 [col_log][3] (null: not written)
  uint64_t* p1;
  uint32_t l, lh, ll, nlo;
  uint32_t row_log, col_log;
  uint32_t claim_given;  // 0: the switch states the trace's value at r_hi (word-level statements)
  uint32_t pad_;
};

// Device scratch (besides SwSmall) of a switch over 2^l elements, and its layout at `base`
// (256-byte aligned): fills e_hi, e_lo, eq, a, p and lh, ll.
size_t sw_scratch_bytes(uint32_t l);
void sw_layout(SwInst& inst, uint8_t* base);

// The switch of `count` instances (table d_inst on the device, its host copy h_inst) in stream
// order, with no host round trip: eq tables and partials; the statement and the partials
// absorbed and the batch sampled; then per round the message, its absorb, the challenge and the
// fold; the opened value and the evaluation point. Launches are counted into *launches.
cudaError_t enqueue_switch(const SwInst* d_inst, const SwInst* h_inst, int count, cudaStream_t st,
                           uint64_t* launches);

// Launches of enqueue_switch for the instances h[0..count).
uint64_t sw_launches(const SwInst* h, int count);

// Transcript bytes a word-level (nlo = 0) or bit-level (nlo = 7) switch over l variables absorbs.
inline uint64_t sw_transcript_bytes(uint32_t l, uint32_t nlo) {
  // "labinius/switch", r_lo, r_hi, [claim], the partials, then one message per round
  return (8 + 15) + (8 + 16ull * nlo) + (8 + 16ull * l) + (8 + 16) + (8 + 16 * 128) + 56ull * l;
}

}  // namespace lbg
