// Host-callable launch wrappers of the device kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace lbg {

struct HotPrime;
struct DevPrime;
struct Ntt648Tables;

// lbg_challenge as the device sees it (40 bytes).
struct lbg_challenge_d {
  uint8_t positions[32];
  uint32_t signs;
  uint32_t weight;
};

struct GarnerConsts {
  uint32_t q[7];
  uint32_t inv[7][7];  // inv[k][m] = q_m^-1 mod q_k
  uint32_t dropped_bits;
};

// A single-block BLAKE3 root node (key words, message words, block length, flags without ROOT|).
struct XofRoot {
  uint32_t cv[8];
  uint32_t m[16];
  uint32_t block_len;
  uint32_t flags;
};

cudaError_t upload_hot(int pi, const HotPrime& h);
cudaError_t launch_key_expand(const uint64_t* jumps, uint64_t state0, uint32_t q, int nb, int16_t* A,
                              cudaStream_t st);
cudaError_t launch_key_components(int pi, const int16_t* A, const DevPrime* D, int len_ring, int4* Ahat,
                                  cudaStream_t st);
size_t commit_smem_bytes();
int commit_blocks_per_sm(int pi);
int commit_cols_per_cta();
int commit_ring_per_step();
// keep (optional): the base limb's transform of every F162, u16 [cols][162][wdim], for the fold.
// tcb (optional): the limb's transform operand (tc_transform_operand, device memory); with it and
// without keep, the transforms run on the tensor cores (k_commit_tc, persistent, one CTA per SM).
cudaError_t launch_commit(int pi, const uint64_t* W, size_t wdim, const int4* Ahat, const DevPrime* D, int cols,
                          int len_ring, int chunk, int nchunks, int32_t* partial, cudaStream_t st,
                          uint16_t* keep = nullptr, const uint8_t* tcb = nullptr);
bool commit_tc_enabled();
// At most `ctas` CTAs for the persistent tensor-core kernels launched from the calling host thread
// (0: one per SM).
void set_persistent_cap(int ctas);
// The tensor-core commit's compute warps (12 or 16; 0: the default) for launches from the calling
// host thread.
void set_commit_warps(int warps);
// 1 (and cleared) when a tensor-core kernel's bounded wait ran out since the last call, else 0;
// -1 when the flag could not be read.
int tc_timeout_take();
cudaError_t launch_commit_finish(int pi, const int32_t* partial, int nchunks, int cols, const DevPrime* D,
                                 int limb, int limbs, int16_t* C, cudaStream_t st);
cudaError_t launch_challenge_slots(int pi, const lbg_challenge_d* ch, int r, const DevPrime* D, uint32_t* chat,
                                   cudaStream_t st);
size_t fold_smem_bytes();
int fold_positions_per_cta();
int fold_cols_per_step();
int fold_blocks_per_sm(int pi);
// The fold over all columns: k_fold accumulates column splits of cols_per_split columns into vhat
// (u32 [wdim][162], zeroed here), then k_fold_finish inverts and centres into v. With vhat null
// the fold runs in one pass over all columns, each CTA inverting its own positions.
// Many instances of the same column length (instances > 1): their columns one after another, each
// split within one instance (split_inst[s] its instance), vhat and v one instance after another.
// tcb (optional): the base limb's transform operand; with it and vhat, the transforms run on the
// tensor cores (k_fold_tc, 128 positions per work item, persistent, one CTA per SM); vhat is then
// read transposed ([instance][162][wdim]).
cudaError_t launch_fold(int pi, const uint64_t* W, size_t wdim, int cols, int cols_per_split, const uint32_t* chat,
                        const DevPrime* D, uint32_t* vhat, int16_t* v, cudaStream_t st, int instances = 1,
                        const int* split_inst = nullptr, const uint8_t* tcb = nullptr);
// The fold with the challenges folded into the tensor-core operand (k_fold_operand + k_fold_gm +
// k_fold_finish_t) for one instance: G is fold_gm_operand_bytes(cols) bytes of device scratch.
bool fold_gm_enabled();
size_t fold_gm_operand_bytes(size_t cols);
cudaError_t launch_fold_gm(int pi, const uint64_t* W, size_t wdim, int cols, int cols_per_split, const uint32_t* chat,
                           const uint8_t* tcb, uint8_t* G, const DevPrime* D, uint32_t* vhat, int16_t* v,
                           cudaStream_t st, int instances = 1, const int* split_inst = nullptr);
bool fold_tc_enabled();
int fold_tc_positions_per_cta();
// The fold from the commit's kept transform instead of the witness (same splits and outputs).
cudaError_t launch_fold_kept(int pi, const uint16_t* keep, size_t wdim, int cols, int cols_per_split,
                             const uint32_t* chat, const DevPrime* D, uint32_t* vhat, int16_t* v, cudaStream_t st,
                             int instances = 1, const int* split_inst = nullptr);
cudaError_t launch_fold_commitment(int pi, const int16_t* C, int cols, int limb, int limbs, const uint32_t* chat,
                                   const DevPrime* D, int16_t* out, cudaStream_t st);
cudaError_t launch_column_residues(int pi, const int16_t* C, int cols, int limb, int limbs, const DevPrime* D,
                                   uint16_t* res, cudaStream_t st);
// The recursive opening's residue vectors of one limb from its coefficients (k_column_residues), and
// the left expansion's vector from the row values.
cudaError_t launch_recursion_residues(const uint16_t* res, int cols, size_t polys, uint32_t q, int16_t* out,
                                      cudaStream_t st);
cudaError_t launch_left_expansion(const uint64_t* u, int cols, size_t rank, int16_t* out, cudaStream_t st);
cudaError_t launch_garner(const uint16_t* res, size_t count, int limbs, const GarnerConsts& g, uint16_t* top,
                          uint16_t* digits, cudaStream_t st);
cudaError_t launch_eq_table(const uint64_t* p, int n, size_t count, uint64_t* eq, cudaStream_t st,
                            int instances = 1);
// u (cols F162, zeroed here) = the row evaluations of W's columns against eq. `tiles` (device,
// x = first column, y = columns (<= row_eval_tile_cols()), z = instance whose eq table
// eq + z * wdim * 3 applies) covers a batch of instances; null means one instance.
cudaError_t launch_row_eval(const uint64_t* W, size_t wdim, int cols, const uint64_t* eq, uint64_t* u,
                            cudaStream_t st, const int4* tiles = nullptr, int ntiles = 0);
int row_eval_tile_cols();

// The verifier's checks (crates/pcs/src/scheme/verifier.rs:157-231). Flags zeroed by the caller.
struct VerifyFlags {
  unsigned long long normsq;
  int worst;
  int wrapped;
  int mismatch;
  int pad_;
};
cudaError_t launch_v_norm(const int16_t* v, size_t len_ring, VerifyFlags* f, cudaStream_t st);
// A v modulo one limb against the folded commitment [4][limbs][162]; vhat: len_ring * 648 u32.
cudaError_t launch_v_limb(int pi, const int16_t* v, size_t len_ring, const DevPrime* D, uint32_t* vhat,
                          const int4* Ahat, int limb, int limbs, const int16_t* fc, VerifyFlags* f, cudaStream_t st,
                          uint32_t* diff = nullptr);
// The bit-dropped residual (crates/pcs/src/bd/residual.rs:66-130): the columns rebuilt from top
// and digits in the commitment's component form C [cols][4][limbs][162] (limb `limb`); A v minus
// the folded commitment (launch_v_limb with diff [4][162]) back to coefficients res [648]; the
// Garner recombination of res [limbs][648] and its squared norm (128 bits, low word first).
cudaError_t launch_bd_columns(int pi, const uint16_t* top, const uint16_t* digits, int cols, int limb,
                              const GarnerConsts& g, int limbs, const DevPrime* D, int16_t* C, cudaStream_t st);
cudaError_t launch_bd_inverse(int pi, const uint32_t* diff, const DevPrime* D, uint32_t* res, cudaStream_t st);
cudaError_t launch_bd_normsq(const uint32_t* res, int limbs, const GarnerConsts& g, unsigned long long* out,
                             cudaStream_t st);
// components_mod_2 of v as 4 len_ring F162.
cudaError_t launch_v_parity(const int16_t* v, size_t len_ring, uint64_t* W, cudaStream_t st);
cudaError_t launch_fold_binary(const uint64_t* u, const lbg_challenge_d* ch, int r, uint64_t* out, cudaStream_t st);
// The reference's 648-point forward transform or its inverse of `count` ring elements (u16 in
// [0, q), [count][648]) for the splitting prime with index pi; T: device copy of its tables.
cudaError_t launch_ntt648(int pi, bool inverse, const uint16_t* in, uint16_t* out, size_t count,
                          const Ntt648Tables* T, cudaStream_t st);
cudaError_t launch_claim(const uint64_t* u, int cols, const uint64_t* p1, int n, uint64_t* out, cudaStream_t st);
cudaError_t launch_xof(const XofRoot& root, size_t nbytes, uint8_t* out, cudaStream_t st);
// Witness::random: the XOF bytes as F162 words, the third limb masked to 34 bits, in one pass.
cudaError_t launch_xof_f162(const XofRoot& root, size_t n, uint64_t* W, cudaStream_t st);
cudaError_t launch_mask_f162(uint64_t* W, size_t n, cudaStream_t st);
// n B128 elements of a keyed XOF written lifted into F162 [lo, hi, 0].
cudaError_t launch_xof_lifted(const XofRoot& root, size_t n, uint64_t* W, cudaStream_t st);
cudaError_t launch_lift_b128(const uint64_t* b, size_t n, uint64_t* W, cudaStream_t st);

}  // namespace lbg
