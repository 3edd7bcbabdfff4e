/*
 * labinius_gpu.h — the C ABI of the B200 prover path for labinius.
 *
 * Every entry point replaces one call of the reference's scheme API (osdnk/labinius,
 * crates/pcs/src/scheme/) for the commit / evaluate / fold hot path. The Rust `scheme` bodies call
 * these through a thin `extern "C"` crate; the public Rust signatures stay.
 *
 * Conventions (after the only FFI the reference has, crates/pcs/src/labrador/ffi.rs:1-30):
 *  - opaque, caller-owned handles with explicit free;
 *  - plain pointers and sizes, host buffers caller-owned, little-endian;
 *  - every call returns LBG_OK (0) or a negative status, with a message in lbg_last_error();
 *    shape misuse the reference answers with a panic (assert!) is LBG_ERR_INVALID here; nothing
 *    panics across the boundary.
 *  - One handle is used from one host thread at a time (the reference's Prover is &mut).
 *
 * Layouts:
 *  - F162: 3 x uint64 limbs, bits 128..161 in limb 2 (crates/pcs/src/fields/scalar.rs:10).
 *  - Commitment matrix: int16 [columns][4 rows][limbs][162], centered, slot s of R_162 in the
 *    reference's POW3_SLOT_EXP order — VerticallyAlignedMatrix column-major
 *    (crates/pcs/src/ring/element.rs:72-117) with each PowerOfThreeRingElementWithLimbs flattened.
 *  - Key (A): int16 [limbs][len_ring][648], row j of A_i in the reference's tree order, centered
 *    (CommitmentKey::row, crates/pcs/src/key.rs:135-141, de-interleaved from Batch32).
 *  - Folded witness: int16 [len_ring][648], centered coefficients (FoldedWitness,
 *    crates/pcs/src/scheme/commitment.rs:249-279).
 *  - Folded commitment: int16 [4 rows][limbs][162] (FoldedCommitment, :281-296).
 *  - Dropped commitment: top uint16 [columns*648], digits uint16 [limbs-1][columns*648]
 *    (crates/pcs/src/bd/mod.rs:7-56).
 */
#ifndef LABINIUS_GPU_H
#define LABINIUS_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C" {
#endif

#define LBG_OK 0
#define LBG_ERR_INVALID (-1)     /* shape or argument misuse (reference: assert! panics) */
#define LBG_ERR_PARAMS (-2)      /* ParamError (crates/pcs/src/scheme/params.rs:20-50) */
#define LBG_ERR_CUDA (-3)        /* a CUDA call failed */
#define LBG_ERR_OOM (-4)         /* device allocation failed */
#define LBG_ERR_UNSUPPORTED (-5) /* a step of the recursive round that LaBRADOR makes on the host */
#define LBG_ERR_WITNESS (-6)     /* WitnessError::WrongLength (crates/pcs/src/scheme/witness.rs:10-23) */

#define LBG_OPENING_CLEAR 0
#define LBG_OPENING_BIT_DROPPED 1
#define LBG_OPENING_RECURSIVE 2

/* Params (crates/pcs/src/scheme/params.rs:62-68): the base modulus first, then the extra ones. */
typedef struct lbg_params {
  uint32_t witness_log_len;
  uint32_t column_log_len;
  uint32_t n_moduli;      /* 1 + extra_moduli.len() */
  uint32_t moduli[7];     /* primes, base first: any of 2917, 3889, 4861, 9721, 12637, 17497, 19441 */
  uint32_t opening;       /* LBG_OPENING_* */
  uint32_t dropped_bits;  /* Opening::BitDropped { bits } */
} lbg_params;

/* ShortChallenge (crates/pcs/src/challenge.rs:227-235): 40 bytes. */
typedef struct lbg_challenge {
  uint8_t positions[32];
  uint32_t signs;
  uint32_t weight;
} lbg_challenge;

typedef struct lbg_pp lbg_pp;                 /* PublicParameters: params + device key */
typedef struct lbg_prover lbg_prover;         /* Prover: stream + device workspace */
typedef struct lbg_witness lbg_witness;       /* Witness: device-resident F162 (refcounted) */
typedef struct lbg_opening lbg_opening;       /* CommitmentOpening: device handle */
typedef struct lbg_transcript lbg_transcript; /* Transcript (host) */

const char* lbg_last_error(void);
int lbg_version(void);

/* Params::with_base validation (crates/pcs/src/scheme/params.rs:172-203). */
int lbg_params_check(const lbg_params* p);

/* PublicParameters::from_seed (crates/pcs/src/scheme/params.rs:320-338): blake3 of the seed on
 * the host, A expanded on the device (xorshift64*, crates/pcs/src/key.rs:48-88) and kept
 * resident with its R_162 component form. */
int lbg_public_parameters_from_seed(const lbg_params* p, const uint8_t matrix_seed[32], lbg_pp** out);
/* Drops the caller's reference: the parameters are freed once the provers and batches made from them
 * are freed too, so handles may be freed in any order. */
void lbg_public_parameters_free(lbg_pp* pp);
/* CommitmentKey::row (crates/pcs/src/key.rs:135-141) for every limb, into int16 [limbs][len_ring][648]. */
int lbg_key_download(const lbg_pp* pp, int16_t* out);

/* Prover::new (crates/pcs/src/scheme/prover.rs:31-53): device workspace + warm-up round. */
int lbg_prover_new(const lbg_pp* pp, lbg_prover** out);
/* Drops the caller's reference: the prover is freed once its openings are freed or folded. */
void lbg_prover_free(lbg_prover* pr);

/* Witness::from_elements (crates/pcs/src/scheme/witness.rs:54-62): upload n F162. */
int lbg_witness_from_host(const lbg_pp* pp, const uint64_t* f162, size_t n, lbg_witness** out);
/* Witness::random (crates/pcs/src/scheme/witness.rs:66-87), generated on the device. */
int lbg_witness_random(const lbg_pp* pp, const uint8_t seed[32], lbg_witness** out);
/* Witness::lifted (crates/pcs/src/scheme/witness.rs:45-52): B128 traces (2 x uint64) lifted. */
int lbg_witness_lifted(const lbg_pp* pp, const uint64_t* b128, size_t n, lbg_witness** out);
int lbg_witness_download(const lbg_witness* w, uint64_t* out, size_t n);
void lbg_witness_free(lbg_witness* w);

/* Prover::commit (crates/pcs/src/scheme/prover.rs:55-91, crates/pcs/src/key.rs:192-234,
 * crates/pcs/src/bd/digits.rs:141-181). Clear mode fills matrix_out; bit-dropped mode fills
 * top_out / digits_out. Any output pointer may be NULL (the value stays on the device, readable
 * from the opening). The opening keeps a reference to the witness. */
int lbg_commit(lbg_prover* pr, const lbg_witness* w, int16_t* matrix_out, uint16_t* top_out,
               uint16_t* digits_out, lbg_opening** opening_out);
/* Witness::from_elements + Prover::commit in one call, the upload pipelined against the commit:
 * the n F162 at f162 (host memory) are copied in column groups on a second stream, and each group's
 * commit starts as soon as it has landed (limb 0 on the prover's stream, each further limb on a
 * stream of its own, so the limbs' commits of a group overlap). Page-locked memory is copied
 * directly; pageable memory (a Rust Vec<F162>) passes group by group through the prover's ring of
 * three page-locked staging buffers (one column group each, allocated on first use), filled by a
 * few host threads while the device copies and commits the groups before. Outputs as lbg_commit;
 * *w_out gets the device witness (free it with lbg_witness_free). */
int lbg_commit_host(lbg_prover* pr, const uint64_t* f162, size_t n, int16_t* matrix_out, uint16_t* top_out,
                    uint16_t* digits_out, lbg_witness** w_out, lbg_opening** opening_out);
int lbg_opening_matrix(const lbg_opening* op, int16_t* matrix_out);
int lbg_opening_dropped(const lbg_opening* op, uint16_t* top_out, uint16_t* digits_out);
/* Prover::recycle (crates/pcs/src/scheme/prover.rs:116-118): drop an unfolded opening. */
void lbg_opening_free(lbg_opening* op);
/* wire::pack_commitment (crates/pcs/src/wire/mod.rs:226-245): the opening's commitment packed on the
 * device from where lbg_commit left it; ceil(log2 q) bits per slot per limb, LSB first, in the
 * matrix's column-major order (Clear), or wire::pack_dropped of the top bits and digits
 * (bit-dropped, :386-397). out null: returns the byte count only; else cap >= that count. Returns the
 * byte count or a negative status. */
long long lbg_opening_pack_commitment(const lbg_opening* op, uint8_t* out, size_t cap);
/* Opening::Recursive, the commitment's half that runs here (crates/pcs/src/scheme/prover.rs:55-91 with
 * the recursion set up): recursion::limbs::residues (crates/pcs/src/recursion/limbs.rs:379-398) of the
 * opening's commitment, computed on the device, for the host's LaBRADOR bridge to commit as
 * T_y = key_y.commit_blocks(residues). out: int16 [limbs * 4][polys][64]; vector 4 k + l holds, for
 * limb k and component l, each column's coefficients 4 m + l centred and times (-1)^m, in chunks of
 * 54 (chunk b of column j is polynomial b * columns + j, positions 0..53), the rest zero. polys >=
 * 3 * columns (the reference pads to a multiple of 32). Clear and recursive commitments. */
int lbg_opening_residues(const lbg_opening* op, size_t polys, int16_t* out);
/* Prover::commit_left_expansion (crates/pcs/src/scheme/prover.rs:95-115), the vector half: u of the
 * row values (columns F162, [columns][3]) on the device, chunk b of lift(u_j) (its bits as 0/1
 * coefficients, crates/pcs/src/recursion/binary.rs:49-51, chunk.rs:76-86) at polynomial b * columns
 * + j of out (int16 [rank][64], rank >= 3 * columns, the recursion setup's ranks[U]), the rest
 * zero. T_u = key_u.commit_blocks(u) is LaBRADOR's, on the host. */
int lbg_left_expansion(const lbg_pp* pp, const uint64_t* row_values, size_t columns, size_t rank, int16_t* out);

/* Witness::row_evaluate (crates/pcs/src/scheme/witness.rs:100-106, crates/pcs/src/eval.rs:171-182):
 * u_out = columns F162. */
int lbg_row_evaluate(const lbg_pp* pp, const lbg_witness* w, const uint64_t* p0, size_t p0_len,
                     uint64_t* u_out);
/* Witness::mle_evaluate (crates/pcs/src/scheme/witness.rs:94-98, crates/pcs/src/eval.rs:185-193). */
/* Witness::row_evaluate followed by wire::pack_row_evaluation (crates/pcs/src/wire/mod.rs:435-459),
 * both on the device: the row values (u_out, optional, [columns][3]) and their 162-bit packing, LSB
 * first (out; out null: returns the byte count only, ceil(162 columns / 8); else cap >= it). Returns
 * the byte count or a negative status. */
long long lbg_row_evaluate_packed(const lbg_pp* pp, const lbg_witness* w, const uint64_t* p0, size_t p0_len,
                                  uint64_t* u_out, uint8_t* out, size_t cap);
int lbg_mle_evaluate(const lbg_pp* pp, const lbg_witness* w, const uint64_t* p0, size_t p0_len,
                     const uint64_t* p1, size_t p1_len, uint64_t out[3]);

/* Prover::fold (crates/pcs/src/scheme/prover.rs:120-133, crates/pcs/src/fold.rs:659-677): consumes
 * the opening (freed on return, also on error). v_out may be NULL (kept on the device). */
int lbg_fold(lbg_prover* pr, lbg_opening* consumed, const lbg_challenge* challenges, size_t r,
             int16_t* v_out);
/* Whether the commit keeps the base limb's transform of the witness for the fold (the reference's
 * AuxData, crates/pcs/src/key.rs:275-326; 324 bytes of device memory per F162 and opening) or the
 * fold transforms the witness again (the default). An opening whose kept buffer cannot be
 * allocated folds by transforming again. Results are identical either way. */
int lbg_prover_set_kept_transform(lbg_prover* pr, int enable);
/* The last fold's result, int16 [len_ring][648]. */
int lbg_prover_folded(const lbg_prover* pr, int16_t* v_out);

/* Verifier::fold_commitment (crates/pcs/src/scheme/verifier.rs:114-146). */
int lbg_fold_commitment(const lbg_pp* pp, const int16_t* matrix, size_t columns,
                        const lbg_challenge* challenges, size_t r, int16_t* out);

/* Verifier::fold_row_evaluation (crates/pcs/src/scheme/verifier.rs:148-154, eval::fold_binary
 * crates/pcs/src/eval.rs:195-200): out = sum_j (c_j mod 2) u_j. */
int lbg_fold_row_evaluation(const lbg_pp* pp, const uint64_t* u, const lbg_challenge* challenges, size_t r,
                            uint64_t out[3]);
/* Verifier::verify_evaluation (crates/pcs/src/scheme/verifier.rs:157-174): *accepted = 1 when
 * u . eq(p1) equals the claimed value (and the lengths match), else 0. */
int lbg_verify_evaluation(const lbg_pp* pp, const uint64_t* p1, size_t p1_len, const uint64_t claimed[3],
                          const uint64_t* u, size_t r, int* accepted);
/* Verifier::verify_folded_opening (crates/pcs/src/scheme/verifier.rs:178-231), Opening::Clear:
 * *accepted = 1 when v (int16 [len_ring][648]) is centred within the base modulus with its squared
 * norm within Params::fold_cap, A v equals the folded commitment (int16 [4][limbs][162]) on every
 * limb, and eq(p0) . (v mod 2) equals the folded row value; else 0. Bit-dropped parameters return
 * LBG_ERR_INVALID (their check is lbg_verify_folded_opening_bd). */
int lbg_verify_folded_opening(const lbg_pp* pp, const int16_t* folded_commitment, const int16_t* v,
                              const uint64_t* p0, size_t p0_len, const uint64_t folded_row_value[3],
                              int* accepted);
/* Verifier::verify_opening, bit-dropped arm (crates/pcs/src/scheme/verifier.rs:232-276): the same
 * norm and binary checks, and the residual of crates/pcs/src/bd/residual.rs:66-130 (the columns
 * rebuilt from the dropped commitment's top (uint16 [columns*648]) and digits (uint16
 * [limbs-1][columns*648]), folded with the r challenges, subtracted from A v, recombined across the
 * limbs) within bd::cap (crates/pcs/src/bd/mod.rs:72-75). residual_out (may be null): its squared
 * norm, 128 bits, low word first. */
int lbg_verify_folded_opening_bd(const lbg_pp* pp, const uint16_t* top, const uint16_t* digits,
                                 const lbg_challenge* challenges, size_t r, const int16_t* v, const uint64_t* p0,
                                 size_t p0_len, const uint64_t folded_row_value[3], int* accepted,
                                 uint64_t residual_out[2]);

/* switch::prove / prove_bits (crates/pcs/src/switch.rs:64-98, 133-168), the cross-field switch
 * prover: the trace is the B128 words of the witness w (limbs 0 and 1 of each F162, as
 * Witness::lifted holds them), r_hi its l = witness_log_len coordinates, r_lo empty (nlo = 0,
 * words) or the 7 bit coordinates (bits), claim the B128 claim; the transcript t is driven as the
 * reference's. Out: partials [128][2], rounds [l][2][3] (F162 pairs), opened [3], and the point
 * the commitment must open at (p0 [row_log][3], p1 [column_log][3]). */
int lbg_switch_prove(const lbg_pp* pp, const lbg_witness* w, const uint64_t* r_lo, size_t nlo, const uint64_t* r_hi,
                     size_t l, const uint64_t claim[2], lbg_transcript* t, uint64_t* partials, uint64_t* rounds,
                     uint64_t opened[3], uint64_t* p0_out, uint64_t* p1_out);

/* wire::encode (crates/pcs/src/wire/rans.rs:18-105): the folded witness, `elements` ring elements
 * of 648 int16 coefficients (host memory), entropy-coded by interleaved static rANS over 64 lanes
 * against its own histogram, base_q recorded in the header. Writes the bytes when out has room
 * (cap >= the returned count; lbg_wire_encode_bound(elements) always is) and returns their count,
 * or a negative status. The lanes, the histogram and the word placement run on the device. */
long long lbg_wire_encode(const int16_t* v, size_t elements, uint32_t base_q, uint8_t* out, size_t cap);
size_t lbg_wire_encode_bound(size_t elements);
/* The same for the prover's last folded witness, read where Prover::fold left it on the device
 * (no upload), base_q = the base modulus. */
long long lbg_prover_encode_folded(lbg_prover* pr, uint8_t* out, size_t cap);

/* Transcript (crates/pcs/src/challenge.rs:66-161), host side. */
lbg_transcript* lbg_transcript_new(const uint8_t* domain, size_t len);
lbg_transcript* lbg_transcript_clone(const lbg_transcript* t);
void lbg_transcript_free(lbg_transcript* t);
void lbg_transcript_absorb_bytes(lbg_transcript* t, const uint8_t* b, size_t len);
void lbg_transcript_absorb_u64(lbg_transcript* t, uint64_t x);
void lbg_transcript_fill(lbg_transcript* t, const char* label, uint8_t* out, size_t n);
/* sample_short_challenge (crates/pcs/src/challenge.rs:517-533). */
int lbg_sample_short_challenge(lbg_transcript* t, uint32_t weight, double bound, lbg_challenge* out,
                               uint64_t* attempts);
/* Verifier::derive_evaluation_point (crates/pcs/src/scheme/verifier.rs:61-100): matrix (Clear) or
 * top/digits (bit-dropped) as produced by lbg_commit. */
int lbg_derive_evaluation_point(const lbg_pp* pp, lbg_transcript* t, const int16_t* matrix,
                                const uint16_t* top, const uint16_t* digits, uint64_t* p0_out,
                                uint64_t* p1_out);
/* FoldingChallenges::derive (crates/pcs/src/scheme/commitment.rs:217-229). */
int lbg_derive_folding_challenges(const lbg_pp* pp, lbg_transcript* t, const uint64_t* u,
                                  lbg_challenge* out);
/* wire::pack_dropped (crates/pcs/src/wire/mod.rs:386-397): returns the byte count; writes when
 * out has room (cap). */
size_t lbg_pack_dropped(const lbg_pp* pp, const uint16_t* top, const uint16_t* digits, uint8_t* out,
                        size_t cap);

/* The same three host steps from the parameters alone (no device handle): what a verifier that
 * holds only Params and the seed runs. */
int lbg_params_derive_evaluation_point(const lbg_params* p, const uint8_t matrix_seed[32], lbg_transcript* t,
                                       const int16_t* matrix, const uint16_t* top, const uint16_t* digits,
                                       uint64_t* p0_out, uint64_t* p1_out);
int lbg_params_derive_folding_challenges(const lbg_params* p, lbg_transcript* t, const uint64_t* u,
                                         lbg_challenge* out);
size_t lbg_params_pack_dropped(const lbg_params* p, const uint16_t* top, const uint16_t* digits, uint8_t* out,
                               size_t cap);

/* Prover::fold for callers that may not allocate device memory. No counterpart in the reference:
 * an embedding runtime that owns all device memory, or replays its steps where allocator calls
 * are not allowed, folds through this entry point, which allocates nothing. Witness (F162,
 * column-major as lbg_witness holds it), challenges and output v (int16 [len_ring][648]) are device
 * pointers the caller owns; the scratch and tables live in static device arrays (about 4 MB per
 * GPU, held until exit). Columns of at most 4096 ring elements are split over several CTAs whose
 * sums meet in that scratch, so short columns still fill the SMs. At most LBG_FOLD_STATIC_MAX_COLUMNS columns; larger shapes are rejected.
 * The first call on a device sets it up and synchronises (make it before any stream capture);
 * calls share the scratch, so calls that overlap on the GPU race. Asynchronous on `stream`. */
#define LBG_FOLD_STATIC_MAX_COLUMNS 1024
int lbg_fold_static(uint32_t base_prime, uint32_t witness_log_len, uint32_t column_log_len,
                    const uint64_t* d_witness, const lbg_challenge* d_challenges, size_t r, int16_t* d_v_out,
                    void* stream);

/* The reference's 648-point transform of ring elements of Z_q[X]/(X^648 - X^324 + 1)
 * (crates/pcs/src/scalar.rs:35-84 forward, :123-177 inverse), the kernels of the NTT
 * microbenchmark: `count` ring elements, u16 coefficients (forward) or slots in the reference's
 * slot order (inverse), all in [0, q), [count][648], device pointers, asynchronous on `stream`
 * (the current device's). Both buffers 4-byte aligned (else LBG_ERR_INVALID); 16-byte aligned
 * buffers take the faster forward kernel. Splitting primes (3889, 9721, 17497, 19441);
 * quadratic-leaf primes return LBG_ERR_UNSUPPORTED. No Rust API entry point corresponds (the
 * reference calls its transforms internally). */
int lbg_ntt648_forward(uint32_t q, const uint16_t* d_in, uint16_t* d_out, size_t count, void* stream);
int lbg_ntt648_inverse(uint32_t q, const uint16_t* d_in, uint16_t* d_out, size_t count, void* stream);

/* Batched rounds: many independent witnesses under one key (all share the public parameters'
 * column length, moduli and opening; instance i has 2^column_log_lens[i] columns). Every stage is
 * one launch over all instances; the device stages can be replayed as CUDA graphs, and
 * lbg_batch_autotune times candidate grid schedules on the batch's own shape. No single reference
 * call corresponds; each instance's outputs are exactly those of Prover::commit, row_evaluate,
 * mle_evaluate and fold run on it alone (crates/pcs/src/scheme/prover.rs:55-133). Layouts:
 * instances one after another (columns, commitments, row values, folded witnesses). */
typedef struct lbg_batch lbg_batch;
int lbg_batch_new(const lbg_pp* pp, const uint32_t* column_log_lens, size_t count, lbg_batch** out);
/* An arena sized once for max_cols columns and max_instances instances; lbg_batch_assign lays a
 * new set of instances out in it without allocating (what a serving loop reuses). */
int lbg_batch_new_capacity(const lbg_pp* pp, size_t max_cols, size_t max_instances, lbg_batch** out);
/* The device bytes lbg_batch_new_capacity allocates for that capacity (the kept transform and the
 * switch workspace come on use, on top); with lbg_device_memory, what a server sizes its arenas by.
 * No counterpart in the reference (it has no server). */
size_t lbg_batch_arena_bytes(const lbg_pp* pp, size_t max_cols, size_t max_instances);
/* cudaMemGetInfo on the parameters' device: free and total bytes of device memory. */
int lbg_device_memory(const lbg_pp* pp, size_t* free_bytes, size_t* total_bytes);
int lbg_batch_assign(lbg_batch* b, const uint32_t* column_log_lens, size_t count);
void lbg_batch_free(lbg_batch* b);
size_t lbg_batch_columns(const lbg_batch* b);
int lbg_batch_witness_random(lbg_batch* b, const uint8_t* seeds /* count x 32 bytes */);
/* kinds[i] = 0: Witness::random(seed_i); 1: a B128 trace (keyed BLAKE3 XOF of "labinius/b128-trace")
 * lifted (Witness::lifted). kinds may be null (all 0). */
int lbg_batch_witness_generate(lbg_batch* b, const uint8_t* seeds, const uint8_t* kinds);
int lbg_batch_witness_upload(lbg_batch* b, size_t instance, const uint64_t* f162, size_t n);
int lbg_batch_witness_download(const lbg_batch* b, size_t instance, uint64_t* out, size_t n);
int lbg_batch_use_graphs(lbg_batch* b, int enable);
/* The autotuner times candidate commit chunkings and fold splits on the batch's own shape, and
 * whether the fold reads the commit's kept transform, and keeps the fastest. */
int lbg_batch_autotune(lbg_batch* b, uint32_t* chunks_out, uint32_t* fold_cols_out);
/* The schedule lbg_batch_autotune chose beyond its two outputs: the tensor-core commit's compute
 * warps (12 with a producer warp, or 16) and whether the fold reads the kept transform. */
int lbg_batch_schedule(const lbg_batch* b, uint32_t* commit_warps, int* kept_transform);
/* The kept transform on or off by hand (off by default; see lbg_prover_set_kept_transform). */
int lbg_batch_set_kept_transform(lbg_batch* b, int enable);
int lbg_batch_commit(lbg_batch* b, int16_t* matrix_out, uint16_t* top_out, uint16_t* digits_out);
int lbg_batch_row_evaluate(lbg_batch* b, const uint64_t* p0 /* [count][row_log][3] */, uint64_t* u_out);
int lbg_batch_mle_evaluate(lbg_batch* b, const uint64_t* p0, const uint64_t* p1 /* concatenated */,
                           uint64_t* out /* [count][3] */);
int lbg_batch_fold(lbg_batch* b, const lbg_challenge* challenges, size_t r, int16_t* v_out);
/* A whole commit + open round of every instance on the device, transcript included: per instance
 * a fresh Transcript::new(domain), then the steps of crates/bench/src/bin/labinius.rs:104-130
 * (Prover::commit, derive_evaluation_point, mle_evaluate, row_evaluate, FoldingChallenges::derive,
 * Prover::fold) with the absorbs, the evaluation point and the challenge sampler run by device
 * kernels in stream order (no host step between commit and fold). The outputs equal those of the
 * host transcript path bit for bit. Every output pointer may be null (not copied back). */
typedef struct lbg_batch_outputs {
  int16_t* matrix;            /* [total_cols][4][limbs][162] (Opening::Clear) */
  uint16_t* top;              /* [total_cols * 648] (bit-dropped) */
  uint16_t* digits;           /* [limbs - 1][total_cols * 648] (bit-dropped) */
  uint64_t* p0;               /* [count][row_log][3] */
  uint64_t* p1;               /* instance i's column_log_len_i coordinates, one instance after another */
  uint64_t* mle;              /* [count][3] */
  uint64_t* u;                /* [total_cols][3] */
  lbg_challenge* challenges;  /* [total_cols] */
  int16_t* v;                 /* [count][len_ring][648] */
} lbg_batch_outputs;
int lbg_batch_round(lbg_batch* b, const uint8_t* domain, size_t domain_len, const lbg_batch_outputs* out);
/* Instances of the assigned layout that are B128 traces (Witness::lifted, e.g. kind 1 of
 * lbg_batch_witness_generate) opened through the cross-field switch. Their device round is that of
 * crates/pcs/examples/two_fields.rs:176-194: Prover::commit, absorb_bytes(Commitment::to_bytes),
 * switch::prove (crates/pcs/src/switch.rs:65-74), row_evaluate at the switch's point,
 * FoldingChallenges::derive, Prover::fold; the mle output is the value at that point. flags[i] = 1
 * marks instance i; r_hi holds, for each marked instance in order, its witness_log_len B128
 * coordinates (2 words each); claims holds one B128 per marked instance, or is null, and then each
 * marked instance states its trace's value at r_hi (word-level statements). Kept until the next
 * lbg_batch_assign; flags null unmarks every instance. */
int lbg_batch_set_switch(lbg_batch* b, const uint8_t* flags, const uint64_t* r_hi, const uint64_t* claims);
/* After lbg_batch_round: each marked instance's switch proof in order (crates/pcs/src/switch.rs:19-27):
 * partials [128][2], rounds [l][2][3] (one instance after another), opened [3], and its claim [2].
 * Any pointer may be null. */
int lbg_batch_switch_outputs(const lbg_batch* b, uint64_t* partials, uint64_t* rounds, uint64_t* opened,
                             uint64_t* claims);
void* lbg_batch_stream(const lbg_batch* b);
/* No reference counterpart (the reference has no server): the batch's stream at the device's
 * greatest (high != 0) or default priority, so that a slot of small requests is scheduled ahead of
 * a slot of large ones when both wait for SMs. Drains the old stream and drops captured graphs. */
int lbg_batch_set_priority(lbg_batch* b, int high);
/* No reference counterpart: at most `ctas` CTAs (one per SM; 0: every SM) for the batch's
 * persistent commit and fold launches, so that a second batch's launches find SMs free while this
 * one runs (a server's slot of large requests beside its slot of small ones). Drops captured graphs. */
int lbg_batch_set_sm_limit(lbg_batch* b, int ctas);
uint64_t lbg_batch_launch_count(const lbg_batch* b);

/* Shape queries. */
size_t lbg_pp_columns(const lbg_pp* pp);
size_t lbg_pp_len_ring(const lbg_pp* pp);
size_t lbg_pp_witness_len(const lbg_pp* pp);
uint32_t lbg_pp_limbs(const lbg_pp* pp);

/* Device synchronisation and timing support for benchmarks: the prover's CUDA stream. */
void* lbg_prover_stream(const lbg_prover* pr);
int lbg_prover_sync(lbg_prover* pr);
/* Kernel accounting of a prover: with profiling on, every launch of the prover is bracketed by
 * CUDA events on its stream; lbg_prover_kernel_stats reads (and keeps) the per-kernel totals of
 * the launches since profiling was last switched on. Kernel names: "commit", "commit_finish",
 * "challenge_slots", "fold", "column_residues", "garner". The launch counter counts every kernel
 * launch of the prover, profiled or not. */
int lbg_prover_profile(lbg_prover* pr, int enable);
int lbg_prover_kernel_stats(lbg_prover* pr, const char* kernel, uint64_t* launches, double* total_ms);
uint64_t lbg_prover_launch_count(const lbg_prover* pr);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* LABINIUS_GPU_H */
