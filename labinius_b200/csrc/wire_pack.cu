// The bit-packed wire forms of the prover's first message, from where the device left it:
// wire::pack_commitment (crates/pcs/src/wire/mod.rs:226-245) of the commitment matrix and
// wire::pack_row_evaluation / pack_f162 (crates/pcs/src/wire/mod.rs:435-459) of the row values.
//
// Both are the reference's LSB-first bit stream (BitWriter::put, crates/pcs/src/wire/mod.rs:85-140):
// value after value, each in its low `bits` bits, least significant bit first, bytes filled from
// bit 0, the last byte zero-padded. On the device one thread makes one output byte: it locates the
// value holding the byte's first bit and walks its eight bits forward.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/labinius_gpu.h"
#include "error.h"
#include "handles.h"
#include "transcript.h"
#include "transcript_dev.h"

using namespace lbg;

namespace {

int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

#define LBG_CU(x)                                                                                    \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) return fail(LBG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// The commitment's residue stream: element e (column-major: column, then its four rows), limb f,
// slot s, value C[e][f][s] mod q_f in bits[f] bits.
struct ResidueStream {
  uint32_t limbs;
  uint32_t q[7];
  uint32_t bits[7];
  uint32_t elem_bits;  // 162 * sum bits[f]
};

__global__ void k_pack_residues(const int16_t* __restrict__ C, uint64_t elements, ResidueStream rs,
                                uint8_t* __restrict__ out, uint64_t nbytes) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nbytes) return;
  const uint64_t g = 8 * k;
  uint64_t e = g / rs.elem_bits;
  uint32_t r = (uint32_t)(g - e * rs.elem_bits);
  uint32_t f = 0;
  while (r >= 162u * rs.bits[f]) {
    r -= 162u * rs.bits[f];
    f++;
  }
  uint32_t s = r / rs.bits[f], b = r - s * rs.bits[f];
  uint32_t byte = 0;
  for (int t = 0; t < 8 && e < elements; t++) {
    const int32_t c = C[(e * rs.limbs + f) * 162 + s];
    const uint32_t v = (uint32_t)(c < 0 ? c + (int32_t)rs.q[f] : c);
    byte |= ((v >> b) & 1u) << t;
    if (++b == rs.bits[f]) {
      b = 0;
      if (++s == 162) {
        s = 0;
        if (++f == rs.limbs) {
          f = 0;
          e++;
        }
      }
    }
  }
  out[k] = (uint8_t)byte;
}

// F162 values at 162 bits each: value i's bit t is bit t % 64 of its word t / 64.
__global__ void k_pack_f162(const uint64_t* __restrict__ u, uint64_t count, uint8_t* __restrict__ out, uint64_t nbytes) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nbytes) return;
  uint32_t byte = 0;
  for (int t = 0; t < 8; t++) {
    const uint64_t g = 8 * k + t;
    const uint64_t i = g / 162;
    if (i >= count) break;
    const uint32_t bit = (uint32_t)(g - 162 * i);
    byte |= (uint32_t)((u[3 * i + bit / 64] >> (bit % 64)) & 1u) << t;
  }
  out[k] = (uint8_t)byte;
}

int grow_scratch(uint8_t** p, size_t* cap, size_t need) {
  if (*cap >= need) return LBG_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc((void**)p, need) != cudaSuccess) {
    cudaGetLastError();
    return fail(LBG_ERR_OOM, "wire scratch");
  }
  *cap = need;
  return LBG_OK;
}

// Bytes of wire::pack_commitment for these parameters (crates/pcs/src/wire/mod.rs:381-384; the
// bit-dropped form is pack_dropped's).
size_t commitment_wire_bytes(const lbg_pp* pp) {
  if (pp->params.opening == LBG_OPENING_BIT_DROPPED) {
    uint64_t bits = top_bits(pp->primes[0], pp->params.dropped_bits);
    for (int k = 1; k < pp->limbs; k++) bits += residue_bits(pp->primes[k]);
    return (size_t)((pp->cols * N648 * bits + 7) / 8);
  }
  uint64_t bits = 0;
  for (int k = 0; k < pp->limbs; k++) bits += residue_bits(pp->primes[k]);
  return (size_t)((4 * pp->cols * N162 * bits + 7) / 8);
}

}  // namespace

long long lbg_opening_pack_commitment(const lbg_opening* op, uint8_t* out, size_t cap) {
  if (!op) return fail(LBG_ERR_INVALID, "null argument");
  lbg_prover* pr = op->pr;
  const lbg_pp* pp = pr->pp;
  const size_t nbytes = commitment_wire_bytes(pp);
  if (!out) return (long long)nbytes;
  if (cap < nbytes) return fail(LBG_ERR_INVALID, "the output holds fewer bytes than the packed commitment");
  LBG_CU(cudaSetDevice(pp->device));
  std::lock_guard<std::mutex> g(pr->mu);
  int rc = grow_scratch(&pr->d_wire, &pr->wire_cap, nbytes);
  if (rc) return rc;
  const unsigned blocks = (unsigned)((nbytes + 255) / 256);
  if (pp->params.opening == LBG_OPENING_BIT_DROPPED) {
    PackDropped pk{};
    pk.limbs = (uint32_t)pp->limbs;
    pk.top_bits = top_bits(pp->primes[0], pp->params.dropped_bits);
    pk.bits_per = pk.top_bits;
    for (int k = 1; k < pp->limbs; k++) {
      pk.residue_bits[k] = residue_bits(pp->primes[k]);
      pk.bits_per += pk.residue_bits[k];
    }
    const uint64_t count = pp->cols * N648;
    LBG_CU(launch_pack_dropped(op->bufs->d_top, op->bufs->d_digits, count, count, pk, pr->d_wire, nbytes, pr->stream));
  } else {
    ResidueStream rs{};
    rs.limbs = (uint32_t)pp->limbs;
    for (int k = 0; k < pp->limbs; k++) {
      rs.q[k] = pp->primes[k];
      rs.bits[k] = residue_bits(pp->primes[k]);
      rs.elem_bits += 162 * rs.bits[k];
    }
    k_pack_residues<<<blocks, 256, 0, pr->stream>>>(op->bufs->d_C, 4 * (uint64_t)pp->cols, rs, pr->d_wire, nbytes);
    LBG_CU(cudaGetLastError());
  }
  LBG_CU(cudaMemcpyAsync(out, pr->d_wire, nbytes, cudaMemcpyDeviceToHost, pr->stream));
  LBG_CU(cudaStreamSynchronize(pr->stream));
  return (long long)nbytes;
}

long long lbg_row_evaluate_packed(const lbg_pp* pp_c, const lbg_witness* w, const uint64_t* p0, size_t p0_len,
                                  uint64_t* u_out, uint8_t* out, size_t cap) {
  if (!pp_c) return fail(LBG_ERR_INVALID, "null argument");
  lbg_pp* pp = const_cast<lbg_pp*>(pp_c);
  const size_t nbytes = (pp->cols * 162 + 7) / 8;  // wire::f162_bytes (crates/pcs/src/wire/mod.rs:472-474)
  if (!out) return (long long)nbytes;
  if (!w || !p0) return fail(LBG_ERR_INVALID, "null argument");
  if (cap < nbytes) return fail(LBG_ERR_INVALID, "the output holds fewer bytes than the packed row evaluation");
  if (p0_len != (size_t)(pp->params.witness_log_len - pp->params.column_log_len) || w->n != pp->n)
    return fail(LBG_ERR_INVALID, "the evaluation point does not match the witness");
  std::lock_guard<std::mutex> g(pp->mu);
  LBG_CU(cudaSetDevice(pp->device));
  int rc = grow_scratch(&pp->d_wire, &pp->wire_cap, nbytes);
  if (rc) return rc;
  LBG_CU(cudaMemcpyAsync(pp->d_p, p0, p0_len * 24, cudaMemcpyHostToDevice, pp->stream));
  LBG_CU(launch_eq_table(pp->d_p, (int)p0_len, pp->wdim, pp->d_eq, pp->stream));
  LBG_CU(launch_row_eval(w->d, pp->wdim, (int)pp->cols, pp->d_eq, pp->d_u, pp->stream));
  k_pack_f162<<<(unsigned)((nbytes + 255) / 256), 256, 0, pp->stream>>>(pp->d_u, pp->cols, pp->d_wire, nbytes);
  LBG_CU(cudaGetLastError());
  if (u_out) LBG_CU(cudaMemcpyAsync(u_out, pp->d_u, pp->cols * 24, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaMemcpyAsync(out, pp->d_wire, nbytes, cudaMemcpyDeviceToHost, pp->stream));
  LBG_CU(cudaStreamSynchronize(pp->stream));
  return (long long)nbytes;
}
