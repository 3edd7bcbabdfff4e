// The 648-point transform as an entry point of its own: the reference's forward NTT and its
// inverse on general coefficients (the NTT microbenchmark's kernels, kernels.cu), with the
// per-prime twiddle tables uploaded once per device.
#include <cuda_runtime.h>

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

std::mutex g_mu;
Ntt648Tables* g_tables[64][7] = {{nullptr}};

int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

int run(uint32_t q, bool inverse, const uint16_t* in, uint16_t* out, size_t count, void* stream) {
  int pi = prime_index(q);
  if (pi < 0) return fail(LBG_ERR_PARAMS, "unsupported modulus");
  const Ntt648Tables* host = ntt648_tables(q);
  if (!host) return fail(LBG_ERR_UNSUPPORTED, "the 648-point transform here covers splitting primes only");
  if (count && (!in || !out)) return fail(LBG_ERR_INVALID, "null argument");
  // the kernels store whole 32-bit words (16-byte chunks where both buffers allow)
  if ((((uintptr_t)in | (uintptr_t)out) & 3) != 0) return fail(LBG_ERR_INVALID, "buffers must be 4-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(LBG_ERR_CUDA, "no current device");
  Ntt648Tables* d = nullptr;
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_tables[dev][pi]) {
      Ntt648Tables* p = nullptr;
      if (cudaMalloc((void**)&p, sizeof(Ntt648Tables)) != cudaSuccess ||
          upload_sync(p, host, sizeof(Ntt648Tables)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return fail(LBG_ERR_CUDA, "transform tables");
      }
      g_tables[dev][pi] = p;
    }
    d = g_tables[dev][pi];
  }
  cudaError_t e = launch_ntt648(pi, inverse, in, out, count, d, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(LBG_ERR_CUDA, std::string("ntt648: ") + cudaGetErrorString(e));
  return LBG_OK;
}

}  // namespace

extern "C" {

int lbg_ntt648_forward(uint32_t q, const uint16_t* d_in, uint16_t* d_out, size_t count, void* stream) {
  return run(q, false, d_in, d_out, count, stream);
}

int lbg_ntt648_inverse(uint32_t q, const uint16_t* d_in, uint16_t* d_out, size_t count, void* stream) {
  return run(q, true, d_in, d_out, count, stream);
}

}  // extern "C"
