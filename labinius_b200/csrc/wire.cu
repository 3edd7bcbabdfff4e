// wire::encode of the folded witness on the device (crates/pcs/src/wire/rans.rs:18-105): interleaved
// static rANS over 64 lanes against the message's own histogram.
//
// The reference codes coefficient i with lane i mod 64, walking the groups of 64 from the last to
// the first and the lanes of a group from the last to the first, and pushes every renormalisation
// word onto one shared stack, which the output holds in reverse. Each lane's state depends on its
// own symbols only, so the lanes run as independent threads that record, per coefficient, the
// words it emits; the output order (the reverse of the push order) is the natural order of the
// coefficients, so an exclusive scan of the per-coefficient word counts places every word.
//  * k_wire_minmax, k_wire_hist: the range and the histogram of the coefficients;
//  * the quantisation of the histogram to 4096 slots, the Elias-gamma frequency table and the
//    encoder's symbols (reciprocal, frequency, bias) on the host: a few thousand entries;
//  * k_wire_lanes: one thread per lane, the coefficients staged through shared memory by tiles
//    of 128 groups;
//  * k_wire_scan_*: the exclusive scan of the word counts; k_wire_scatter: the words into place.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/labinius_gpu.h"
#include "error.h"
#include "handles.h"

namespace lbg {
namespace {

constexpr uint32_t SCALE_BITS = 12, SCALE = 1u << SCALE_BITS, RANS_LOW = 1u << 16;
constexpr size_t HEADER = 16, LANES = 64, MAX_ELEMENTS = (size_t)1 << 24;
constexpr int TILE_GROUPS = 128;
constexpr int SCAN_BLOCK = 1024;

struct WireSym {
  uint64_t reciprocal;
  uint32_t frequency, bias;
};

int fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}

__global__ void k_wire_minmax(const int16_t* __restrict__ v, size_t n, int* __restrict__ lohi) {
  int lo = 32767, hi = -32768;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int x = v[i];
    lo = min(lo, x);
    hi = max(hi, x);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(lohi, lo);
    atomicMax(lohi + 1, hi);
  }
}

// counts[s] for s < length (the symbol x - low); in shared memory when the range is small
__global__ void k_wire_hist(const int16_t* __restrict__ v, size_t n, int low, uint32_t length,
                            unsigned long long* __restrict__ counts) {
  extern __shared__ uint32_t h[];
  const bool local = length <= 8192;
  if (local)
    for (uint32_t s = threadIdx.x; s < length; s += blockDim.x) h[s] = 0;
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t s = (uint32_t)(v[i] - low);
    if (local)
      atomicAdd(h + s, 1u);
    else
      atomicAdd(counts + s, 1ull);
  }
  __syncthreads();
  if (local)
    for (uint32_t s = threadIdx.x; s < length; s += blockDim.x)
      if (h[s]) atomicAdd(counts + s, (unsigned long long)h[s]);
}

// x / f as the reference divides (x * reciprocal) >> 64, for x < 2^32: two 32 x 32 products.
__device__ __forceinline__ uint32_t quotient(uint32_t x, uint64_t r) {
  const uint64_t lo = (uint64_t)x * (uint32_t)r;
  return (uint32_t)(((uint64_t)x * (uint32_t)(r >> 32) + (lo >> 32)) >> 32);
}

// One thread per lane. cnt[i]: the words coefficient i pushed (0, 1 or 2); w2[i]: those words in
// the output's order (the reverse of the push order), the first in the low half; states: the
// lanes' final states. The symbol table is copied to shared memory when it fits (sym_smem); the
// step loop is unrolled so the table reads of later steps overlap a step's state update.
__global__ void __launch_bounds__(LANES) k_wire_lanes(const int16_t* __restrict__ v, uint32_t coefficients, int low,
                                                      uint32_t length, uint32_t raw, const WireSym* __restrict__ gsyms,
                                                      int sym_smem, uint8_t* __restrict__ cnt,
                                                      uint32_t* __restrict__ w2, uint32_t* __restrict__ states) {
  __shared__ __align__(16) int16_t tile[TILE_GROUPS * LANES];
  extern __shared__ WireSym ssyms[];
  const uint32_t k = threadIdx.x;
  if (sym_smem)
    for (uint32_t e = k; e <= length; e += LANES) ssyms[e] = gsyms[e];
  const WireSym* syms = sym_smem ? ssyms : gsyms;
  const uint32_t groups = (coefficients + (uint32_t)LANES - 1) / (uint32_t)LANES;
  __syncthreads();
  const WireSym esc = syms[length];
  uint32_t x = RANS_LOW;
  for (uint32_t end = groups; end > 0;) {
    const uint32_t first = end > (uint32_t)TILE_GROUPS ? end - TILE_GROUPS : 0;
    const uint32_t base = first * (uint32_t)LANES, span = (end - first) * (uint32_t)LANES;
    if (base + span <= coefficients) {  // 8 coefficients a load (base is a multiple of 64)
      const uint4* src = reinterpret_cast<const uint4*>(v + base);
      uint4* dst = reinterpret_cast<uint4*>(tile);
      for (uint32_t t = k; t < span / 8; t += LANES) dst[t] = src[t];
    } else {
      for (uint32_t t = k; t < span; t += LANES) tile[t] = base + t < coefficients ? v[base + t] : 0;
    }
    __syncthreads();
    const bool full = end * (uint32_t)LANES <= coefficients;  // every lane of this tile's groups is coded
#pragma unroll 4
    for (uint32_t g = end; g-- > first;) {
      const uint32_t i = g * (uint32_t)LANES + k;
      const uint32_t s = (uint32_t)(tile[(g - first) * LANES + k] - low);
      WireSym y = syms[s < length ? s : length];
      if (!full && i >= coefficients) continue;
      uint32_t bits_word = 0, sym_word = 0, n_bits = 0, n_sym = 0;
      if (y.frequency == 0) {  // the escape symbol after the raw index
        if (raw) {
          n_bits = (x >> (32 - raw)) != 0;
          bits_word = x & 0xFFFF;
          x = n_bits ? x >> 16 : x;
          x = (x << raw) | s;
        }
        y = esc;
      }
      n_sym = (x >> (32 - SCALE_BITS)) >= y.frequency;  // renormalise
      sym_word = x & 0xFFFF;
      x = n_sym ? x >> 16 : x;
      const uint32_t q = quotient(x, y.reciprocal);
      x = (q << SCALE_BITS) + (x - q * y.frequency) + y.bias;
      cnt[i] = (uint8_t)(n_bits + n_sym);
      // output order: the symbol's word, then the raw bits' word
      w2[i] = n_sym ? (sym_word | (n_bits ? bits_word << 16 : 0)) : bits_word;
    }
    __syncthreads();
    end = first;
  }
  states[k] = x;
}

// exclusive scan of cnt: per-block sums, their scan (one block), the offsets added per element
__global__ void k_wire_scan_blocks(const uint8_t* __restrict__ cnt, size_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t red[SCAN_BLOCK / 32];
  const size_t i = (size_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
  uint32_t x = i < n ? cnt[i] : 0;
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < SCAN_BLOCK / 32; w++) t += red[w];
    sums[blockIdx.x] = t;
  }
}

__global__ void k_wire_scan_sums(uint32_t* __restrict__ sums, size_t nb, uint32_t* __restrict__ total) {
  // one block: a sequential carry over chunks of blockDim entries, each scanned in shared memory
  __shared__ uint32_t buf[SCAN_BLOCK];
  uint32_t carry = 0;
  for (size_t c0 = 0; c0 < nb; c0 += SCAN_BLOCK) {
    const size_t i = c0 + threadIdx.x;
    buf[threadIdx.x] = i < nb ? sums[i] : 0;
    __syncthreads();
    for (int o = 1; o < SCAN_BLOCK; o <<= 1) {
      uint32_t y = threadIdx.x >= (unsigned)o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < nb) sums[i] = carry + buf[threadIdx.x];  // inclusive
    const uint32_t chunk_total = buf[SCAN_BLOCK - 1];
    __syncthreads();
    carry += chunk_total;
  }
  if (threadIdx.x == 0) *total = carry;
}

// sums[b] is now the inclusive scan of the block sums; element i's position is the block's
// exclusive offset plus its exclusive rank within the block
__global__ void k_wire_scatter(const uint8_t* __restrict__ cnt, const uint32_t* __restrict__ w2, size_t n,
                               const uint32_t* __restrict__ sums, uint8_t* __restrict__ out_words) {
  __shared__ uint32_t wsum[SCAN_BLOCK / 32];
  const size_t i = (size_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
  const uint32_t c = i < n ? cnt[i] : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < SCAN_BLOCK / 32 ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < SCAN_BLOCK / 32) wsum[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t block_off = blockIdx.x ? sums[blockIdx.x - 1] : 0;
  const uint32_t pos = block_off + (warp ? wsum[warp - 1] : 0) + incl - c;
  const uint32_t ws = c ? w2[i] : 0;
  for (uint32_t e = 0; e < c; e++) {
    const uint32_t w = ws >> (16 * e);
    out_words[2 * (pos + e)] = (uint8_t)w;
    out_words[2 * (pos + e) + 1] = (uint8_t)(w >> 8);
  }
}

// ---- host side of the coder: the quantised histogram and the symbols -----------------------
struct Bits {
  std::vector<uint8_t> bytes;
  uint64_t acc = 0;
  uint32_t n = 0;
  void put(uint64_t value, uint32_t bits) {
    acc |= (value & ((1ull << bits) - 1)) << n;
    n += bits;
    while (n >= 8) {
      bytes.push_back((uint8_t)acc);
      acc >>= 8;
      n -= 8;
    }
  }
  // Elias gamma of value >= 1 (crates/pcs/src/wire/mod.rs:123-130), each field LSB first
  void gamma(uint64_t value) {
    uint32_t k = 63 - __builtin_clzll(value);
    put(0, k);
    put(1, 1);
    if (k <= 32) {
      put(value & ((1ull << k) - 1), k);
    } else {
      put(value, 32);
      put(value >> 32, k - 32);
    }
  }
};

// The counts scaled to a total of exactly 4096 (crates/pcs/src/wire/rans.rs:231-268): every
// occupied symbol keeps a slot, the rest by largest remainder (ties to the lower symbol), and
// beyond 4095 occupied symbols the rarest fold into the escape symbol, the last entry.
std::vector<uint32_t> quantise(std::vector<uint64_t> w) {
  const size_t escape = w.size() - 1;
  std::vector<size_t> occupied;
  for (size_t i = 0; i < escape; i++)
    if (w[i]) occupied.push_back(i);
  if (occupied.size() > SCALE - 1) {
    std::stable_sort(occupied.begin(), occupied.end(), [&](size_t a, size_t b) { return w[a] > w[b]; });
    for (size_t j = SCALE - 1; j < occupied.size(); j++) {
      w[escape] += w[occupied[j]];
      w[occupied[j]] = 0;
    }
  }
  uint64_t total = 0;
  occupied.clear();
  for (size_t i = 0; i < w.size(); i++) {
    total += w[i];
    if (w[i]) occupied.push_back(i);
  }
  std::vector<uint32_t> f(w.size(), 0);
  if (occupied.empty()) return f;
  const uint64_t spare = SCALE - occupied.size();
  uint64_t used = 0;
  std::vector<std::pair<uint64_t, size_t>> rem;
  rem.reserve(occupied.size());
  for (size_t i : occupied) {
    const uint64_t share = w[i] * spare / total;
    f[i] = 1 + (uint32_t)share;
    used += share;
    rem.push_back({w[i] * spare - share * total, i});
  }
  std::stable_sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  for (uint64_t j = 0; j < spare - used; j++) f[rem[j].second] += 1;
  return f;
}

void put_le(std::vector<uint8_t>& out, uint64_t v, int bytes) {
  for (int i = 0; i < bytes; i++) out.push_back((uint8_t)(v >> (8 * i)));
}

// The coder's device scratch, kept per device between calls (grown on demand); a call holds mu.
struct Scratch {
  std::mutex mu;
  void* p[9] = {nullptr};
  size_t cap[9] = {0};
  cudaError_t get(int slot, size_t bytes, void** out) {
    if (bytes > cap[slot]) {
      cudaFree(p[slot]);
      p[slot] = nullptr;
      cap[slot] = 0;
      cudaError_t e = cudaMalloc(&p[slot], bytes);
      if (e != cudaSuccess) return e;
      cap[slot] = bytes;
    }
    *out = p[slot];
    return cudaSuccess;
  }
};
Scratch& scratch(int device) {
  static Scratch s[64];
  return s[device & 63];
}

}  // namespace

// The coder over `elements` ring elements of 648 coefficients at d_v (device memory), on stream
// st; bytes into out (host, cap bytes). Returns the byte count, or a negative status.
long long wire_encode_device(const int16_t* d_v, size_t elements, uint16_t base_q, uint8_t* out, size_t cap,
                             cudaStream_t st) {
  if (elements > MAX_ELEMENTS) return fail(LBG_ERR_INVALID, "more elements than the wire format holds");
  const size_t n = elements * 648;
  if (n >= ((size_t)1 << 31)) return fail(LBG_ERR_INVALID, "the word positions are 32-bit: at most 2^31 coefficients");
  std::vector<uint8_t> head;
  head.push_back(1);
  head.push_back(0);  // Representation::Coefficients
  put_le(head, base_q, 2);
  put_le(head, (uint32_t)elements, 4);
  if (n == 0) {
    put_le(head, 0, 4);
    put_le(head, 0, 4);
    if (out && cap >= head.size()) std::memcpy(out, head.data(), head.size());
    return (long long)head.size();
  }
  int device = 0;
  cudaGetDevice(&device);
  Scratch& S = scratch(device);
  std::lock_guard<std::mutex> lock(S.mu);
  int* d_lohi = nullptr;
  unsigned long long* d_counts = nullptr;
  WireSym* d_syms = nullptr;
  uint8_t *d_cnt = nullptr, *d_out = nullptr;
  uint32_t* d_w2 = nullptr;
  uint32_t *d_states = nullptr, *d_sums = nullptr, *d_total = nullptr;
  auto cuda_fail = [&](cudaError_t e) {
    cudaGetLastError();
    return (long long)fail(LBG_ERR_CUDA, std::string("wire encode: ") + cudaGetErrorString(e));
  };
  const size_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  cudaError_t e = S.get(0, 8, (void**)&d_lohi);
  if (e == cudaSuccess) e = S.get(1, n, (void**)&d_cnt);
  if (e == cudaSuccess) e = S.get(2, 4 * n, (void**)&d_w2);
  if (e == cudaSuccess) e = S.get(3, 4 * LANES, (void**)&d_states);
  if (e == cudaSuccess) e = S.get(4, 4 * nb, (void**)&d_sums);
  if (e == cudaSuccess) e = S.get(5, 4, (void**)&d_total);
  if (e != cudaSuccess) return cuda_fail(e);
  int lohi[2] = {32767, -32768};
  e = cudaMemcpyAsync(d_lohi, lohi, 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_wire_minmax<<<592, 256, 0, st>>>(d_v, n, d_lohi);
    e = cudaMemcpyAsync(lohi, d_lohi, 8, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e);
  const int low = lohi[0];
  const uint32_t length = (uint32_t)(lohi[1] - lohi[0] + 1);
  put_le(head, (uint32_t)low, 4);
  put_le(head, length, 4);
  e = S.get(6, 8 * (size_t)length, (void**)&d_counts);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_counts, 0, 8 * (size_t)length, st);
  if (e == cudaSuccess) {
    k_wire_hist<<<592, 256, length <= 8192 ? length * 4 : 0, st>>>(d_v, n, low, length, d_counts);
    e = cudaGetLastError();
  }
  std::vector<uint64_t> counts(length + 1, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(counts.data(), d_counts, 8 * (size_t)length, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e);
  // the frequencies, their gamma codes, the symbols
  std::vector<uint32_t> f = quantise(counts);
  Bits bits;
  for (uint32_t x : f) bits.gamma((uint64_t)x + 1);
  if (bits.n) bits.bytes.push_back((uint8_t)bits.acc);
  head.insert(head.end(), bits.bytes.begin(), bits.bytes.end());
  std::vector<WireSym> syms(length + 1);
  uint32_t start = 0;
  for (size_t s = 0; s <= length; s++) {
    const uint32_t fr = f[s];
    if (fr == 0)
      syms[s] = {0, 0, 0};
    else if (fr == 1)
      syms[s] = {~0ull, 1, start + SCALE - 1};
    else
      syms[s] = {~0ull / fr + 1, fr, start};
    start += fr;
  }
  const uint32_t raw = length <= 1 ? 0 : 64 - __builtin_clzll((uint64_t)(length - 1));
  e = S.get(7, sizeof(WireSym) * (length + 1), (void**)&d_syms);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_syms, syms.data(), sizeof(WireSym) * (length + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    const size_t sym_bytes = sizeof(WireSym) * (length + 1);
    const int sym_smem = sym_bytes <= 160 * 1024;
    if (sym_smem)
      cudaFuncSetAttribute(k_wire_lanes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_bytes);
    k_wire_lanes<<<1, LANES, sym_smem ? sym_bytes : 0, st>>>(d_v, (uint32_t)n, low, length, raw, d_syms, sym_smem,
                                                             d_cnt, d_w2, d_states);
    k_wire_scan_blocks<<<(unsigned)nb, SCAN_BLOCK, 0, st>>>(d_cnt, n, d_sums);
    k_wire_scan_sums<<<1, SCAN_BLOCK, 0, st>>>(d_sums, nb, d_total);
    e = cudaGetLastError();
  }
  uint32_t top = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&top, d_total, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e);
  const size_t total = head.size() + 4 * LANES + 2 * (size_t)top;
  if (!out || cap < total) {
    return (long long)total;  // the size; nothing written
  }
  e = S.get(8, 4 * LANES + 2 * (size_t)top + 16, (void**)&d_out);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, d_states, 4 * LANES, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    k_wire_scatter<<<(unsigned)nb, SCAN_BLOCK, 0, st>>>(d_cnt, d_w2, n, d_sums, d_out + 4 * LANES);
    e = cudaGetLastError();
  }
  std::memcpy(out, head.data(), head.size());
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out + head.size(), d_out, 4 * LANES + 2 * (size_t)top, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e);
  return (long long)total;
}

}  // namespace lbg

using namespace lbg;

extern "C" {

size_t lbg_wire_encode_bound(size_t elements) {
  // header, the gamma table (at most 65537 entries of at most 2 * 13 + 1 bits), the states, and
  // at most two words per coefficient
  return HEADER + (65537 * 27 + 7) / 8 + 4 * LANES + 2 * (2 * elements * 648 + 1);
}

long long lbg_wire_encode(const int16_t* v, size_t elements, uint32_t base_q, uint8_t* out, size_t cap) {
  if ((!v && elements) || base_q > 0xFFFF) return fail(LBG_ERR_INVALID, "null argument");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(LBG_ERR_CUDA, "no CUDA device");
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail(LBG_ERR_CUDA, "stream");
  int16_t* d_v = nullptr;
  const size_t n = elements * 648;
  long long r;
  if (n && cudaMalloc((void**)&d_v, 2 * n) != cudaSuccess) {
    cudaGetLastError();
    r = fail(LBG_ERR_OOM, "wire encode: device allocation failed");
  } else if (n && cudaMemcpyAsync(d_v, v, 2 * n, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    r = fail(LBG_ERR_CUDA, "wire encode: upload");
  } else {
    r = wire_encode_device(d_v, elements, (uint16_t)base_q, out, cap, st);
  }
  cudaStreamSynchronize(st);
  cudaFree(d_v);
  cudaStreamDestroy(st);
  return r;
}

long long lbg_prover_encode_folded(lbg_prover* pr, uint8_t* out, size_t cap) {
  if (!pr) return fail(LBG_ERR_INVALID, "null prover");
  const lbg_pp* pp = pr->pp;
  if (cudaSetDevice(pp->device) != cudaSuccess) return fail(LBG_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(pr->mu);
  return wire_encode_device(pr->d_v, pp->len_ring, (uint16_t)pp->primes[0], out, cap, pr->stream);
}

}  // extern "C"
