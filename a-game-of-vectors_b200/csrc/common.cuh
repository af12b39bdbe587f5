// common.cuh — shared device helpers of the sm_100a query path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sieve_gpu.h"

#define SG_DEV __device__ __forceinline__

namespace sg {

// Monotonic map of an f32 to u32 (larger float -> larger key). -0.0 is mapped with +0.0 so the
// key order equals the float `<` / `==` the reference's partial_cmp uses.
SG_DEV uint32_t ord(float f) {
  uint32_t u = __float_as_uint(__fadd_rn(f, 0.0f));
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
// Total order of f32::total_cmp (-0.0 < +0.0), used where the reference sorts by total_cmp.
SG_DEV uint32_t ord_total(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
SG_DEV float unord(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
  return __uint_as_float(u);
}

// (score desc, id asc) as one u64 where larger is better: the order TopK::into_sorted emits.
SG_DEV uint64_t rank_key(float score, uint32_t id) {
  return ((uint64_t)ord(score) << 32) | (uint64_t)(0xFFFFFFFFu - id);
}
SG_DEV float key_score(uint64_t k) { return unord((uint32_t)(k >> 32)); }
SG_DEV uint32_t key_id(uint64_t k) { return 0xFFFFFFFFu - (uint32_t)k; }

SG_DEV uint32_t warp_sum(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}
SG_DEV int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// Block-wide exclusive scan of one u32 per thread (blockDim.x <= 1024, multiple of 32).
// `tmp` needs 32 words of shared memory. Returns the exclusive prefix; *total gets the sum.
SG_DEV uint32_t block_exclusive_scan(uint32_t v, uint32_t* tmp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nw ? tmp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    tmp[lane] = w;  // inclusive prefix over warps
  }
  __syncthreads();
  uint32_t base = warp > 0 ? tmp[warp - 1] : 0;
  uint32_t t = tmp[nw - 1];
  __syncthreads();
  if (total) *total = t;
  return base + x - v;
}

SG_DEV uint32_t block_sum(uint32_t v, uint32_t* tmp) {
  uint32_t total;
  block_exclusive_scan(v, tmp, &total);
  return total;
}

// Radix select over u64 keys held in a caller-provided iterator: finds the n-th largest key
// (1-based) among `m` keys. All threads of the block call it; `hist` needs 256 words and `tmp`
// 32 words of shared memory. Keys are fetched through get(i) for i in [0, m).
template <typename Get>
SG_DEV uint64_t block_select_nth_u64(Get get, uint32_t m, uint32_t n, uint32_t* hist,
                                     uint32_t* tmp) {
  uint64_t prefix = 0, mask = 0;
  uint32_t remaining = n;
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      uint64_t k = get(i);
      if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    // find digit d such that count(digits > d) < remaining <= count(digits >= d)
    __shared__ uint32_t s_digit, s_above;
    if (threadIdx.x < 32) {
      // each lane owns 8 consecutive digits, from the top
      const int lane = threadIdx.x;
      uint32_t c[8], sum = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        c[j] = hist[255 - (lane * 8 + j)];
        sum += c[j];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t excl = incl - sum;
      if (excl < remaining && remaining <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          if (run < remaining && remaining <= run + c[j]) {
            s_digit = 255 - (lane * 8 + j);
            s_above = run;
          }
          run += c[j];
        }
      }
    }
    __syncthreads();
    uint32_t d = s_digit;
    remaining -= s_above;
    prefix |= (uint64_t)d << shift;
    mask |= (uint64_t)255 << shift;
    __syncthreads();
  }
  (void)tmp;
  return prefix;
}

// Bitonic sort of `n` u64 keys in shared memory, descending. n must be a power of two; pad with 0.
SG_DEV void block_bitonic_sort_desc(uint64_t* a, uint32_t n) {
  for (uint32_t size = 2; size <= n; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < n / 2; i += blockDim.x) {
        uint32_t lo = 2 * i - (i & (stride - 1));
        uint32_t hi = lo + stride;
        bool desc = ((lo & size) == 0);
        uint64_t x = a[lo], y = a[hi];
        if ((x < y) == desc) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      __syncthreads();
    }
  }
}

SG_DEV uint32_t next_pow2(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Allow-bitset membership of View::hidden (src/ivf.rs:474-483).
SG_DEV bool allowed(const uint64_t* allow, uint64_t words, uint32_t id) {
  uint64_t w = (uint64_t)id >> 6;
  return w < words && ((allow[w] >> (id & 63)) & 1ull);
}


// Radix select over u32 keys (4 passes of 8 bits): the n-th largest (1-based) of m keys read
// through get(i). Same contract as block_select_nth_u64.
template <typename Get>
SG_DEV uint32_t block_select_nth_u32(Get get, uint32_t m, uint32_t n, uint32_t* hist) {
  uint32_t prefix = 0, mask = 0, remaining = n;
  __shared__ uint32_t s_digit32, s_above32;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      uint32_t k = get(i);
      if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      uint32_t c[8], sum = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        c[j] = hist[255 - (lane * 8 + j)];
        sum += c[j];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t excl = incl - sum;
      if (excl < remaining && remaining <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          if (run < remaining && remaining <= run + c[j]) {
            s_digit32 = 255 - (lane * 8 + j);
            s_above32 = run;
          }
          run += c[j];
        }
      }
    }
    __syncthreads();
    uint32_t d = s_digit32;
    remaining -= s_above32;
    prefix |= d << shift;
    mask |= 255u << shift;
    __syncthreads();
  }
  return prefix;
}

// The same select over the ordered keys of a float row in global memory, with each thread's
// loads issued eight at a time before their histogram updates (a row of a routing score matrix
// is re-read once per pass; one load in flight per thread left the passes latency-bound).
SG_DEV uint32_t block_select_nth_row(const float* __restrict__ row, uint32_t m, uint32_t n, uint32_t* hist) {
  constexpr uint32_t kBatch = 8;
  uint32_t prefix = 0, mask = 0, remaining = n;
  __shared__ uint32_t s_digitr, s_abover;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t i0 = threadIdx.x; i0 < m; i0 += kBatch * blockDim.x) {
      uint32_t k[kBatch];
#pragma unroll
      for (uint32_t j = 0; j < kBatch; j++) {
        const uint32_t i = i0 + j * blockDim.x;
        k[j] = i < m ? ord(__ldg(row + i)) : 0u;
      }
#pragma unroll
      for (uint32_t j = 0; j < kBatch; j++)
        if (i0 + j * blockDim.x < m && (k[j] & mask) == prefix) atomicAdd(&hist[(k[j] >> shift) & 255], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      uint32_t c[8], sum = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        c[j] = hist[255 - (lane * 8 + j)];
        sum += c[j];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t excl = incl - sum;
      if (excl < remaining && remaining <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          if (run < remaining && remaining <= run + c[j]) {
            s_digitr = 255 - (lane * 8 + j);
            s_abover = run;
          }
          run += c[j];
        }
      }
    }
    __syncthreads();
    uint32_t d = s_digitr;
    remaining -= s_abover;
    prefix |= d << shift;
    mask |= 255u << shift;
    __syncthreads();
  }
  return prefix;
}

// Bitonic sort of (key, payload) pairs in shared memory by key, descending (n a power of two).
SG_DEV void block_bitonic_sort_desc_kv(uint64_t* a, uint32_t* v, uint32_t n) {
  for (uint32_t size = 2; size <= n; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < n / 2; i += blockDim.x) {
        uint32_t lo = 2 * i - (i & (stride - 1));
        uint32_t hi = lo + stride;
        bool desc = ((lo & size) == 0);
        uint64_t x = a[lo], y = a[hi];
        if ((x < y) == desc) {
          a[lo] = y;
          a[hi] = x;
          uint32_t t = v[lo];
          v[lo] = v[hi];
          v[hi] = t;
        }
      }
      __syncthreads();
    }
  }
}

SG_DEV uint32_t prmt(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// Four 16-entry u8 table lookups: the four nibbles of s[15:0] index table t (16 bytes). PRMT
// indexes 8 bytes with 3 bits, so entries 0-7 and 8-15 are looked up separately and bit 3 of each
// nibble then picks between the two results, byte by byte.
SG_DEV uint32_t lut4(uint32_t s, const uint4& t) {
  uint32_t idx = s & 0x7777u;
  uint32_t lo = prmt(t.x, t.y, idx);
  uint32_t hi = prmt(t.z, t.w, idx);
  uint32_t sel = ((s >> 1) & 0x4444u) | 0x3210u;
  return prmt(lo, hi, sel);
}

// One 4-byte word of a block's group (bytes 4j..4j+3 of the group's 16): adds the table values of
// its eight nibbles into four packed u16 pairs:
//   acc[0] += (doc 4j, 4j+1), acc[1] += (doc 4j+16, 4j+17),
//   acc[2] += (doc 4j+2, 4j+3), acc[3] += (doc 4j+18, 4j+19)   (low half, high half).
// Sums stay below 64 * 255 = 16320, so the halves never carry into each other.
SG_DEV void lut_word(uint32_t w, const uint4& t, uint32_t* acc) {
  uint32_t ra = lut4(w, t), rb = lut4(w >> 16, t);
  acc[0] += prmt(ra, 0u, 0x4240u);
  acc[1] += prmt(ra, 0u, 0x4341u);
  acc[2] += prmt(rb, 0u, 0x4240u);
  acc[3] += prmt(rb, 0u, 0x4341u);
}


SG_DEV uint32_t block_reduce_min(uint32_t v, uint32_t* tmp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t r = 0xFFFFFFFFu;
  for (uint32_t w = 0; w < (blockDim.x >> 5); w++) r = min(r, tmp[w]);
  __syncthreads();
  return r;
}

SG_DEV uint32_t block_reduce_max(uint32_t v, uint32_t* tmp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t r = 0;
  for (uint32_t w = 0; w < (blockDim.x >> 5); w++) r = max(r, tmp[w]);
  __syncthreads();
  return r;
}

// Range-adaptive radix select: the n-th largest (1-based, n <= m) of m u32 keys read through
// get(i). Keys of a query cluster in a narrow value range (the ordered bits of estimates that
// agree in sign, exponent and leading mantissa bits), so the select first reduces min and max
// and then runs 11-bit digits over (key - min) only: at most 3 passes, and the keys spread over
// the bins instead of piling onto one (same-address shared atomics serialise). `hist` needs 2048
// words and `tmp` 32 words of shared memory; every thread of the block calls it.
template <typename Get>
SG_DEV uint32_t block_select_nth_u32r(Get get, uint32_t m, uint32_t n, uint32_t* hist, uint32_t* tmp) {
  uint32_t lo = 0xFFFFFFFFu, hi = 0;
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const uint32_t k = get(i);
    lo = min(lo, k);
    hi = max(hi, k);
  }
  lo = block_reduce_min(lo, tmp);
  hi = block_reduce_max(hi, tmp);
  const uint32_t span = hi - lo;
  int top = span ? 32 - __clz(span) : 0;  // significant bits of (key - lo)
  uint32_t want = 0;                      // selected value of (key - lo) >> top
  uint32_t remaining = n;
  __shared__ uint32_t s_dig, s_above;
  while (top > 0) {
    const int shift = top > 11 ? top - 11 : 0;
    const int width = top - shift;
    const uint32_t nbins = 1u << width;
    for (uint32_t i = threadIdx.x; i < nbins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      const uint32_t r = get(i) - lo;
      if ((top >= 32 ? 0u : (r >> top)) == want) atomicAdd(&hist[(r >> shift) & (nbins - 1)], 1u);
    }
    __syncthreads();
    // bins from the top: thread t owns bins nbins-1-t*per .. (descending), per <= 8
    const uint32_t per = (nbins + blockDim.x - 1) / blockDim.x;
    uint32_t loc = 0;
    for (uint32_t j = 0; j < per; j++) {
      const uint32_t b = threadIdx.x * per + j;
      if (b < nbins) loc += hist[nbins - 1 - b];
    }
    uint32_t tot;
    const uint32_t excl = block_exclusive_scan(loc, tmp, &tot);
    if (excl < remaining && remaining <= excl + loc) {
      uint32_t run = excl;
      for (uint32_t j = 0; j < per; j++) {
        const uint32_t b = threadIdx.x * per + j;
        if (b >= nbins) break;
        const uint32_t c = hist[nbins - 1 - b];
        if (run < remaining && remaining <= run + c) {
          s_dig = nbins - 1 - b;
          s_above = run;
          break;
        }
        run += c;
      }
    }
    __syncthreads();
    want = (want << width) | s_dig;
    remaining -= s_above;
    top = shift;
    __syncthreads();
  }
  return lo + want;
}

// TopK(P) by (score desc, id asc) over ids 0..K-1 (1 <= P <= K), the scores read through
// score(i) (several times: min/max, up to three digit passes, a count, the gather): the winners'
// rank keys go to keys[0..P), unordered. `hist` needs 2048 words and `tmp` 32; every thread of the
// block calls it.
template <typename Score>
SG_DEV void block_top_keys(Score score, uint32_t K, uint32_t P, uint64_t* keys, uint32_t* hist, uint32_t* tmp) {
  __shared__ uint32_t s_top_n;
  auto okey = [&](uint32_t i) { return ord(score(i)); };
  const uint32_t T = block_select_nth_u32r(okey, K, P, hist, tmp);
  uint32_t gt = 0, eq = 0;
  for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
    const uint32_t o = okey(i);
    gt += o > T;
    eq += o == T;
  }
  const uint32_t n_gt = block_sum(gt, tmp), n_eq = block_sum(eq, tmp);
  const uint32_t need = P - n_gt;  // >= 1: T is the P-th largest
  uint32_t Kt = 0;  // among ids at T, keep those with 0xFFFFFFFF - id >= Kt (the lowest `need`)
  if (n_eq > need)
    Kt = block_select_nth_u32r([&](uint32_t i) { return okey(i) == T ? 0xFFFFFFFFu - i : 0u; }, K, need, hist, tmp);
  if (threadIdx.x == 0) s_top_n = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
    const float v = score(i);
    const uint32_t o = ord(v);
    if (o > T || (o == T && 0xFFFFFFFFu - i >= Kt)) keys[atomicAdd(&s_top_n, 1u)] = rank_key(v, i);
  }
  __syncthreads();
}

}  // namespace sg
