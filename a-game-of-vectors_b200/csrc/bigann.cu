// bigann.cu — the billion-scale L2 query path of bigann::Index (src/bigann.rs:634-747) on one GPU.
//
// Rows are int8 x 100; a query q (int8 x 100) ranks rows by s(x) = 2<q,x> - |x|^2. The stages:
//   route      (src/bigann.rs:660-678): the TopK(nprobe) of 2<q,c> - |c|^2 over every leaf, then the
//              margin rule on |q - c|^2. By default on the tcgen05 tensor cores with an exact FP32
//              rescoring window (bg_route.cu); params.route_fp32 scores every leaf with the
//              reference's sequential f32 dot instead (k_bg_scores + k_bg_select). Both give the
//              same probe lists.
//   candidates (src/bigann.rs:683-732): 32-group LUT scan of the probed leaves' 128-bit codes,
//              est = 2 (cent + mul (a s + b)) - |x|^2, a TopK of the best `cand` (or, on a
//              multi-bit index with refine > 0, a 1-bit shortlist TopK(max(refine, cand)) whose
//              admissions are re-estimated from all bit planes (Refiner) into a TopK(cand)).
//   rerank     (src/bigann.rs:735-747): exact 2 <q, x> - |x|^2 from the base rows, TopK(k).
// Every record is resident in HBM, so leaves are scanned in probe order, as Postings::fetch_each
// does when every record is pinned (src/postings.rs:287-303).
//
// The shortlist's admissions depend on the order slots arrive in: its threshold rises each time
// its buffer of 2K admitted entries is compacted to the best K (src/topk.rs:26-45). k_bg_scan
// therefore runs one CTA per query and replays that sequence exactly, a chunk of 2048 slots at a
// time: the chunk is scored in parallel, then admitted in slot order with block-wide prefix
// counts, stopping at each compaction to raise the threshold before admitting the rest.
#include <float.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace sg {

constexpr int BD = SG_BG_DIM, BPD = SG_BG_PDIM, BGR = SG_BG_GROUPS, BCODE = SG_BG_CODE;
constexpr int BBB = SG_BG_BLOCK_BYTES;
constexpr uint32_t kBgMax = 4096;      // largest nprobe, cand, refine and k
constexpr uint32_t kBgStepBlocks = 64;  // blocks scored per step of the scan (2048 slots)

// ---- per-query preparation: one CTA of 128 threads per query --------------------------------
// rabitq::Query::new over the padded query (src/rabitq.rs:119-125) for 32 groups, |q|^2 for the
// margin rule, and the Refiner tables (src/bigann.rs:575-585) when the index refines.
__global__ void __launch_bounds__(128) k_bg_prep(const int8_t* __restrict__ qin,
                                                 const float* __restrict__ signs, float rot_norm,
                                                 uint32_t bits, int refine,
                                                 uint8_t* __restrict__ tables,
                                                 float4* __restrict__ qp, float* __restrict__ qq,
                                                 float* __restrict__ rtab,
                                                 float* __restrict__ roff) {
  __shared__ float v[BPD];
  __shared__ float f[BGR * 16];
  __shared__ float mins[BGR], maxs[BGR];
  __shared__ float tab[BCODE * 256];
  __shared__ float s_scale;
  const int q = blockIdx.x, t = threadIdx.x;
  const int8_t* x = qin + (size_t)q * BD;
  if (t == 0) {
    float s = -0.0f;
    for (int i = 0; i < BD; i++) s = __fadd_rn(s, __fmul_rn((float)x[i], (float)x[i]));
    qq[q] = s;
  }
  v[t] = t < BD ? (float)x[t] : 0.0f;
  __syncthreads();
  for (int r = 0; r < 3; r++) {
    v[t] = __fmul_rn(v[t], signs[r * BPD + t]);
    __syncthreads();
    for (int h = 1; h < BPD; h *= 2) {
      if (t < BPD / 2) {
        const int blk = t / h, i = t % h;
        const int a = blk * 2 * h + i, b = a + h;
        const float xa = v[a], yb = v[b];
        v[a] = __fadd_rn(xa, yb);
        v[b] = __fsub_rn(xa, yb);
      }
      __syncthreads();
    }
  }
  v[t] = __fmul_rn(v[t], rot_norm);
  __syncthreads();
  for (int e = t; e < BGR * 16; e += blockDim.x) {
    const int g = e >> 4, c = e & 15;
    float s = -0.0f;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if ((c >> j) & 1) s = __fadd_rn(s, v[4 * g + j]);
    f[e] = s;
  }
  __syncthreads();
  if (t < BGR) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int c = 0; c < 16; c++) {
      mn = fminf(mn, f[t * 16 + c]);
      mx = fmaxf(mx, f[t * 16 + c]);
    }
    mins[t] = mn;
    maxs[t] = mx;
  }
  __syncthreads();
  if (t == 0) {
    float max_range = 0.0f;
    for (int g = 0; g < BGR; g++) max_range = fmaxf(max_range, __fsub_rn(maxs[g], mins[g]));
    const float scale = max_range > 0.0f ? __fdiv_rn(255.0f, max_range) : 1.0f;
    float bias = -0.0f;
    for (int g = 0; g < BGR; g++) bias = __fadd_rn(bias, mins[g]);
    float sum = -0.0f;
    for (int i = 0; i < BPD; i++) sum = __fadd_rn(sum, v[i]);
    qp[q] = make_float4(scale, bias, __fdiv_rn(2.0f, scale), __fsub_rn(__fmul_rn(2.0f, bias), sum));
    s_scale = scale;
    if (refine) {
      const float h = __fdiv_rn((float)((1u << bits) - 1), 2.0f);
      roff[q] = __fmul_rn(h, sum);
    }
  }
  __syncthreads();
  const float scale = s_scale;
  uint8_t* tq = tables + (size_t)q * BGR * 16;
  for (int e = t; e < BGR * 16; e += blockDim.x) {
    float r = roundf(__fmul_rn(__fsub_rn(f[e], mins[e >> 4]), scale));
    r = fminf(fmaxf(r, 0.0f), 255.0f);
    tq[e] = (uint8_t)r;
  }
  if (!refine) return;
  // Refiner tables: tab[k][v] = tab[k][v & (v - 1)] + qr[8k + tz(v)], by rising popcount so
  // every entry is the reference's single add of the same two operands.
  for (int e = t; e < BCODE * 256; e += blockDim.x)
    if ((e & 255) == 0) tab[e] = 0.0f;
  __syncthreads();
  for (int pc = 1; pc <= 8; pc++) {
    for (int e = t; e < BCODE * 256; e += blockDim.x) {
      const int k = e >> 8, w = e & 255;
      if (__popc(w) == pc) tab[e] = __fadd_rn(tab[(k << 8) | (w & (w - 1))], v[8 * k + __ffs(w) - 1]);
    }
    __syncthreads();
  }
  float* out = rtab + (size_t)q * BCODE * 256;
  for (int e = t; e < BCODE * 256; e += blockDim.x) out[e] = tab[e];
}

// |c|^2 of every leaf, sequential from -0.0 (norms(), src/bigann.rs:134-136).
__global__ void k_bg_leaf_norm(const float* __restrict__ leaves, uint32_t K, float* __restrict__ ln) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  float s = -0.0f;
  for (int i = 0; i < BD; i++) {
    const float y = leaves[(size_t)c * BD + i];
    s = __fadd_rn(s, __fmul_rn(y, y));
  }
  ln[c] = s;
}

// ---- routing scores: 2 <q, c> - |c|^2 for every (query, leaf) ---------------------------------
// One thread per leaf, 8 queries per CTA row; leaves transposed ([100][K]) so the reads coalesce.
// The dot runs in the reference's order: x[0]*y[0] + x[1]*y[1] + ... from -0.0 (gemm_abt).
constexpr int kBgRouteQ = 8;
__global__ void __launch_bounds__(256) k_bg_scores(const int8_t* __restrict__ qin, uint32_t nq,
                                                   const float* __restrict__ leaves_t,
                                                   const float* __restrict__ ln, uint32_t K,
                                                   float* __restrict__ scores) {
  __shared__ float qs[kBgRouteQ][BD];
  const uint32_t q0 = blockIdx.y * kBgRouteQ;
  for (int e = threadIdx.x; e < kBgRouteQ * BD; e += blockDim.x) {
    const uint32_t qi = q0 + e / BD;
    qs[e / BD][e % BD] = qi < nq ? (float)qin[(size_t)qi * BD + e % BD] : 0.0f;
  }
  __syncthreads();
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  float acc[kBgRouteQ];
#pragma unroll
  for (int j = 0; j < kBgRouteQ; j++) acc[j] = -0.0f;
  for (int i = 0; i < BD; i++) {
    const float y = leaves_t[(size_t)i * K + c];
#pragma unroll
    for (int j = 0; j < kBgRouteQ; j++) acc[j] = __fadd_rn(acc[j], __fmul_rn(qs[j][i], y));
  }
  const float n = ln[c];
#pragma unroll
  for (int j = 0; j < kBgRouteQ; j++)
    if (q0 + j < nq) scores[(size_t)(q0 + j) * K + c] = __fsub_rn(__fmul_rn(2.0f, acc[j]), n);
}

// ---- probe selection: one CTA (1024 threads) per query ----------------------------------------
// TopK(nprobe) by (score desc, leaf asc), the margin rule, and for each kept leaf its exact dot
// <q, c> (the `cent` of the candidates' estimates).
__global__ void __launch_bounds__(1024) k_bg_select(const float* __restrict__ scores, uint32_t K,
                                                    uint32_t P, float margin,
                                                    const float* __restrict__ qq,
                                                    const int8_t* __restrict__ qin,
                                                    const float* __restrict__ leaves,
                                                    uint32_t* __restrict__ probe,
                                                    float* __restrict__ probe_cent,
                                                    uint32_t* __restrict__ probe_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw);  // [next_pow2(P)]
  __shared__ uint32_t hist[2048], tmp[32], s_n, s_m;
  __shared__ float qf[BD];
  const uint32_t q = blockIdx.x;
  if (P == 0) {
    if (threadIdx.x == 0) probe_n[q] = 0;
    return;
  }
  const float* row = scores + (size_t)q * K;
  auto okey = [&](uint32_t i) { return ord(row[i]); };
  const uint32_t T = block_select_nth_u32r(okey, K, P, hist, tmp);
  uint32_t gt = 0, eq = 0;
  for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
    const uint32_t o = okey(i);
    gt += o > T;
    eq += o == T;
  }
  const uint32_t n_gt = block_sum(gt, tmp), n_eq = block_sum(eq, tmp);
  const uint32_t need = P - n_gt;
  uint32_t Kt = 0;
  if (n_eq > need)
    Kt = block_select_nth_u32r([&](uint32_t i) { return okey(i) == T ? 0xFFFFFFFFu - i : 0u; }, K,
                               need, hist, tmp);
  if (threadIdx.x == 0) s_n = 0;
  if (threadIdx.x < BD) qf[threadIdx.x] = (float)qin[(size_t)q * BD + threadIdx.x];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
    const uint32_t o = okey(i);
    if (o > T || (o == T && 0xFFFFFFFFu - i >= Kt)) keys[atomicAdd(&s_n, 1u)] = rank_key(row[i], i);
  }
  __syncthreads();
  const uint32_t n2 = next_pow2(P);
  for (uint32_t i = P + threadIdx.x; i < n2; i += blockDim.x) keys[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc(keys, n2);
  if (threadIdx.x == 0) {
    uint32_t m = P;
    if (margin > 0.0f) {
      // route score = |q|^2 - |q - c|^2; keep |q - c|^2 <= (1 + margin) |q - c1|^2
      const float Q = qq[q];
      const float lim = __fmul_rn(__fsub_rn(Q, key_score(keys[0])), __fadd_rn(1.0f, margin));
      uint32_t w = 0;
      while (w < m && __fsub_rn(Q, key_score(keys[w])) <= lim) w++;
      m = w;
    }
    s_m = m;
    probe_n[q] = m;
  }
  __syncthreads();
  const uint32_t m = s_m;
  for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) {
    const uint32_t c = key_id(keys[r]);
    float d = -0.0f;
    for (int i = 0; i < BD; i++) d = __fadd_rn(d, __fmul_rn(qf[i], leaves[(size_t)c * BD + i]));
    probe[(size_t)q * P + r] = c;
    probe_cent[(size_t)q * P + r] = d;
  }
}

// ---- the candidate scan: one CTA (256 threads) per query --------------------------------------
struct BgScanArgs {
  const uint8_t* blocks;
  const float2* factors;
  const uint32_t* ids;
  const uint8_t* ext;
  uint32_t extra, bits;
  const uint32_t* block_off;
  const uint8_t* tables;
  const float4* qp;
  const float* rtab;
  const float* roff;
  const uint32_t* probe;
  const float* probe_cent;
  const uint32_t* probe_n;
  uint32_t P;
  uint32_t cand;  // C: the final TopK
  uint32_t kc;    // the shortlist's K (refine: max(refine, cand); else cand)
  uint32_t* out_id;
  float* out_est;
  float* out_nx;
  uint32_t* out_n;
  uint64_t* scanned;
};

SG_DEV uint4 bg_ldg(const uint4* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// The byte g*16 + (j & 15) of a block holds nibble g of slot j (low half for j < 16).
SG_DEV uint32_t bg_nibble(const uint8_t* blk, uint32_t g, uint32_t j) {
  return (blk[g * 16 + (j & 15)] >> (4 * (j >> 4))) & 15u;
}

// Shared memory of one scan CTA, carved from dynamic shared memory.
struct BgSmem {
  uint64_t* ekey;   // [2C] entries of the final TopK: (ord(est) << 32) | ~admission
  uint32_t* eid;    // [2C]
  float* enx;       // [2C]
  uint32_t* gate;   // [2 kc] shortlist ords (refine only)
  float* rtab;      // [16 * 256] (refine only)
  float* sest;      // [2048] estimates of the step's slots
  uint32_t* sslot;  // [2048] global slot of each (PAD: 0xFFFFFFFF)
};

// Keeps the C best entries (by key) of the n in E, stably compacted to the front.
SG_DEV uint32_t bg_compact_entries(BgSmem& s, uint32_t n, uint32_t C, uint32_t* hist,
                                   uint32_t* tmp) {
  const uint64_t T = block_select_nth_u64([&](uint32_t i) { return s.ekey[i]; }, n, C, hist, tmp);
  uint32_t written = 0;
  for (uint32_t b = 0; b < n; b += blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const bool keep = i < n && s.ekey[i] >= T;
    uint64_t k = 0;
    uint32_t id = 0;
    float nx = 0.0f;
    if (keep) {
      k = s.ekey[i];
      id = s.eid[i];
      nx = s.enx[i];
    }
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan(keep ? 1u : 0u, tmp, &tot);
    if (keep) {
      s.ekey[written + ex] = k;
      s.eid[written + ex] = id;
      s.enx[written + ex] = nx;
    }
    written += tot;
    __syncthreads();
  }
  return written;
}

// Keeps K of the n shortlist ords: every one above the K-th largest and enough equal to it.
// Returns the K-th largest (the new threshold's ord).
SG_DEV uint32_t bg_compact_gate(uint32_t* g, uint32_t n, uint32_t K, uint32_t* hist, uint32_t* tmp) {
  const uint32_t T = block_select_nth_u32([&](uint32_t i) { return g[i]; }, n, K, hist);
  uint32_t gt = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) gt += g[i] > T;
  const uint32_t need = K - block_sum(gt, tmp);
  uint32_t written = 0, eq_seen = 0;
  for (uint32_t b = 0; b < n; b += blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t o = i < n ? g[i] : 0u;
    const bool eq = i < n && o == T;
    uint32_t teq;
    const uint32_t eq_ex = block_exclusive_scan(eq ? 1u : 0u, tmp, &teq);
    const bool keep = i < n && (o > T || (eq && eq_seen + eq_ex < need));
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan(keep ? 1u : 0u, tmp, &tot);
    if (keep) g[written + ex] = o;
    written += tot;
    eq_seen += teq;
    __syncthreads();
  }
  return T;
}

// The refined estimate of slot gs (block gs/32, position gs%32): Refiner::estimate over the
// slot's sign code and bit planes (src/bigann.rs:592-601), then 2 (cent + est) - |x|^2.
SG_DEV float bg_refined(const BgScanArgs& a, const float* rtab, float roff, float cent, uint32_t gs,
                        float nx) {
  const uint32_t blk = gs / SG_BLOCK, j = gs % SG_BLOCK;
  const uint8_t* bp = a.blocks + (size_t)blk * BBB;
  const uint8_t* ex8 = a.ext + (size_t)gs * a.extra;
  float ps = -0.0f;
  for (int k = 0; k < BCODE; k++) {
    const uint32_t byte = bg_nibble(bp, 2 * k, j) | (bg_nibble(bp, 2 * k + 1, j) << 4);
    ps = __fadd_rn(ps, rtab[k * 256 + byte]);
  }
  float u = __fmul_rn((float)(1u << (a.bits - 1)), ps);
  for (uint32_t pl = 0; pl + 1 < a.bits; pl++) {
    float pv = -0.0f;
    for (int k = 0; k < BCODE; k++) pv = __fadd_rn(pv, rtab[k * 256 + ex8[pl * BCODE + k]]);
    u = __fadd_rn(u, __fmul_rn((float)(1u << pl), pv));
  }
  const float fs = *reinterpret_cast<const float*>(ex8 + a.extra - 4);
  return __fsub_rn(__fmul_rn(2.0f, __fadd_rn(cent, __fmul_rn(fs, __fsub_rn(u, roff)))), nx);
}

template <bool REFINE>
__global__ void __launch_bounds__(256) k_bg_scan(BgScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint4 s_tab[BGR];
  __shared__ uint32_t hist[256], tmp[32];
  __shared__ uint32_t s_nE, s_nG, s_ninfo, s_stop, s_hasG;
  __shared__ float s_thG;
  const uint32_t q = blockIdx.x, tid = threadIdx.x;
  const uint32_t C = a.cand, KC = a.kc;
  BgSmem s;
  {
    unsigned char* p = smem_raw;
    s.ekey = reinterpret_cast<uint64_t*>(p);
    p += (size_t)2 * C * 8;
    s.eid = reinterpret_cast<uint32_t*>(p);
    p += (size_t)2 * C * 4;
    s.enx = reinterpret_cast<float*>(p);
    p += (size_t)2 * C * 4;
    s.sest = reinterpret_cast<float*>(p);
    p += kBgStepBlocks * SG_BLOCK * 4;
    s.sslot = reinterpret_cast<uint32_t*>(p);
    p += kBgStepBlocks * SG_BLOCK * 4;
    s.rtab = reinterpret_cast<float*>(p);
    if (REFINE) p += BCODE * 256 * 4;
    s.gate = reinterpret_cast<uint32_t*>(p);
  }
  if (C == 0) {
    if (tid == 0) {
      a.out_n[q] = 0;
      a.scanned[q] = 0;
    }
    return;
  }
  if (tid < BGR) s_tab[tid] = reinterpret_cast<const uint4*>(a.tables + (size_t)q * BGR * 16)[tid];
  if (REFINE)
    for (uint32_t e = tid; e < BCODE * 256; e += blockDim.x) s.rtab[e] = a.rtab[(size_t)q * BCODE * 256 + e];
  if (tid == 0) {
    s_nE = s_nG = s_ninfo = 0;
    s_hasG = 0;
    s_thG = 0.0f;
  }
  __syncthreads();
  const float4 qp = a.qp[q];
  const float roff = REFINE ? a.roff[q] : 0.0f;
  const uint32_t np = a.probe_n[q];
  uint64_t scanned = 0;
  // The gate is the TopK whose threshold decides admission: the shortlist (refine) or the final
  // TopK itself; capG = 2 x its K. E, the final TopK, holds 2C entries before it compacts.
  const uint32_t capG = REFINE ? 2 * KC : 2 * C;
  const uint32_t capE = 2 * C;
  const int t4 = tid & 3, lb = tid >> 2;
  for (uint32_t r = 0; r < np; r++) {
    const uint32_t c = a.probe[(size_t)q * a.P + r];
    const float cent = a.probe_cent[(size_t)q * a.P + r];
    const uint32_t b0 = a.block_off[c], b1 = a.block_off[c + 1];
    scanned += (uint64_t)(b1 - b0) * SG_BLOCK;
    for (uint32_t pb = b0; pb < b1; pb += kBgStepBlocks) {
      const uint32_t nbk = min(kBgStepBlocks, b1 - pb);
      const uint32_t nslot = nbk * SG_BLOCK;
      // ---- score: four threads per block, eight groups each (all lanes join the shuffles) ----
      {
        const bool have = (uint32_t)lb < nbk;
        const uint32_t blk = pb + (have ? lb : 0);
        const uint4* src = reinterpret_cast<const uint4*>(a.blocks + (size_t)blk * BBB);
        uint32_t acc[16];
#pragma unroll
        for (int e = 0; e < 16; e++) acc[e] = 0;
        if (have) {
#pragma unroll
          for (int i = 0; i < BGR / 4; i++) {
            const int g = 4 * i + t4;
            const uint4 code = bg_ldg(src + g);
            const uint4 tb = s_tab[g];
            lut_word(code.x, tb, acc + 0);
            lut_word(code.y, tb, acc + 4);
            lut_word(code.z, tb, acc + 8);
            lut_word(code.w, tb, acc + 12);
          }
        }
#pragma unroll
        for (int e = 0; e < 16; e++) {
          acc[e] += __shfl_xor_sync(0xFFFFFFFFu, acc[e], 1);
          acc[e] += __shfl_xor_sync(0xFFFFFFFFu, acc[e], 2);
        }
        if (have) {
          uint32_t x0 = acc[0], x1 = acc[1], x2 = acc[2], x3 = acc[3];
          if (t4 == 1) {
            x0 = acc[4]; x1 = acc[5]; x2 = acc[6]; x3 = acc[7];
          } else if (t4 == 2) {
            x0 = acc[8]; x1 = acc[9]; x2 = acc[10]; x3 = acc[11];
          } else if (t4 == 3) {
            x0 = acc[12]; x1 = acc[13]; x2 = acc[14]; x3 = acc[15];
          }
          const uint32_t sc[8] = {x0 & 0xFFFFu, x0 >> 16, x2 & 0xFFFFu, x2 >> 16,
                                  x1 & 0xFFFFu, x1 >> 16, x3 & 0xFFFFu, x3 >> 16};
#pragma unroll
          for (int d = 0; d < 8; d++) {
            const uint32_t doc = d < 4 ? 4 * t4 + d : 16 + 4 * t4 + (d - 4);
            const uint32_t gs = blk * SG_BLOCK + doc;
            const uint32_t id = a.ids[gs];
            const float2 fm = a.factors[gs];
            const float est = __fsub_rn(
                __fmul_rn(2.0f, __fadd_rn(cent, __fmul_rn(fm.x, __fadd_rn(__fmul_rn(qp.z, (float)sc[d]), qp.w)))),
                fm.y);
            s.sest[lb * SG_BLOCK + doc] = est;
            s.sslot[lb * SG_BLOCK + doc] = id == SG_PAD ? 0xFFFFFFFFu : gs;
          }
        }
      }
      __syncthreads();
      // ---- admission in slot order (thread tid owns slots [i0, i1), <= 8 of them) -------------
      const uint32_t per = (nslot + blockDim.x - 1) / blockDim.x;
      const uint32_t i0 = min(nslot, tid * per), i1 = min(nslot, i0 + per);
      uint32_t pos = 0;
      for (;;) {
        const bool hasG = s_hasG != 0;
        const float thG = s_thG;
        const uint32_t nG = s_nG, base_idx = s_ninfo;
        uint32_t mask = 0, cnt = 0;
        for (uint32_t i = max(i0, pos); i < i1; i++) {
          if (s.sslot[i] != 0xFFFFFFFFu && (!hasG || s.sest[i] > thG)) {
            mask |= 1u << (i - i0);
            cnt++;
          }
        }
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(cnt, tmp, &total);
        const uint32_t room = capG - nG;
        const uint32_t take = min(total, room);
        // admitted entries of rank < take; the one of rank room - 1 fills the gate
        uint32_t rank = ex;
        for (uint32_t i = i0; i < i1; i++) {
          if (!(mask & (1u << (i - i0)))) continue;
          if (rank < take) {
            if (REFINE) s.gate[nG + rank] = ord(s.sest[i]);
            if (take == room && rank == room - 1) s_stop = i + 1;
          }
          rank++;
        }
        // E receives the same admissions (refine: their refined estimates), in pieces that fit
        for (uint32_t done = 0; done < take;) {
          const uint32_t nE = s_nE;
          const uint32_t piece = min(take - done, capE - nE);
          uint32_t rk = ex;
          for (uint32_t i = i0; i < i1; i++) {
            if (!(mask & (1u << (i - i0)))) continue;
            if (rk >= done && rk < done + piece) {
              const uint32_t gs = s.sslot[i];
              const float nx = a.factors[gs].y;
              const float e = REFINE ? bg_refined(a, s.rtab, roff, cent, gs, nx) : s.sest[i];
              const uint32_t w = nE + rk - done;
              s.ekey[w] = ((uint64_t)ord(e) << 32) | (uint64_t)(0xFFFFFFFFu - (base_idx + rk));
              s.eid[w] = a.ids[gs];
              s.enx[w] = nx;
            }
            rk++;
          }
          __syncthreads();
          uint32_t nE2 = nE + piece;
          if (nE2 == capE) nE2 = bg_compact_entries(s, capE, C, hist, tmp);
          if (tid == 0) s_nE = nE2;
          __syncthreads();
          done += piece;
        }
        const bool full = take == room;
        if (full) {
          float th;
          if (REFINE) {
            th = unord(bg_compact_gate(s.gate, capG, KC, hist, tmp));
          } else {
            // E (= the gate) compacted above: its threshold is the smallest kept estimate
            uint32_t lo = 0xFFFFFFFFu;
            for (uint32_t i = tid; i < C; i += blockDim.x) lo = min(lo, (uint32_t)(s.ekey[i] >> 32));
            th = unord(block_reduce_min(lo, tmp));
          }
          if (tid == 0) {
            s_thG = th;
            s_hasG = 1;
          }
        }
        if (tid == 0) {
          s_ninfo = base_idx + take;
          s_nG = full ? (REFINE ? KC : C) : nG + take;
        }
        __syncthreads();
        if (!full) break;
        pos = s_stop;
      }
      __syncthreads();
    }
  }
  // ---- into_sorted: the best C of E by (estimate desc, admission asc) ----------------------------
  uint32_t n = s_nE;
  if (n > C) n = bg_compact_entries(s, n, C, hist, tmp);
  __syncthreads();
  constexpr uint32_t kSortCap = kBgStepBlocks * SG_BLOCK / 2;  // keys that fit in sest (8 KB)
  uint64_t* keys = reinterpret_cast<uint64_t*>(s.sest);
  uint32_t* perm = s.sslot;
  if (n <= kSortCap) {
    const uint32_t n2 = next_pow2(n > 0 ? n : 1);
    for (uint32_t i = tid; i < n2; i += blockDim.x) {
      keys[i] = i < n ? s.ekey[i] : 0ull;
      perm[i] = i;
    }
    __syncthreads();
    block_bitonic_sort_desc_kv(keys, perm, n2);
    for (uint32_t i = tid; i < n; i += blockDim.x) {
      const uint32_t src = perm[i];
      const size_t o = (size_t)q * C + i;
      a.out_id[o] = s.eid[src];
      a.out_est[o] = key_score(s.ekey[src]);
      a.out_nx[o] = s.enx[src];
    }
  } else {
    // larger C: each entry's place is the number of keys above it (keys are distinct)
    for (uint32_t i = tid; i < n; i += blockDim.x) {
      const uint64_t k = s.ekey[i];
      uint32_t rnk = 0;
      for (uint32_t j = 0; j < n; j++) rnk += s.ekey[j] > k;
      const size_t o = (size_t)q * C + rnk;
      a.out_id[o] = s.eid[i];
      a.out_est[o] = key_score(k);
      a.out_nx[o] = s.enx[i];
    }
  }
  if (tid == 0) {
    a.out_n[q] = n;
    a.scanned[q] = scanned;
  }
}

// ---- rerank: exact 2 <q, x> - |x|^2 of every candidate -----------------------------------------
// One warp per candidate: lanes 0..24 take one 4-byte word of the 100-byte rows each (dp4a).
__global__ void __launch_bounds__(256) k_bg_rerank(const int8_t* __restrict__ base,
                                                   const int8_t* __restrict__ qin,
                                                   const uint32_t* __restrict__ cid,
                                                   const float* __restrict__ cnx,
                                                   const uint32_t* __restrict__ cn, uint32_t C,
                                                   float* __restrict__ lsc) {
  const uint32_t q = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t j = blockIdx.x * 8 + warp;
  if (j >= cn[q]) return;
  const uint32_t id = cid[(size_t)q * C + j];
  int s = 0;
  if (lane < BD / 4) {
    const int a = *reinterpret_cast<const int*>(qin + (size_t)q * BD + 4 * lane);
    const int b = *reinterpret_cast<const int*>(base + (size_t)id * BD + 4 * lane);
    s = __dp4a(a, b, 0);
  }
  s = warp_sum_i(s);
  if (lane == 0)
    lsc[(size_t)q * C + j] = __fsub_rn(__fmul_rn(2.0f, (float)s), cnx[(size_t)q * C + j]);
}

}  // namespace sg

// ================================================================================================
// Host side: the index in HBM, per-call scratch, and the C ABI.
// ================================================================================================
namespace {

using sg::fail;

#define BG_CK(call)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(SG_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int bg_alloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(SG_ERR_OOM, "cudaMalloc " + std::to_string(n * sizeof(T)) + " B: " + cudaGetErrorString(e));
  }
  return SG_OK;
}

template <typename T>
void bg_free(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

template <typename T>
int bg_grow(T** p, uint64_t* cap, uint64_t want) {
  if (want <= *cap && *p) return SG_OK;
  bg_free(*p);
  *cap = 0;
  int rc = bg_alloc(p, want);
  if (!rc) *cap = want;
  return rc;
}

struct BgWork {
  uint64_t nq_cap = 0, scores_cap = 0, probe_cap = 0, cand_cap = 0, k_cap = 0;
  int8_t* q = nullptr;
  uint8_t* tables = nullptr;
  float4* qp = nullptr;
  float* qq = nullptr;
  float* rtab = nullptr;
  float* roff = nullptr;
  float* scores = nullptr;
  uint32_t* probe = nullptr;
  float* probe_cent = nullptr;
  uint32_t* probe_n = nullptr;
  uint64_t* scanned = nullptr;
  uint32_t* cid = nullptr;
  float* cest = nullptr;
  float* cnx = nullptr;
  uint32_t* cn = nullptr;
  float* lsc = nullptr;
  float* out_sc = nullptr;
  uint32_t* out_id = nullptr;
  uint32_t* out_n = nullptr;
  // tcgen05 routing
  uint64_t tc_nq_cap = 0, sub_cap = 0, ent_cap = 0;
  __nv_bfloat16* qhl = nullptr;
  float* lim = nullptr;
  uint32_t* cnt = nullptr;
  float* sub_scores = nullptr;
  uint2* ent = nullptr;
  uint32_t* status = nullptr;
  cudaEvent_t ev[4] = {};
  bool events = false;
};

}  // namespace

struct sg_bigann {
  int device = 0;
  uint32_t k = 0, bits = 1, extra = 0;
  uint64_t n = 0, nblocks = 0;
  float* leaves = nullptr;    // [k*100]
  float* leaves_t = nullptr;  // [100*k]
  float* leaf_norm = nullptr;
  __nv_bfloat16* hl = nullptr;  // [k x 208] bf16 hi/lo rows of the leaves (tcgen05 routing)
  float cmax = 0.0f, cmax2 = 0.0f;
  bool route_tc = false;        // the tcgen05 routing is available
  uint64_t route_exact_fallbacks = 0;  // passes in which a query fell back to exact FP32 routing
  uint32_t* block_off = nullptr;
  uint8_t* blocks = nullptr;
  float2* factors = nullptr;
  uint32_t* ids = nullptr;
  uint8_t* ext = nullptr;
  float* rot = nullptr;
  float rot_norm = 0.0f;
  int8_t* base = nullptr;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  BgWork w;
  int sms = 148;
};

namespace {

void bg_free_all(sg_bigann* h) {
  BgWork& w = h->w;
  bg_free(w.q); bg_free(w.tables); bg_free(w.qp); bg_free(w.qq); bg_free(w.rtab); bg_free(w.roff);
  bg_free(w.scores); bg_free(w.probe); bg_free(w.probe_cent); bg_free(w.probe_n); bg_free(w.scanned);
  bg_free(w.cid); bg_free(w.cest); bg_free(w.cnx); bg_free(w.cn); bg_free(w.lsc);
  bg_free(w.out_sc); bg_free(w.out_id); bg_free(w.out_n);
  bg_free(w.qhl); bg_free(w.lim); bg_free(w.cnt); bg_free(w.sub_scores); bg_free(w.ent); bg_free(w.status);
  if (w.events)
    for (auto& e : w.ev) cudaEventDestroy(e);
  w.events = false;
  bg_free(h->leaves); bg_free(h->leaves_t); bg_free(h->leaf_norm); bg_free(h->hl); bg_free(h->block_off);
  bg_free(h->blocks); bg_free(h->factors); bg_free(h->ids); bg_free(h->ext); bg_free(h->rot);
  bg_free(h->base);
  if (h->stream) cudaStreamDestroy(h->stream);
  h->stream = nullptr;
}

int bg_check_params(const sg_bigann* h, const sg_bigann_params* p) {
  if (!p) return fail(SG_ERR_INVALID, "params is null");
  if (std::min<uint32_t>(p->nprobe, h->k) > sg::kBgMax || p->cand > sg::kBgMax ||
      p->refine > sg::kBgMax || p->k > sg::kBgMax)
    return fail(SG_ERR_INVALID, "nprobe, cand, refine and k must be <= 4096");
  if (!(p->margin == p->margin)) return fail(SG_ERR_INVALID, "margin is NaN");
  return SG_OK;
}

bool bg_uses_tc(const sg_bigann* h, const sg_bigann_params& p) { return h->route_tc && !p.route_fp32; }

// Queries per pass: the routing scratch of a pass stays under 1 GiB: [nq x k] f32 scores on the
// FP32 path; the subset scores and the emitted lists ([nq x ksub] f32 + [nq x cap] 8 B) on the
// tcgen05 path.
uint32_t bg_pass(const sg_bigann* h, uint32_t nq, const sg_bigann_params& p) {
  uint64_t per_query = (uint64_t)std::max<uint32_t>(h->k, 1) * 4;
  if (bg_uses_tc(h, p)) {
    const sg::BgRoutePlan pl = sg::bg_route_plan(h->k, std::min<uint32_t>(p.nprobe, h->k));
    per_query = (pl.subset ? (uint64_t)pl.ksub * 4 : 0) + (uint64_t)pl.cap * 8;
  }
  const uint64_t per = std::max<uint64_t>(1, (1ull << 30) / per_query);
  return (uint32_t)std::min<uint64_t>(nq, std::min<uint64_t>(per, 65535ull));  // grid.y
}

int bg_ensure(sg_bigann* h, uint32_t nq, const sg_bigann_params& p) {
  BgWork& w = h->w;
  int rc;
  const uint32_t P = std::max<uint32_t>(std::min<uint32_t>(p.nprobe, h->k), 1);
  const uint32_t C = std::max<uint32_t>(p.cand, 1), K = std::max<uint32_t>(p.k, 1);
  if (nq > w.nq_cap) {
    bg_free(w.q); bg_free(w.tables); bg_free(w.qp); bg_free(w.qq); bg_free(w.roff);
    bg_free(w.probe_n); bg_free(w.scanned); bg_free(w.cn); bg_free(w.out_n); bg_free(w.rtab);
    w.nq_cap = 0;
    w.scores_cap = w.probe_cap = w.cand_cap = w.k_cap = 0;
    bg_free(w.scores); bg_free(w.probe); bg_free(w.probe_cent); bg_free(w.cid); bg_free(w.cest);
    bg_free(w.cnx); bg_free(w.lsc); bg_free(w.out_sc); bg_free(w.out_id);
    if ((rc = bg_alloc(&w.q, (size_t)nq * SG_BG_DIM)) || (rc = bg_alloc(&w.tables, (size_t)nq * 512)) ||
        (rc = bg_alloc(&w.qp, nq)) || (rc = bg_alloc(&w.qq, nq)) || (rc = bg_alloc(&w.roff, nq)) ||
        (rc = bg_alloc(&w.probe_n, nq)) || (rc = bg_alloc(&w.scanned, nq)) || (rc = bg_alloc(&w.cn, nq)) ||
        (rc = bg_alloc(&w.out_n, nq)) ||
        (rc = bg_alloc(&w.rtab, h->bits > 1 ? (size_t)nq * SG_BG_CODE * 256 : 1)))
      return rc;
    w.nq_cap = nq;
  }
  const uint64_t n = w.nq_cap;
  if (bg_uses_tc(h, p)) {
    const sg::BgRoutePlan pl = sg::bg_route_plan(h->k, std::min<uint32_t>(p.nprobe, h->k));
    if (n > w.tc_nq_cap) {
      bg_free(w.qhl); bg_free(w.lim); bg_free(w.cnt);
      w.tc_nq_cap = 0;
      if ((rc = bg_alloc(&w.qhl, sg::bg_route_tc_hl_elems((uint32_t)n))) || (rc = bg_alloc(&w.lim, n)) ||
          (rc = bg_alloc(&w.cnt, n)))
        return rc;
      w.tc_nq_cap = n;
    }
    if ((rc = bg_grow(&w.sub_scores, &w.sub_cap, pl.subset ? n * pl.ksub : 1)) ||
        (rc = bg_grow(&w.ent, &w.ent_cap, n * pl.cap)))
      return rc;
  } else if ((rc = bg_grow(&w.scores, &w.scores_cap, n * h->k))) {
    return rc;
  }
  if (!w.status && (rc = bg_alloc(&w.status, 1))) return rc;
  if (n * P > w.probe_cap) {
    bg_free(w.probe_cent);
    uint64_t cap = w.probe_cap;
    if ((rc = bg_grow(&w.probe, &cap, n * P)) || (rc = bg_alloc(&w.probe_cent, n * P))) return rc;
    w.probe_cap = n * P;
  }
  if (n * C > w.cand_cap) {
    bg_free(w.cest); bg_free(w.cnx); bg_free(w.lsc);
    uint64_t cap = w.cand_cap;
    if ((rc = bg_grow(&w.cid, &cap, n * C)) || (rc = bg_alloc(&w.cest, n * C)) ||
        (rc = bg_alloc(&w.cnx, n * C)) || (rc = bg_alloc(&w.lsc, n * C)))
      return rc;
    w.cand_cap = n * C;
  }
  if (n * K > w.k_cap) {
    bg_free(w.out_id);
    uint64_t cap = w.k_cap;
    if ((rc = bg_grow(&w.out_sc, &cap, n * K)) || (rc = bg_alloc(&w.out_id, n * K))) return rc;
    w.k_cap = n * K;
  }
  if (!w.events) {
    for (auto& e : w.ev) BG_CK(cudaEventCreate(&e));
    w.events = true;
  }
  return SG_OK;
}

size_t bg_scan_smem(uint32_t C, uint32_t KC, bool refine) {
  size_t b = (size_t)2 * C * 16 + (size_t)sg::kBgStepBlocks * SG_BLOCK * 8;
  if (refine) b += (size_t)SG_BG_CODE * 256 * 4 + (size_t)2 * KC * 4;
  return b;
}

enum BgStage { kBgRoute = 1, kBgCandidates = 2, kBgSearch = 3 };

// The stages on the queries in w.q (nq of them); times route / scan / rerank when `timed`.
int bg_run(sg_bigann* h, uint32_t nq, const sg_bigann_params& p, BgStage stage, bool timed,
           uint32_t* launches) {
  BgWork& w = h->w;
  cudaStream_t st = h->stream;
  const uint32_t P = std::min<uint32_t>(p.nprobe, h->k);
  const bool refine = h->bits > 1 && p.refine > 0;
  const uint32_t KC = refine ? std::max(p.refine, p.cand) : p.cand;
  uint32_t L = 0;
  BG_CK(cudaMemsetAsync(w.status, 0, sizeof(uint32_t), st));
  if (timed) BG_CK(cudaEventRecord(w.ev[0], st));
  sg::k_bg_prep<<<nq, 128, 0, st>>>(w.q, h->rot, h->rot_norm, h->bits, refine ? 1 : 0, w.tables,
                                    w.qp, w.qq, w.rtab, w.roff);
  static sg::PerDeviceOnce attr;
  const cudaError_t smem_limits = attr([] {
    cudaError_t e = cudaFuncSetAttribute(sg::k_bg_select, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sg::kBgMax * 8));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(sg::k_bg_scan<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bg_scan_smem(sg::kBgMax, sg::kBgMax, true));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(sg::k_bg_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bg_scan_smem(sg::kBgMax, sg::kBgMax, false));
    return e;
  });
  BG_CK(smem_limits);
  if (bg_uses_tc(h, p)) {
    sg::BgRouteTc r;
    r.K = h->k;
    r.P = P;
    r.nq = nq;
    r.sms = h->sms;
    r.margin = p.margin;
    r.cmax = h->cmax;
    r.cmax2 = h->cmax2;
    r.q = w.q;
    r.qhl = w.qhl;
    r.hl = h->hl;
    r.leaves = h->leaves;
    r.ln = h->leaf_norm;
    r.qq = w.qq;
    r.sub_scores = w.sub_scores;
    r.lim = w.lim;
    r.ent = w.ent;
    r.cnt = w.cnt;
    r.probe = w.probe;
    r.probe_cent = w.probe_cent;
    r.probe_n = w.probe_n;
    r.status = w.status;
    BG_CK(sg::launch_bg_route_tc(r, st));
    L += 1 + (sg::bg_route_plan(h->k, P).subset ? 5 : 4);
  } else {
    dim3 g1((h->k + 255) / 256, (nq + sg::kBgRouteQ - 1) / sg::kBgRouteQ);
    sg::k_bg_scores<<<g1, 256, 0, st>>>(w.q, nq, h->leaves_t, h->leaf_norm, h->k, w.scores);
    const size_t sel_smem = (size_t)sg::next_pow2_host(std::max<uint32_t>(P, 1)) * 8;
    sg::k_bg_select<<<nq, 1024, sel_smem, st>>>(w.scores, h->k, P, p.margin, w.qq, w.q, h->leaves,
                                                w.probe, w.probe_cent, w.probe_n);
    L += 3;
  }
  if (timed) BG_CK(cudaEventRecord(w.ev[1], st));
  if (stage >= kBgCandidates) {
    sg::BgScanArgs a;
    a.blocks = h->blocks;
    a.factors = h->factors;
    a.ids = h->ids;
    a.ext = h->ext;
    a.extra = h->extra;
    a.bits = h->bits;
    a.block_off = h->block_off;
    a.tables = w.tables;
    a.qp = w.qp;
    a.rtab = w.rtab;
    a.roff = w.roff;
    a.probe = w.probe;
    a.probe_cent = w.probe_cent;
    a.probe_n = w.probe_n;
    a.P = std::max<uint32_t>(P, 1);
    a.cand = p.cand;
    a.kc = KC;
    a.out_id = w.cid;
    a.out_est = w.cest;
    a.out_nx = w.cnx;
    a.out_n = w.cn;
    a.scanned = w.scanned;
    const size_t smem = bg_scan_smem(std::max<uint32_t>(p.cand, 1), std::max<uint32_t>(KC, 1), refine);
    if (refine) sg::k_bg_scan<true><<<nq, 256, smem, st>>>(a);
    else sg::k_bg_scan<false><<<nq, 256, smem, st>>>(a);
    L++;
  }
  if (timed) BG_CK(cudaEventRecord(w.ev[2], st));
  if (stage >= kBgSearch) {
    const uint32_t C = std::max<uint32_t>(p.cand, 1);
    dim3 g2((C + 7) / 8, nq);
    sg::k_bg_rerank<<<g2, 256, 0, st>>>(h->base, w.q, w.cid, w.cnx, w.cn, C, w.lsc);
    sg::launch_top_list(w.lsc, w.cid, w.cn, C, C, p.k, w.out_sc, w.out_id, w.out_n,
                        std::max<uint32_t>(p.k, 1), nq, st);
    L += 2;
  }
  if (timed) BG_CK(cudaEventRecord(w.ev[3], st));
  BG_CK(cudaGetLastError());
  *launches = L;
  return SG_OK;
}

int bg_upload_bytes(void* dst, const void* src, size_t n) {
  if (n == 0) return SG_OK;
  BG_CK(cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice));
  return SG_OK;
}

int bg_build(const sg_bigann_arrays* a, int device, sg_bigann** out) {
  if (!a || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  const uint32_t K = a->k;
  if (K == 0 || !a->leaves || !a->block_off || !a->rotation || !a->base)
    return fail(SG_ERR_INVALID, "bigann arrays incomplete");
  if (a->bits < 1 || a->bits > SG_BG_MAX_BITS) return fail(SG_ERR_INVALID, "bits must be 1..3");
  if (a->block_off[0] != 0) return fail(SG_ERR_INVALID, "block_off[0] != 0");
  for (uint32_t c = 0; c < K; c++)
    if (a->block_off[c + 1] < a->block_off[c]) return fail(SG_ERR_INVALID, "block_off not monotonic");
  const uint64_t nb = a->block_off[K];
  if (nb * SG_BLOCK >= 0xFFFFFFFFull) return fail(SG_ERR_INVALID, "more than 2^32 slots");
  if (nb && (!a->ids || !a->blocks || !a->factors)) return fail(SG_ERR_INVALID, "records missing");
  const uint32_t extra = a->bits > 1 ? (a->bits - 1) * SG_BG_CODE + 4 : 0;
  if (extra && nb && !a->ext) return fail(SG_ERR_INVALID, "bits > 1 needs the extra section");
  for (uint64_t s = 0; s < nb * SG_BLOCK; s++)
    if (a->ids[s] != SG_PAD && a->ids[s] >= a->n) return fail(SG_ERR_INVALID, "record id out of range");
  int ndev = 0;
  BG_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(SG_ERR_DEVICE, "no such CUDA device");
  BG_CK(cudaSetDevice(device));
  std::unique_ptr<sg_bigann> h(new sg_bigann());
  h->device = device;
  h->k = K;
  h->bits = a->bits;
  h->extra = extra;
  h->n = a->n;
  h->nblocks = nb;
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
  h->rot_norm = powf((float)SG_BG_PDIM, -1.5f);  // Rotation::apply's d^-1.5 (libm powf)
  std::vector<float> lt((size_t)K * SG_BG_DIM);
  for (uint32_t c = 0; c < K; c++)
    for (int i = 0; i < SG_BG_DIM; i++) lt[(size_t)i * K + c] = a->leaves[(size_t)c * SG_BG_DIM + i];
  std::vector<uint32_t> bo(K + 1);
  for (uint32_t c = 0; c <= K; c++) bo[c] = (uint32_t)a->block_off[c];
  int rc;
  auto bail = [&](int code) {
    bg_free_all(h.get());
    return code;
  };
  if ((rc = bg_alloc(&h->leaves, (size_t)K * SG_BG_DIM)) || (rc = bg_alloc(&h->leaves_t, (size_t)K * SG_BG_DIM)) ||
      (rc = bg_alloc(&h->leaf_norm, K)) || (rc = bg_alloc(&h->block_off, K + 1)) ||
      (rc = bg_alloc(&h->blocks, nb * SG_BG_BLOCK_BYTES)) || (rc = bg_alloc(&h->factors, nb * SG_BLOCK)) ||
      (rc = bg_alloc(&h->ids, nb * SG_BLOCK)) || (rc = bg_alloc(&h->ext, nb * SG_BLOCK * extra)) ||
      (rc = bg_alloc(&h->rot, 3 * SG_BG_PDIM)) || (rc = bg_alloc(&h->base, a->n * SG_BG_DIM)))
    return bail(rc);
  if ((rc = bg_upload_bytes(h->leaves, a->leaves, (size_t)K * SG_BG_DIM * 4)) ||
      (rc = bg_upload_bytes(h->leaves_t, lt.data(), lt.size() * 4)) ||
      (rc = bg_upload_bytes(h->block_off, bo.data(), bo.size() * 4)) ||
      (rc = bg_upload_bytes(h->blocks, a->blocks, nb * SG_BG_BLOCK_BYTES)) ||
      (rc = bg_upload_bytes(h->factors, a->factors, nb * SG_BLOCK * 8)) ||
      (rc = bg_upload_bytes(h->ids, a->ids, nb * SG_BLOCK * 4)) ||
      (rc = bg_upload_bytes(h->ext, a->ext, nb * SG_BLOCK * extra)) ||
      (rc = bg_upload_bytes(h->rot, a->rotation, 3 * SG_BG_PDIM * 4)) ||
      (rc = bg_upload_bytes(h->base, a->base, a->n * SG_BG_DIM)))
    return bail(rc);
  sg::k_bg_leaf_norm<<<(K + 255) / 256, 256>>>(h->leaves, K, h->leaf_norm);
  if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(SG_ERR_DEVICE, "leaf norms"));
  // the tcgen05 routing: the bf16 hi/lo leaf matrix and the largest leaf norm (rounded up)
  {
    double m2 = 0.0;
    for (uint32_t c = 0; c < K; c++) {
      double s2 = 0.0;
      for (int i = 0; i < SG_BG_DIM; i++) {
        const double v = a->leaves[(size_t)c * SG_BG_DIM + i];
        s2 += v * v;
      }
      m2 = std::max(m2, s2);
    }
    h->cmax2 = (float)(m2 * (1.0 + 1e-6)) ;
    h->cmax = (float)(std::sqrt(m2) * (1.0 + 1e-6));
    h->route_tc = sg::route_gemm_ready() && std::isfinite(h->cmax2);
    if (h->route_tc) {
      if ((rc = bg_alloc(&h->hl, sg::bg_route_tc_hl_elems(K)))) return bail(rc);
      if (sg::bg_route_tc_prepare(h->leaves, K, h->hl, 0) || cudaDeviceSynchronize() != cudaSuccess)
        return bail(fail(SG_ERR_DEVICE, "bf16 leaf matrix"));
    }
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(SG_ERR_DEVICE, "stream"));
  *out = h.release();
  return SG_OK;
}

bool bg_read(const std::string& path, std::vector<char>& out, bool optional, int* rc) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    if (!optional) *rc = fail(SG_ERR_IO, "cannot open " + path);
    return false;
  }
  const std::streamsize n = f.tellg();
  f.seekg(0);
  out.resize((size_t)n);
  if (n && !f.read(out.data(), n)) {
    *rc = fail(SG_ERR_IO, "cannot read " + path);
    return false;
  }
  return true;
}

// After a pass has synchronised: a tensor-core wait that ran out fails the call.
int bg_check_status(sg_bigann* h) {
  uint32_t st = 0;
  BG_CK(cudaMemcpy(&st, h->w.status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "bigann routing: a tensor-core pipeline wait timed out");
  if (st & sg::kStatusWindow) h->route_exact_fallbacks++;
  return SG_OK;
}

// Copies results of a pass out and accumulates timing.
int bg_search_impl(sg_bigann* h, uint32_t nq, const int8_t* q, const sg_bigann_params& p,
                   float* out_sc, uint32_t* out_id, uint32_t* out_n, sg_bigann_timing* t,
                   bool device) {
  int rc;
  if ((rc = bg_check_params(h, &p))) return rc;
  if (nq == 0) return SG_OK;
  if (!q) return fail(SG_ERR_INVALID, "q is null");
  BG_CK(cudaSetDevice(h->device));
  const uint32_t per = bg_pass(h, nq, p);
  if ((rc = bg_ensure(h, per, p))) return rc;
  BgWork& w = h->w;
  const uint32_t K = p.k;
  const cudaMemcpyKind ik = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind ok = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  std::vector<uint64_t> scanned(per);
  std::vector<uint32_t> probes(per);
  for (uint32_t q0 = 0; q0 < nq; q0 += per) {
    const uint32_t m = std::min(per, nq - q0);
    BG_CK(cudaMemcpyAsync(w.q, q + (size_t)q0 * SG_BG_DIM, (size_t)m * SG_BG_DIM, ik, h->stream));
    uint32_t launches = 0;
    if ((rc = bg_run(h, m, p, kBgSearch, t != nullptr, &launches))) return rc;
    if (K) {
      BG_CK(cudaMemcpyAsync(out_sc + (size_t)q0 * K, w.out_sc, (size_t)m * K * 4, ok, h->stream));
      BG_CK(cudaMemcpyAsync(out_id + (size_t)q0 * K, w.out_id, (size_t)m * K * 4, ok, h->stream));
      BG_CK(cudaMemcpyAsync(out_n + q0, w.out_n, (size_t)m * 4, ok, h->stream));
    } else {
      BG_CK(cudaMemsetAsync(device ? (void*)(out_n + q0) : (void*)w.out_n, 0, (size_t)m * 4, h->stream));
      if (!device) BG_CK(cudaMemcpyAsync(out_n + q0, w.out_n, (size_t)m * 4, ok, h->stream));
    }
    if (t) {
      BG_CK(cudaMemcpyAsync(scanned.data(), w.scanned, (size_t)m * 8, cudaMemcpyDeviceToHost, h->stream));
      BG_CK(cudaMemcpyAsync(probes.data(), w.probe_n, (size_t)m * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    BG_CK(cudaStreamSynchronize(h->stream));
    if ((rc = bg_check_status(h))) return rc;
    if (t) {
      float r = 0, s = 0, x = 0;
      BG_CK(cudaEventElapsedTime(&r, w.ev[0], w.ev[1]));
      BG_CK(cudaEventElapsedTime(&s, w.ev[1], w.ev[2]));
      BG_CK(cudaEventElapsedTime(&x, w.ev[2], w.ev[3]));
      t->route += (uint64_t)(r * 1e6);
      t->scan += (uint64_t)(s * 1e6);
      t->rerank += (uint64_t)(x * 1e6);
      for (uint32_t i = 0; i < m; i++) {
        t->scanned += scanned[i];
        t->probes += probes[i];
      }
    }
  }
  return SG_OK;
}

}  // namespace

extern "C" {

int sg_open_bigann_arrays(const sg_bigann_arrays* a, int device, sg_bigann** out) {
  try {
    return bg_build(a, device, out);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, e.what());
  }
}

int sg_open_bigann(const char* index_dir, const char* base_dir, int device, sg_bigann** out) {
  if (!index_dir || !base_dir || !out) return fail(SG_ERR_INVALID, "null argument");
  try {
    const std::string X(index_dir), B(base_dir);
    int rc = SG_OK;
    std::vector<char> leaves, bo, off, rec, rot, bits;
    if (!bg_read(X + "/centroids.f32", leaves, false, &rc) || !bg_read(X + "/block_off.u64", bo, false, &rc) ||
        !bg_read(X + "/postings.off", off, false, &rc) || !bg_read(X + "/postings.bin", rec, false, &rc) ||
        !bg_read(X + "/rotation.f32", rot, false, &rc))
      return rc;
    uint64_t nbits = 1;
    if (bg_read(X + "/bits.u64", bits, true, &rc) && bits.size() >= 8) memcpy(&nbits, bits.data(), 8);
    if (nbits < 1 || nbits > SG_BG_MAX_BITS) return fail(SG_ERR_INVALID, "bits.u64 must be 1..3");
    const uint32_t extra = nbits > 1 ? (uint32_t)(nbits - 1) * SG_BG_CODE + 4 : 0;
    if (leaves.size() % (SG_BG_DIM * 4) || bo.size() % 8 || bo.size() < 16 || off.size() != bo.size())
      return fail(SG_ERR_INVALID, "bigann index file sizes disagree");
    if (rot.size() != 3 * SG_BG_PDIM * 4) return fail(SG_ERR_INVALID, "rotation.f32 is not 128-dim");
    const uint32_t K = (uint32_t)(bo.size() / 8 - 1);
    if (leaves.size() / (SG_BG_DIM * 4) != K) return fail(SG_ERR_INVALID, "centroids.f32 has the wrong leaf count");
    const uint64_t* bo64 = reinterpret_cast<const uint64_t*>(bo.data());
    const uint64_t* off64 = reinterpret_cast<const uint64_t*>(off.data());
    const uint64_t nb = bo64[K];
    std::vector<uint8_t> blocks(nb * SG_BG_BLOCK_BYTES), ext(nb * SG_BLOCK * extra);
    std::vector<float> factors(nb * SG_BLOCK * 2);
    std::vector<uint32_t> ids(nb * SG_BLOCK);
    // de-interleave the records (src/postings.rs:31-34, :57-75)
    for (uint32_t c = 0; c < K; c++) {
      if (bo64[c + 1] < bo64[c]) return fail(SG_ERR_INVALID, "block_off not monotonic");
      const uint64_t b0 = bo64[c], n = bo64[c + 1] - b0;
      const uint64_t bytes = n * (SG_BG_BLOCK_BYTES + SG_BLOCK * 12 + (uint64_t)SG_BLOCK * extra);
      if (off64[c] + bytes > rec.size()) return fail(SG_ERR_INVALID, "postings.bin is short");
      const char* p = rec.data() + off64[c];
      memcpy(blocks.data() + b0 * SG_BG_BLOCK_BYTES, p, n * SG_BG_BLOCK_BYTES);
      p += n * SG_BG_BLOCK_BYTES;
      memcpy(factors.data() + b0 * SG_BLOCK * 2, p, n * SG_BLOCK * 8);
      p += n * SG_BLOCK * 8;
      memcpy(ids.data() + b0 * SG_BLOCK, p, n * SG_BLOCK * 4);
      p += n * SG_BLOCK * 4;
      if (extra) memcpy(ext.data() + b0 * SG_BLOCK * extra, p, n * SG_BLOCK * extra);
    }
    // base.00, base.01, ... while base.NN.done exists (bigann::Base::open, src/bigann.rs:476-487)
    std::vector<int8_t> base;
    for (int c = 0;; c++) {
      char name[32];
      snprintf(name, sizeof name, "/base.%02d", c);
      std::vector<char> done, chunk;
      if (!bg_read(B + name + ".done", done, true, &rc)) break;
      if (!bg_read(B + name, chunk, false, &rc)) return rc;
      base.insert(base.end(), chunk.begin(), chunk.end());
    }
    if (base.empty()) return fail(SG_ERR_IO, "no base.NN chunks in " + B);
    sg_bigann_arrays a;
    memset(&a, 0, sizeof a);
    a.n = base.size() / SG_BG_DIM;
    a.k = K;
    a.bits = (uint32_t)nbits;
    a.leaves = reinterpret_cast<const float*>(leaves.data());
    a.block_off = bo64;
    a.ids = ids.data();
    a.blocks = blocks.data();
    a.factors = factors.data();
    a.ext = extra ? ext.data() : nullptr;
    a.rotation = reinterpret_cast<const float*>(rot.data());
    a.base = base.data();
    return bg_build(&a, device, out);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, e.what());
  }
}

int sg_close_bigann(sg_bigann* h) {
  if (!h) return SG_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  bg_free_all(h);
  delete h;
  return SG_OK;
}

int sg_bigann_info(const sg_bigann* h, uint32_t* k, uint64_t* n, uint64_t* nblocks, uint32_t* bits) {
  if (!h) return fail(SG_ERR_INVALID, "null index");
  if (k) *k = h->k;
  if (n) *n = h->n;
  if (nblocks) *nblocks = h->nblocks;
  if (bits) *bits = h->bits;
  return SG_OK;
}

int sg_bigann_route_fallbacks(const sg_bigann* h, uint64_t* passes) {
  if (!h || !passes) return fail(SG_ERR_INVALID, "null argument");
  *passes = h->route_exact_fallbacks;
  return SG_OK;
}

int sg_search_bigann(sg_bigann* h, uint32_t nq, const int8_t* q100, const sg_bigann_params* params,
                     float* out_scores, uint32_t* out_ids, uint32_t* out_counts,
                     sg_bigann_timing* timing) {
  if (!h || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  try {
    return bg_search_impl(h, nq, q100, *params, out_scores, out_ids, out_counts, timing, false);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, e.what());
  }
}

int sg_search_bigann_device(sg_bigann* h, uint32_t nq, const int8_t* d_q100,
                            const sg_bigann_params* params, float* d_out_scores,
                            uint32_t* d_out_ids, uint32_t* d_out_counts, void* stream) {
  if (!h || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  cudaEvent_t ev;
  BG_CK(cudaSetDevice(h->device));
  BG_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  BG_CK(cudaEventRecord(ev, (cudaStream_t)stream));
  BG_CK(cudaStreamWaitEvent(h->stream, ev, 0));
  int rc = bg_search_impl(h, nq, d_q100, *params, d_out_scores, d_out_ids, d_out_counts, nullptr, true);
  cudaEventDestroy(ev);
  return rc;
}

int sg_bigann_route(sg_bigann* h, uint32_t nq, const int8_t* q100, const sg_bigann_params* params,
                    uint32_t* out_probe, uint32_t* out_counts) {
  if (!h || !params || !q100) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  int rc;
  if ((rc = bg_check_params(h, params))) return rc;
  if (nq == 0) return SG_OK;
  BG_CK(cudaSetDevice(h->device));
  const uint32_t per = bg_pass(h, nq, *params);
  if ((rc = bg_ensure(h, per, *params))) return rc;
  BgWork& w = h->w;
  const uint32_t P = std::min<uint32_t>(params->nprobe, h->k);
  for (uint32_t q0 = 0; q0 < nq; q0 += per) {
    const uint32_t m = std::min(per, nq - q0);
    BG_CK(cudaMemcpyAsync(w.q, q100 + (size_t)q0 * SG_BG_DIM, (size_t)m * SG_BG_DIM, cudaMemcpyHostToDevice, h->stream));
    uint32_t L;
    if ((rc = bg_run(h, m, *params, kBgRoute, false, &L))) return rc;
    if (P) BG_CK(cudaMemcpyAsync(out_probe + (size_t)q0 * P, w.probe, (size_t)m * P * 4, cudaMemcpyDeviceToHost, h->stream));
    BG_CK(cudaMemcpyAsync(out_counts + q0, w.probe_n, (size_t)m * 4, cudaMemcpyDeviceToHost, h->stream));
    BG_CK(cudaStreamSynchronize(h->stream));
    if ((rc = bg_check_status(h))) return rc;
  }
  return SG_OK;
}

int sg_bigann_candidates(sg_bigann* h, uint32_t nq, const int8_t* q100, const sg_bigann_params* params,
                         uint32_t* out_ids, float* out_est, float* out_nx, uint32_t* out_counts) {
  if (!h || !params || !q100) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  int rc;
  if ((rc = bg_check_params(h, params))) return rc;
  if (nq == 0) return SG_OK;
  BG_CK(cudaSetDevice(h->device));
  const uint32_t per = bg_pass(h, nq, *params);
  if ((rc = bg_ensure(h, per, *params))) return rc;
  BgWork& w = h->w;
  const uint32_t C = params->cand;
  for (uint32_t q0 = 0; q0 < nq; q0 += per) {
    const uint32_t m = std::min(per, nq - q0);
    BG_CK(cudaMemcpyAsync(w.q, q100 + (size_t)q0 * SG_BG_DIM, (size_t)m * SG_BG_DIM, cudaMemcpyHostToDevice, h->stream));
    uint32_t L;
    if ((rc = bg_run(h, m, *params, kBgCandidates, false, &L))) return rc;
    if (C) {
      BG_CK(cudaMemcpyAsync(out_ids + (size_t)q0 * C, w.cid, (size_t)m * C * 4, cudaMemcpyDeviceToHost, h->stream));
      BG_CK(cudaMemcpyAsync(out_est + (size_t)q0 * C, w.cest, (size_t)m * C * 4, cudaMemcpyDeviceToHost, h->stream));
      BG_CK(cudaMemcpyAsync(out_nx + (size_t)q0 * C, w.cnx, (size_t)m * C * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    BG_CK(cudaMemcpyAsync(out_counts + q0, w.cn, (size_t)m * 4, cudaMemcpyDeviceToHost, h->stream));
    BG_CK(cudaStreamSynchronize(h->stream));
    if ((rc = bg_check_status(h))) return rc;
  }
  return SG_OK;
}

}  // extern "C"
