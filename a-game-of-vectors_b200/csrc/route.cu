// route.cu — centroid routing, ivf::Index::route (src/ivf.rs:589-618).
//
// Two ways to score q256 against the K centroids:
//   FP32: every (query, centroid) dot in the reference's order — a sequential f32 sum from -0.0
//         of rounded products (blas::gemm_abt portable, src/blas.rs:43-54). Exact by construction.
//   BF16: a tcgen05 tensor-core GEMM [nq x 256] x [256 x K] with FP32 accumulation, then, per
//         query, every centroid whose BF16 score lies within 2*delta of the nprobe-th best BF16
//         score is rescored with the FP32 sequential dot. delta bounds |BF16 score - FP32 score|:
//         inputs rounded to bf16 (unit roundoff 2^-8) give a product error <= (2^-7 + 2^-16)|q_i c_i|;
//         FP32 accumulation of 256 exact bf16 products adds <= 256*2^-23 * sum|q_i c_i|, and the
//         reference's own sequential sum differs from the real dot by <= 256*2^-24 * sum|q_i c_i|.
//         With sum|q_i c_i| <= |q||c|, delta = 0.0085 |q| max|c| covers all three. The true top
//         nprobe is inside the window (its members score >= s_np - 2 delta in BF16), so the probe
//         set and its scores equal the FP32 path's bit for bit.
// Then TopK(nprobe) ordering (score desc, id asc), the margin cut v >= best - m, and the slot
// budget (take while the running slot count stays <= b, keep at least one), and the scan work
// items of each probe (chunks of at most chunk_blocks blocks).
#include <cudaTypedefs.h>
#include <float.h>

#include <mutex>

#include "common.cuh"
#include "internal.hpp"
#include "tcgen05.cuh"

namespace sg {

constexpr int kRouteQB = 8;  // queries per thread in the exact kernel

__global__ void __launch_bounds__(256) k_route_fp32(const float* __restrict__ q256,
                                                    const float* __restrict__ cent_t, uint32_t K,
                                                    uint32_t nq, float* __restrict__ scores) {
  __shared__ float qs[kRouteQB][SG_PDIM];
  const uint32_t q0 = blockIdx.y * kRouteQB;
  for (int i = threadIdx.x; i < kRouteQB * SG_PDIM; i += blockDim.x) {
    uint32_t qq = q0 + i / SG_PDIM;
    qs[i / SG_PDIM][i % SG_PDIM] = qq < nq ? q256[(size_t)qq * SG_PDIM + i % SG_PDIM] : 0.0f;
  }
  __syncthreads();
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  float acc[kRouteQB];
#pragma unroll
  for (int j = 0; j < kRouteQB; j++) acc[j] = -0.0f;
#pragma unroll 4
  for (int t = 0; t < SG_PDIM; t++) {
    float cv = __ldg(cent_t + (size_t)t * K + c);
#pragma unroll
    for (int j = 0; j < kRouteQB; j++) acc[j] = __fadd_rn(acc[j], __fmul_rn(qs[j][t], cv));
  }
#pragma unroll
  for (int j = 0; j < kRouteQB; j++)
    if (q0 + j < nq) scores[(size_t)(q0 + j) * K + c] = acc[j];
}

// ---- BF16 GEMM on the tcgen05 tensor cores: 128 centroids x 64 queries per CTA --------------
// D[centroid][query] = sum_k c_bf16[k] * bf16(q[k]) in FP32 tensor memory (M = 128 TMEM lanes,
// N = 64 columns). Both operands come into shared memory by TMA in the 128-byte-swizzled K-major
// layout: one tiled copy per 64-element (128 B) k-block brings that block of all the tile's rows,
// 128 B per row, to kb * rows * 128 B, each row's 16-byte chunks permuted by the row index
// (chunk j of row r at j ^ (r & 7)), 8-row groups 1024 B apart (SBO). The MMA descriptors carry the
// same swizzle mode, and an MMA's K step (16 elements, 32 B) moves the start 32 B within the
// 128-byte row. One elected lane issues the 16 MMAs (K = 16 each). All warps then read the
// accumulators with tcgen05.ld: warp w takes TMEM lanes 32*(w&3).. (the tile's centroids) and
// columns 32*(w>>2).. (queries), and stores each query's 32 centroid scores as one coalesced
// 128 B row segment. Rows past K or nq come in as zeros (the maps' bounds).
constexpr int kRtM = 128, kRtN = 64, kRtThreads = 256;
constexpr uint32_t kRtCols = 64;  // TMEM columns: the f32 accumulators
constexpr int kRtABytes = kRtM * SG_PDIM * 2, kRtBBytes = kRtN * SG_PDIM * 2;
constexpr int kRtSmem = kRtABytes + kRtBBytes;  // 96 KB: two CTAs per SM

SG_DEV uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);  // round to nearest even
  return *reinterpret_cast<uint32_t*>(&p);
}

// q256 -> bf16, 4 values per thread.
__global__ void k_q_bf16(const float4* __restrict__ q, uint32_t n4, uint2* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const float4 v = q[i];
  out[i] = make_uint2(pack_bf16x2(v.x, v.y), pack_bf16x2(v.z, v.w));
}

__global__ void __launch_bounds__(kRtThreads) k_route_tc(const __grid_constant__ CUtensorMap map_c,
                                                         const __grid_constant__ CUtensorMap map_q,
                                                         uint32_t K, uint32_t nq,
                                                         float* __restrict__ scores,
                                                         uint32_t* __restrict__ status) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar_load, bar_done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t m0 = blockIdx.x * kRtM, q0 = blockIdx.y * kRtN;
  if (warp == 0) {
    tc_alloc(&s_tmem, kRtCols);
    tc_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar_load, 1);
    mbar_init(&bar_done, 1);
    s_abort = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (warp == 0) {
    const uint32_t a = smem_addr(smem), b = a + kRtABytes;
    if (lane == 0) {
      mbar_expect_tx(&bar_load, kRtABytes + kRtBBytes);
      for (int kb = 0; kb < SG_PDIM / 64; kb++) {
        tma_load_2d(a + kb * (kRtM * 128), &map_c, 64 * kb, (int32_t)m0, &bar_load);
        tma_load_2d(b + kb * (kRtN * 128), &map_q, 64 * kb, (int32_t)q0, &bar_load);
      }
    }
    __syncwarp();
    if (__all_sync(0xffffffffu, mbar_wait(&bar_load, 0, &s_abort))) {
      tc_fence_after();
      // kind::f16 instruction descriptor: F32 accumulators, BF16 A and B, both K-major
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kRtN >> 3) << 17) |
                             ((uint32_t)(kRtM >> 4) << 24);
      // K step s: k-block s/4 (rows * 128 B further on), then 32 B into its rows
#pragma unroll
      for (uint32_t s = 0; s < SG_PDIM / 16; s++)
        tc_mma_bf16_ss_elect(tmem, smem_desc_sw128(a + (s >> 2) * (kRtM * 128) + (s & 3) * 32),
                             smem_desc_sw128(b + (s >> 2) * (kRtN * 128) + (s & 3) * 32), idesc, s != 0);
      tc_commit_elect(&bar_done);
    }
    __syncwarp();
  }
  const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar_done, 0, &s_abort));
  tc_fence_after();
  if (ok) {
    const uint32_t qd = warp & 3, n0 = 32u * (warp >> 2);
    uint32_t r[32];
    tc_ld32(tmem + ((32u * qd) << 16) + n0, r);
    tc_wait_ld();
    const uint32_t c = m0 + 32 * qd + lane;
    if (c < K) {
#pragma unroll
      for (uint32_t j = 0; j < 32; j++)
        if (q0 + n0 + j < nq) scores[(size_t)(q0 + n0 + j) * K + c] = __uint_as_float(r[j]);
    }
  } else if (lane == 0) {
    atomicOr(status, kStatusTimeout);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tmem, kRtCols);
  }
}

// cuTensorMapEncodeTiled from the driver, looked up once (the library links the CUDA runtime
// statically and has no link-time dependency on the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

bool route_gemm_ready() { return tensor_map_encoder() != nullptr; }

bool encode_bf16_rows(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint64_t row_bytes,
                      uint32_t box_rows, bool sw128) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || rows == 0 || row_bytes % 16 || box_rows == 0 || box_rows > 256) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {row_bytes};
  const cuuint32_t box[2] = {sw128 ? 64u : 8u, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, sw128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A map over a row-major [rows x 256] bf16 matrix (16-byte aligned) whose box is one 128-byte
// k-block (64 elements) of box_rows rows in the 128-byte swizzle; rows past `rows` read as zeros.
static bool encode_rows(CUtensorMap* m, const __nv_bfloat16* base, uint64_t rows, uint32_t box_rows) {
  return encode_bf16_rows(m, base, SG_PDIM, rows, SG_PDIM * sizeof(__nv_bfloat16), box_rows, true);
}

// The reference's sequential FP32 dot of one query with one centroid row.
SG_DEV float exact_dot(const float* __restrict__ q, const float* __restrict__ c) {
  float s = -0.0f;
  const float4* c4 = reinterpret_cast<const float4*>(c);
#pragma unroll 8
  for (int t = 0; t < SG_PDIM / 4; t++) {
    float4 v = __ldg(c4 + t);
    s = __fadd_rn(s, __fmul_rn(q[4 * t + 0], v.x));
    s = __fadd_rn(s, __fmul_rn(q[4 * t + 1], v.y));
    s = __fadd_rn(s, __fmul_rn(q[4 * t + 2], v.z));
    s = __fadd_rn(s, __fmul_rn(q[4 * t + 3], v.w));
  }
  return s;
}

constexpr uint32_t kWinCap = 4096;

struct SelectArgs {
  const float* q256;
  const float* cent;
  const float* qnorm;
  float cent_norm_max;
  const uint32_t* block_off;
  uint32_t K;
  float* scores;
  uint32_t P;        // stride of the probe arrays (probe_stride)
  uint32_t Pb;       // probes routing selects: min(nprobe, K)
  uint32_t live_kc;  // a live index's centroid count (delta list of c = cluster kc + c), else 0
  int bf16;
  sg_params p;
  uint32_t chunk_blocks;
  uint32_t seed_blocks;
  uint32_t alu_ranks;
  uint4* seed_items;
  float* probe_sc;
  uint32_t* probe_cl;
  uint32_t* probe_off;
  uint32_t* probe_n;
  uint64_t* scanned;
  uint4* items;
  uint64_t item_cap;
  uint32_t* counters;
};

// Writes query q's probe list (keys[0..m) sorted best first: probe ranks 0..m-1), the admission
// offset of each probe's first slot, its seed descriptor and its ALU scan items. All threads of
// the block call it.
SG_DEV void emit_probes(const SelectArgs& a, const uint64_t* keys, uint32_t m, uint32_t q,
                        uint32_t* tmp) {
  const uint32_t P = a.P;
  // probe list, admission offsets and chunk counts (block scans over probe ranks)
  uint32_t nloc = (m + blockDim.x - 1) / blockDim.x;  // probes per thread (contiguous)
  uint32_t r0 = threadIdx.x * nloc, r1 = min(m, r0 + nloc);
  // The seed: the first probes, whole clusters while they fit in seed_blocks (at most kMaxSegs),
  // or the first seed_blocks blocks of probe 0 when that cluster alone is larger. It is scanned
  // first, one CTA per query, to set a tight admission threshold; everything else is cut into
  // chunks (or, with alu_ranks off, left to the tensor-core scan).
  __shared__ uint32_t s_rs, s_partial, s_nb[kMaxSegs];
  // the first probes' block counts, read in parallel (thread 0 then walks them)
  for (uint32_t r = threadIdx.x; r < m && r < kMaxSegs; r += blockDim.x) {
    const uint32_t c = key_id(keys[r]);
    s_nb[r] = a.block_off[c + 1] - a.block_off[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t used = 0, rs = 0, partial = 0;
    for (uint32_t r = 0; r < m && r < kMaxSegs; r++) {
      const uint32_t nb = s_nb[r];
      if (r == 0 && nb > a.seed_blocks) {
        rs = 1;
        partial = a.seed_blocks;
        break;
      }
      if (used + nb > a.seed_blocks) break;
      used += nb;
      rs++;
    }
    s_rs = rs;
    s_partial = partial;
    a.seed_items[q] = make_uint4(q, rs, partial, 0);
  }
  __syncthreads();
  const uint32_t rs = s_rs, partial = s_partial;
  auto nchunks = [&](uint32_t r, uint32_t nb) {
    uint32_t rest = r < rs ? (r == 0 && partial ? nb - partial : 0) : (a.alu_ranks ? nb : 0);
    return (rest + a.chunk_blocks - 1) / a.chunk_blocks;
  };
  uint32_t slots = 0, chunks = 0;
  for (uint32_t r = r0; r < r1; r++) {
    uint32_t c = key_id(keys[r]);
    uint32_t nb = a.block_off[c + 1] - a.block_off[c];
    slots += nb * SG_BLOCK;
    chunks += nchunks(r, nb);
  }
  uint32_t tot_slots, tot_chunks;
  uint32_t soff = block_exclusive_scan(slots, tmp, &tot_slots);
  uint32_t coff = block_exclusive_scan(chunks, tmp, &tot_chunks);
  __shared__ uint32_t s_base;
  if (threadIdx.x == 0) {
    uint32_t base = atomicAdd(&a.counters[0], tot_chunks);
    if ((uint64_t)base + tot_chunks > a.item_cap) atomicOr(&a.counters[2], kStatusOverflow);
    s_base = base;
    a.probe_n[q] = m;
    a.scanned[q] = tot_slots;
  }
  __syncthreads();
  uint64_t ibase = (uint64_t)s_base + coff;
  for (uint32_t r = r0; r < r1; r++) {
    uint32_t c = key_id(keys[r]);
    a.probe_cl[(size_t)q * P + r] = c;
    a.probe_sc[(size_t)q * P + r] = key_score(keys[r]);
    a.probe_off[(size_t)q * P + r] = soff;
    uint32_t b0 = a.block_off[c], b1 = a.block_off[c + 1];
    soff += (b1 - b0) * SG_BLOCK;
    if (r < rs) {
      if (!(r == 0 && partial)) continue;
      b0 += partial;  // probe 0's blocks past the seed
    } else if (!a.alu_ranks) {
      continue;
    }
    for (uint32_t b = b0; b < b1; b += a.chunk_blocks) {
      if (ibase < a.item_cap) a.items[ibase] = make_uint4(q, r, b, min(b1, b + a.chunk_blocks));
      ibase++;
    }
  }
}

// A live index: every probe c whose delta list holds slots is followed by cluster kc + c with the
// same centroid score, so the delta list is scanned right after the base list and its slots come
// after the base list's in admission order (src/ivf.rs:679-684). keys[0..m) hold the probes best
// first and have room for 2m; returns the expanded count.
SG_DEV uint32_t expand_delta(const SelectArgs& a, uint64_t* keys, uint32_t m) {
  __shared__ uint32_t s_m2;
  if (threadIdx.x == 0) {
    const uint32_t kc = a.live_kc;
    auto has_delta = [&](uint32_t c) { return a.block_off[kc + c + 1] > a.block_off[kc + c]; };
    uint32_t extra = 0;
    for (uint32_t r = 0; r < m; r++) extra += has_delta(key_id(keys[r]));
    uint32_t pos = m + extra;
    for (int r = (int)m - 1; r >= 0; r--) {  // back to front: an entry only moves to a later place
      const uint64_t k = keys[r];
      const uint32_t c = key_id(k);
      if (has_delta(c)) keys[--pos] = rank_key(key_score(k), kc + c);
      keys[--pos] = k;
    }
    s_m2 = m + extra;
  }
  __syncthreads();
  return s_m2;
}

__global__ void __launch_bounds__(256) k_route_select(SelectArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw);  // [kWinCap]
  __shared__ float qv[SG_PDIM];
  __shared__ uint32_t hist[256], tmp[32];
  __shared__ uint32_t s_nw, s_m, s_keep;
  const uint32_t q = blockIdx.x, P = a.Pb, K = a.K;
  float* row = a.scores + (size_t)q * K;
  for (int i = threadIdx.x; i < SG_PDIM; i += blockDim.x) qv[i] = a.q256[(size_t)q * SG_PDIM + i];
  if (threadIdx.x == 0) s_nw = 0;
  __syncthreads();
  if (P == 0) {
    if (threadIdx.x == 0) {
      a.probe_n[q] = 0;
      a.scanned[q] = 0;
      a.seed_items[q] = make_uint4(q, 0, 0, 0);
    }
    return;
  }
  bool exact = !a.bf16;
  if (a.bf16) {
    // the P-th largest BF16 score and the window below it
    const uint32_t kth = block_select_nth_row(row, K, P, hist);
    const float sP = unord(kth);
    float delta = 0.0085f * a.qnorm[q] * a.cent_norm_max;
    float lim = sP - 2.0f * delta;
    for (uint32_t c0 = threadIdx.x; c0 < K; c0 += 8 * blockDim.x) {
      float v[8];
#pragma unroll
      for (uint32_t j = 0; j < 8; j++) {
        const uint32_t c = c0 + j * blockDim.x;
        v[j] = c < K ? __ldg(row + c) : -INFINITY;
      }
#pragma unroll
      for (uint32_t j = 0; j < 8; j++)
        if (v[j] >= lim && c0 + j * blockDim.x < K) {
          uint32_t slot = atomicAdd(&s_nw, 1u);
          if (slot < kWinCap) keys[slot] = c0 + j * blockDim.x;
        }
    }
    __syncthreads();
    uint32_t nw = s_nw;
    // a window narrower than P means a non-finite score or norm: take the exact path
    if (nw >= P && nw <= kWinCap) {
      for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) {
        uint32_t c = (uint32_t)keys[i];
        keys[i] = rank_key(exact_dot(qv, a.cent + (size_t)c * SG_PDIM), c);
      }
      __syncthreads();
      uint64_t T = block_select_nth_u64([&](uint32_t i) { return keys[i]; }, nw, P, hist, tmp);
      __syncthreads();
      // compact the P winners to the front
      if (threadIdx.x == 0) s_m = 0;
      __syncthreads();
      uint64_t mine[kWinCap / 256];
      uint32_t nm = 0;
      for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x)
        if (keys[i] >= T) mine[nm++] = keys[i];
      __syncthreads();
      for (uint32_t j = 0; j < nm; j++) keys[atomicAdd(&s_m, 1u)] = mine[j];
      __syncthreads();
    } else {
      // window too wide for the buffer (or degenerate): score every centroid exactly
      if (threadIdx.x == 0) atomicOr(&a.counters[2], kStatusWindow);
      for (uint32_t c = threadIdx.x; c < K; c += blockDim.x)
        row[c] = exact_dot(qv, a.cent + (size_t)c * SG_PDIM);
      __syncthreads();
      exact = true;
    }
  }
  if (exact) {
    uint64_t T = block_select_nth_u64([&](uint32_t i) { return rank_key(row[i], i); }, K, P, hist,
                                      tmp);
    if (threadIdx.x == 0) s_m = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < K; c += blockDim.x) {
      uint64_t k = rank_key(row[c], c);
      if (k >= T) keys[atomicAdd(&s_m, 1u)] = k;
    }
    __syncthreads();
  }
  // keys[0..P) hold the winners: sort best first
  uint32_t n2 = next_pow2(P);
  for (uint32_t i = P + threadIdx.x; i < n2; i += blockDim.x) keys[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc(keys, n2);
  // margin (prefix of the sorted list) and budget
  if (threadIdx.x == 0) {
    uint32_t m = P;
    if (a.p.has_margin) {
      float lim = __fsub_rn(key_score(keys[0]), a.p.margin);
      uint32_t w = 0;
      while (w < m && key_score(keys[w]) >= lim) w++;
      m = w;
    }
    if (a.p.has_budget) {
      uint64_t used = 0;
      uint32_t keep = 0;
      for (uint32_t i = 0; i < m; i++) {
        uint32_t c = key_id(keys[i]);
        used += (uint64_t)(a.block_off[c + 1] - a.block_off[c]) * SG_BLOCK;
        if (used <= a.p.budget) keep++;
        else break;
      }
      if (keep < 1) keep = 1;
      if (keep < m) m = keep;
    }
    s_keep = m;
  }
  __syncthreads();
  const uint32_t m = a.live_kc ? expand_delta(a, keys, s_keep) : s_keep;
  emit_probes(a, keys, m, q, tmp);
}

// filter::search with Plan::Expand (src/filter.rs:79-93): every cluster in route order (exact f32
// scores, score desc then cluster asc: the TopK(k) of Index::route with no margin or budget),
// clusters without allowed slots dropped, kept while the allowed slots covered by the clusters
// before it stay below the target (so the cluster that crosses the target is kept). One CTA per
// query sorts the K keys in shared memory (K <= kExpandMaxK).
__global__ void __launch_bounds__(1024) k_route_expand(SelectArgs a,
                                                       const uint32_t* __restrict__ per_cluster,
                                                       uint64_t target) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw);  // [next_pow2(K)]
  __shared__ uint32_t tmp[32], s_n;
  const uint32_t q = blockIdx.x, K = a.K;
  const float* row = a.scores + (size_t)q * K;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < K; c += blockDim.x)
    if (per_cluster[c] > 0) keys[atomicAdd(&s_n, 1u)] = rank_key(row[c], c);
  __syncthreads();
  const uint32_t n = s_n, n2 = next_pow2(n > 0 ? n : 1);
  for (uint32_t i = n + threadIdx.x; i < n2; i += blockDim.x) keys[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc(keys, n2);
  // covered-before of each cluster in sorted order; it only grows, so the kept clusters are the
  // prefix whose covered-before is below the target. (Allowed slots < 2^32: the index has fewer
  // than 2^32 slots.)
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t i0 = min(n, threadIdx.x * per), i1 = min(n, i0 + per);
  uint32_t loc = 0;
  for (uint32_t i = i0; i < i1; i++) loc += per_cluster[key_id(keys[i])];
  uint32_t total;
  uint32_t before = block_exclusive_scan(loc, tmp, &total);
  uint32_t take = 0;
  for (uint32_t i = i0; i < i1; i++) {
    take += (uint64_t)before < target;
    before += per_cluster[key_id(keys[i])];
  }
  const uint32_t m = block_sum(take, tmp);
  emit_probes(a, keys, m, q, tmp);
}

// Index::candidates over a caller's probe list (src/ivf.rs:647-681): query q's probes
// given_cl/given_sc [q * P + r], r < given_n[q], in the given order (their admission order),
// become the probe list, seed and scan items exactly as a routed list would.
__global__ void __launch_bounds__(256) k_route_given(SelectArgs a, const float* __restrict__ given_sc,
                                                     const uint32_t* __restrict__ given_cl,
                                                     const uint32_t* __restrict__ given_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw);  // [P]
  __shared__ uint32_t tmp[32];
  const uint32_t q = blockIdx.x;
  const uint32_t m = min(given_n[q], a.P);
  for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) {
    const uint32_t c = given_cl[(size_t)q * a.P + r];
    keys[r] = rank_key(given_sc[(size_t)q * a.P + r], c < a.K ? c : 0u);
  }
  __syncthreads();
  emit_probes(a, keys, m, q, tmp);
}

cudaError_t launch_route_scores(const DevIndex& ix, Workspace& w, uint32_t nq, int precision,
                                cudaStream_t st) {
  if (nq == 0 || ix.kc == 0) return cudaSuccess;
  if (precision == SG_ROUTE_BF16) {
    static PerDeviceOnce attr;
    attr([] { return cudaFuncSetAttribute(k_route_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kRtSmem); });
    CUtensorMap map_c, map_q;
    if (!encode_rows(&map_c, ix.cent_bf16, ix.kc, kRtM) || !encode_rows(&map_q, w.q16, nq, kRtN))
      return cudaErrorInvalidValue;
    const uint32_t n4 = nq * (SG_PDIM / 4);
    k_q_bf16<<<(n4 + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4*>(w.q256), n4,
                                               reinterpret_cast<uint2*>(w.q16));
    dim3 grid((ix.kc + kRtM - 1) / kRtM, (nq + kRtN - 1) / kRtN);
    k_route_tc<<<grid, kRtThreads, kRtSmem, st>>>(map_c, map_q, ix.kc, nq, w.scores, w.counters + 2);
  } else {
    dim3 grid((ix.kc + 255) / 256, (nq + kRouteQB - 1) / kRouteQB);
    k_route_fp32<<<grid, 256, 0, st>>>(w.q256, ix.cent_t, ix.kc, nq, w.scores);
  }
  return cudaGetLastError();
}

void launch_route_select(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                         int precision, uint32_t chunk_blocks, uint32_t seed_blocks,
                         bool alu_ranks, cudaStream_t st) {
  SelectArgs a;
  a.q256 = w.q256;
  a.cent = ix.cent;
  a.qnorm = w.qnorm;
  a.cent_norm_max = ix.cent_norm_max;
  a.block_off = ix.block_off;
  a.K = ix.kc;
  a.scores = w.scores;
  a.P = probe_stride(ix, p.nprobe);
  a.Pb = p.nprobe < ix.kc ? p.nprobe : ix.kc;
  a.live_kc = ix.live ? ix.kc : 0;
  a.bf16 = precision == SG_ROUTE_BF16;
  a.p = p;
  a.chunk_blocks = chunk_blocks;
  a.seed_blocks = seed_blocks;
  a.alu_ranks = alu_ranks ? 1u : 0u;
  a.seed_items = w.seed_items;
  a.probe_sc = w.probe_sc;
  a.probe_cl = w.probe_cl;
  a.probe_off = w.probe_off;
  a.probe_n = w.probe_n;
  a.scanned = w.scanned;
  a.items = w.items;
  a.item_cap = w.item_cap;
  a.counters = w.counters;
  static PerDeviceOnce attr;
  const size_t smem = kWinCap * sizeof(uint64_t);
  attr([&] {
    return cudaFuncSetAttribute(k_route_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  k_route_select<<<nq, 256, smem, st>>>(a);
}

void launch_route_given(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p, uint32_t chunk_blocks,
                        uint32_t seed_blocks, bool alu_ranks, const float* given_sc, const uint32_t* given_cl,
                        const uint32_t* given_n, cudaStream_t st) {
  SelectArgs a;
  memset(&a, 0, sizeof a);
  a.block_off = ix.block_off;
  a.K = ix.kc;
  a.P = probe_stride(ix, p.nprobe);
  a.Pb = p.nprobe < ix.kc ? p.nprobe : ix.kc;
  a.live_kc = ix.live ? ix.kc : 0;
  a.p = p;
  a.chunk_blocks = chunk_blocks;
  a.seed_blocks = seed_blocks;
  a.alu_ranks = alu_ranks ? 1u : 0u;
  a.seed_items = w.seed_items;
  a.probe_sc = w.probe_sc;
  a.probe_cl = w.probe_cl;
  a.probe_off = w.probe_off;
  a.probe_n = w.probe_n;
  a.scanned = w.scanned;
  a.items = w.items;
  a.item_cap = w.item_cap;
  a.counters = w.counters;
  static PerDeviceOnce attr;
  attr([] {
    return cudaFuncSetAttribute(k_route_given, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(4096 * sizeof(uint64_t)));
  });
  k_route_given<<<nq, 256, (size_t)std::max<uint32_t>(a.P, 1) * sizeof(uint64_t), st>>>(a, given_sc, given_cl,
                                                                                      given_n);
}

void launch_route_expand(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                         uint32_t chunk_blocks, uint32_t seed_blocks,
                         const uint32_t* per_cluster, uint64_t target, cudaStream_t st) {
  SelectArgs a;
  memset(&a, 0, sizeof a);
  a.q256 = w.q256;
  a.cent = ix.cent;
  a.qnorm = w.qnorm;
  a.cent_norm_max = ix.cent_norm_max;
  a.block_off = ix.block_off;
  a.K = ix.kc;
  a.scores = w.scores;
  a.P = ix.kc;
  a.Pb = ix.kc;
  a.bf16 = 0;
  a.p = p;
  a.chunk_blocks = chunk_blocks;
  a.seed_blocks = seed_blocks;
  a.alu_ranks = 1;
  a.seed_items = w.seed_items;
  a.probe_sc = w.probe_sc;
  a.probe_cl = w.probe_cl;
  a.probe_off = w.probe_off;
  a.probe_n = w.probe_n;
  a.scanned = w.scanned;
  a.items = w.items;
  a.item_cap = w.item_cap;
  a.counters = w.counters;
  const size_t smem = (size_t)next_pow2_host(ix.kc) * sizeof(uint64_t);
  static PerDeviceOnce attr;
  attr([] {
    return cudaFuncSetAttribute(k_route_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kExpandMaxK * sizeof(uint64_t)));
  });
  k_route_expand<<<nq, 1024, smem, st>>>(a, per_cluster, target);
}

}  // namespace sg
