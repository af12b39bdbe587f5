// scan.cu — the LUT scan with the RaBitQ estimator and the candidate admission
// (ivf::Index::candidates, src/ivf.rs:647-698; lut::scan, src/lut.rs:96-126;
// rabitq::Query::estimate, src/rabitq.rs:127-130).
//
// Work: a persistent grid drains the (query, probe, chunk) work queue the routing kernel wrote.
// One CTA scores one chunk (<= CHB blocks of 32 slots) of one probed cluster for one query:
//   - the query's 64 u8 nibble tables sit in shared memory (1 KB);
//   - four threads share a block: thread t takes groups t, t+4, ..., t+60, so each warp-wide
//     16-byte load covers 64 contiguous bytes of each of 8 blocks (full 32-byte sectors);
//   - lookups are register PRMTs (lut4), sums are packed u16 pairs (never above 16320);
//   - the four partial sums are combined by shuffles; est = cent + mul*(a*score + b) in f32
//     with the reference's rounding (no FMA).
// Admission is exact. The reference keeps the best `cand` slots by estimate (TopK<f32>,
// src/topk.rs), breaking ties by admission order. Here a chunk keeps its own best `cand`
// eligible slots (est desc, then slot order) at or above the query's running threshold, appends
// them to the query's candidate buffer and raises the threshold to its cand-th estimate (a valid
// lower bound of the final cand-th). The cut kernel then takes the global best `cand` of the buffer.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

struct ScanArgs {
  const uint8_t* blocks;
  const float* mul;
  const uint32_t* ids;
  const uint32_t* block_off;
  const uint32_t* clen;
  const uint8_t* tables;
  const float4* qp;
  const float* probe_sc;
  const uint32_t* probe_cl;
  const uint32_t* probe_off;
  uint32_t P;
  const uint4* items;
  const uint4* seed_items;
  uint64_t item_cap;
  uint32_t* counters;
  uint32_t* thr;
  uint32_t* ccount;
  uint32_t* cbuf_est;
  uint2* cbuf_info;
  uint32_t cap;
  uint8_t* overflow;
  uint32_t cand;
  const uint64_t* allow;
  uint64_t allow_words;
  const uint64_t* const* allow_q;  // per-query allow bitsets (null entries: no filter), or null
  const uint64_t* allow_wq;
  // global sign codes: estimates are the LUT scores (centroid score 0), the admission key is the
  // row (ties by row, src/ivf.rs:700-717), and a chunk keeps every slot tied at its cut
  uint32_t global;
};

SG_DEV uint4 ldg_nc(const uint4* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

SG_DEV uint32_t ld_cg(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Slot i's key lives at word i + i/32 of the key array: one padding word per block, so the
// admission loops (thread t walks its own contiguous range of slots) and the per-block key
// writes of the scoring spread over the shared-memory banks instead of hitting one bank.
constexpr uint32_t kKeyWordsPerBlock = SG_BLOCK + 1;
SG_DEV uint32_t kx(uint32_t i) { return i + (i >> 5); }

// Scores one block's 32 slots into 16 packed accumulators (sum over this thread's 16 groups).
SG_DEV void score_block_quarter(const uint8_t* __restrict__ block, const uint4* s_tab, int t4,
                                uint32_t* acc) {
  const uint4* src = reinterpret_cast<const uint4*>(block);
#pragma unroll
  for (int e = 0; e < 16; e++) acc[e] = 0;
#pragma unroll 4
  for (int i = 0; i < 16; i++) {
    const int g = 4 * i + t4;
    uint4 code = ldg_nc(src + g);
    uint4 tab = s_tab[g];
    lut_word(code.x, tab, acc + 0);
    lut_word(code.y, tab, acc + 4);
    lut_word(code.z, tab, acc + 8);
    lut_word(code.w, tab, acc + 12);
  }
}

// Up to kMaxSegs (probe, block range) segments scored into one key array: a work item is one
// segment; a seed is the query's first probes (whole clusters, or the first blocks of one).
struct Segs {
  uint32_t start[kMaxSegs + 1];  // first block (in the key array) of each segment; [n] = total
  uint32_t b0[kMaxSegs];         // first block of the segment in the index
  int32_t cl[kMaxSegs];          // eligible (non-PAD) slots counted from the segment's first slot
  uint32_t kb[kMaxSegs];         // admission key of the segment's first slot
  float cent[kMaxSegs];          // centroid score of the segment's probe
  uint32_t n;
};

SG_DEV uint32_t seg_of(const Segs& S, uint32_t gb) {
  uint32_t lo = 0, hi = S.n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (S.start[mid] <= gb) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Fills segment `i` for probe r of query q, blocks [b0, b1) of its cluster, starting at key block
// `start`.
SG_DEV void set_seg(const ScanArgs& a, Segs& S, uint32_t i, uint32_t q, uint32_t r, uint32_t b0,
                    uint32_t start) {
  const uint32_t c = a.probe_cl[(size_t)q * a.P + r];
  const uint32_t cb0 = a.block_off[c];
  S.start[i] = start;
  S.b0[i] = b0;
  S.cl[i] = (int32_t)a.clen[c] - (int32_t)((b0 - cb0) * SG_BLOCK);
  S.kb[i] = a.probe_off[(size_t)q * a.P + r] + (b0 - cb0) * SG_BLOCK;
  S.cent[i] = a.global ? 0.0f : a.probe_sc[(size_t)q * a.P + r];
}

// One CTA: score every segment's blocks, then admit the best `cand` eligible slots at or above
// the query's threshold (est desc, then admission order) and raise the threshold to their
// cand-th estimate. Keys (ordered estimates, 0 = not eligible) live in dynamic shared memory.
SG_DEV void scan_segments(const ScanArgs& a, uint32_t q, const Segs& S, uint32_t* s_key,
                          uint4* s_tab, uint32_t* hist, uint32_t* tmp, uint32_t* s_base) {
  const int tid = threadIdx.x, t4 = tid & 3, lbw = tid >> 2;
  const uint32_t NB = S.start[S.n];
  if (NB == 0) return;  // uniform
  const float4 qp = a.qp[q];
  if (tid < SG_GROUPS)
    s_tab[tid] = reinterpret_cast<const uint4*>(a.tables + (size_t)q * SG_GROUPS * 16)[tid];
  __syncthreads();
  // ---- scoring: 64 blocks per pass, four threads per block ----------------------------------
  for (uint32_t pb = 0; pb < NB; pb += 64) {
    const uint32_t gb = pb + lbw;
    uint32_t acc[16];
    uint32_t sg = 0, blk = 0;
    if (gb < NB) {
      sg = seg_of(S, gb);
      blk = S.b0[sg] + (gb - S.start[sg]);
      score_block_quarter(a.blocks + (size_t)blk * SG_BLOCK_BYTES, s_tab, t4, acc);
    } else {
#pragma unroll
      for (int e = 0; e < 16; e++) acc[e] = 0;
    }
#pragma unroll
    for (int e = 0; e < 16; e++) {
      acc[e] += __shfl_xor_sync(0xFFFFFFFFu, acc[e], 1);
      acc[e] += __shfl_xor_sync(0xFFFFFFFFu, acc[e], 2);
    }
    if (gb < NB) {
      uint32_t x0 = acc[0], x1 = acc[1], x2 = acc[2], x3 = acc[3];
      if (t4 == 1) {
        x0 = acc[4]; x1 = acc[5]; x2 = acc[6]; x3 = acc[7];
      } else if (t4 == 2) {
        x0 = acc[8]; x1 = acc[9]; x2 = acc[10]; x3 = acc[11];
      } else if (t4 == 3) {
        x0 = acc[12]; x1 = acc[13]; x2 = acc[14]; x3 = acc[15];
      }
      const float* mrow = a.mul + (size_t)blk * SG_BLOCK;
      const float4 mlo = __ldg(reinterpret_cast<const float4*>(mrow + 4 * t4));
      const float4 mhi = __ldg(reinterpret_cast<const float4*>(mrow + 16 + 4 * t4));
      const uint32_t sc[8] = {x0 & 0xFFFFu, x0 >> 16, x2 & 0xFFFFu, x2 >> 16,
                              x1 & 0xFFFFu, x1 >> 16, x3 & 0xFFFFu, x3 >> 16};
      const float mv[8] = {mlo.x, mlo.y, mlo.z, mlo.w, mhi.x, mhi.y, mhi.z, mhi.w};
      const float cent = S.cent[sg];
      const int32_t rel0 = (int32_t)((gb - S.start[sg]) * SG_BLOCK);
#pragma unroll
      for (int d = 0; d < 8; d++) {
        const uint32_t doc = d < 4 ? 4 * t4 + d : 16 + 4 * t4 + (d - 4);
        const float est =
            __fadd_rn(cent, __fmul_rn(mv[d], __fadd_rn(__fmul_rn(qp.z, (float)sc[d]), qp.w)));
        s_key[gb * kKeyWordsPerBlock + doc] = (rel0 + (int32_t)doc < S.cl[sg]) ? ord(est) : 0u;
      }
    }
  }
  __syncthreads();
  // ---- admission ------------------------------------------------------------------------------
  const uint32_t thr = ld_cg(a.thr + q);
  const uint64_t* al = a.allow_q ? a.allow_q[q] : a.allow;
  const uint64_t aw = a.allow_q ? a.allow_wq[q] : a.allow_words;
  const uint32_t nloc = NB * SG_BLOCK;
  const uint32_t per = (nloc + blockDim.x - 1) / blockDim.x;  // <= 64 slots per thread
  const uint32_t i0 = tid * per, i1 = min(nloc, i0 + per);
  auto slot_of = [&](uint32_t i) {
    const uint32_t gb = i / SG_BLOCK, sg = seg_of(S, gb);
    return (S.b0[sg] + gb - S.start[sg]) * SG_BLOCK + (i % SG_BLOCK);
  };
  uint32_t cnt = 0;
  for (uint32_t i = i0; i < i1; i++) {
    const uint32_t k = s_key[kx(i)];
    bool surv = k != 0u && k >= thr;
    if (surv && al) surv = allowed(al, aw, a.ids[slot_of(i)]);
    if (!surv) s_key[kx(i)] = 0u;
    cnt += surv;
  }
  const uint32_t n_s = block_sum(cnt, tmp);
  if (n_s == 0) return;  // uniform
  const bool cut = n_s > a.cand;
  uint32_t T = 0, need = 0;
  if (cut) {
    T = block_select_nth_u32([&](uint32_t i) { return s_key[kx(i)]; }, nloc, a.cand, hist);
    uint32_t gt = 0;
    for (uint32_t i = i0; i < i1; i++) gt += s_key[kx(i)] > T;
    need = a.cand - block_sum(gt, tmp);
  }
  uint32_t ties = 0;
  if (cut)
    for (uint32_t i = i0; i < i1; i++) ties += s_key[kx(i)] == T;
  uint32_t tr = block_exclusive_scan(ties, tmp, nullptr);
  uint64_t selmask = 0;
  uint32_t nsel = 0;
  for (uint32_t i = i0; i < i1; i++) {
    const uint32_t k = s_key[kx(i)];
    bool sel;
    if (!cut) sel = k != 0u;
    else if (k > T) sel = true;
    else sel = (k == T) && (a.global || tr++ < need);
    if (sel) {
      selmask |= 1ull << (i - i0);
      nsel++;
    }
  }
  uint32_t total;
  uint32_t off = block_exclusive_scan(nsel, tmp, &total);
  if (tid == 0) {
    *s_base = atomicAdd(a.ccount + q, total);
    if (cut) atomicMax(a.thr + q, T);
  }
  __syncthreads();
  const uint32_t base = *s_base;
  const size_t qbase = (size_t)q * a.cap;
  for (uint32_t i = i0; i < i1; i++) {
    if (selmask & (1ull << (i - i0))) {
      const uint32_t pos = base + off++;
      if (pos < a.cap) {
        const uint32_t gb = i / SG_BLOCK, sg = seg_of(S, gb);
        const uint32_t rel = (gb - S.start[sg]) * SG_BLOCK + (i % SG_BLOCK);
        a.cbuf_est[qbase + pos] = __float_as_uint(unord(s_key[kx(i)]));
        const uint32_t slot = S.b0[sg] * SG_BLOCK + rel;
        a.cbuf_info[qbase + pos] = make_uint2(a.global ? a.ids[slot] : S.kb[sg] + rel, slot);
      } else {
        a.overflow[q] = 1;
      }
    }
  }
}

// Seed pass: CTA q scores query q's seed — its first probes, whole clusters while they fit in
// the seed's block budget (or the first blocks of probe 0 when that one cluster is larger) —
// so that its threshold is the cand-th estimate over enough slots to bound the rest tightly.
// seed_items[q] = (q, probes covered, blocks of probe 0 when partial else 0, -).
__global__ void __launch_bounds__(256, 2) k_scan_seed(ScanArgs a) {
  extern __shared__ __align__(16) uint32_t s_key[];
  __shared__ uint4 s_tab[SG_GROUPS];
  __shared__ uint32_t hist[256], tmp[32], s_base;
  __shared__ Segs S;
  const uint4 it = a.seed_items[blockIdx.x];
  const uint32_t q = it.x, rs = it.y, partial = it.z;
  if (threadIdx.x == 0) {
    S.n = rs;
    uint32_t start = 0;
    for (uint32_t r = 0; r < rs; r++) {
      const uint32_t c = a.probe_cl[(size_t)q * a.P + r];
      const uint32_t b0 = a.block_off[c];
      const uint32_t nb = partial ? partial : a.block_off[c + 1] - b0;
      set_seg(a, S, r, q, r, b0, start);
      start += nb;
    }
    S.start[rs] = start;
  }
  __syncthreads();
  scan_segments(a, q, S, s_key, s_tab, hist, tmp, &s_base);
}

// Main pass: a persistent grid drains the (query, probe, chunk) queue.
__global__ void __launch_bounds__(256, 2) k_scan(ScanArgs a) {
  extern __shared__ __align__(16) uint32_t s_key[];
  __shared__ uint4 s_tab[SG_GROUPS];
  __shared__ uint32_t hist[256], tmp[32], s_base, s_item;
  __shared__ Segs S;
  uint32_t nitems = a.counters[0];
  if (nitems > a.item_cap) nitems = (uint32_t)a.item_cap;
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(&a.counters[1], 1u);
      if (s_item < nitems) {
        const uint4 it = a.items[s_item];
        S.n = 1;
        set_seg(a, S, 0, it.x, it.y, it.z, 0);
        S.start[1] = it.w - it.z;
      }
    }
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= nitems) break;
    scan_segments(a, a.items[item].x, S, s_key, s_tab, hist, tmp, &s_base);
    __syncthreads();
  }
}

void launch_scan(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                 const uint64_t* allow, uint64_t allow_words, int sms, uint32_t chunk_blocks,
                 uint32_t seed_blocks, int ctas_per_sm, cudaStream_t st) {
  ScanArgs a;
  a.blocks = ix.blocks;
  a.mul = ix.mul;
  a.ids = ix.ids;
  a.block_off = ix.block_off;
  a.clen = ix.clen;
  a.tables = w.tables;
  a.qp = w.qp;
  a.probe_sc = w.probe_sc;
  a.probe_cl = w.probe_cl;
  a.probe_off = w.probe_off;
  a.P = probe_stride(ix, p.nprobe);
  a.items = w.items;
  a.seed_items = w.seed_items;
  a.item_cap = w.item_cap;
  a.counters = w.counters;
  a.thr = w.thr;
  a.ccount = w.ccount;
  a.cbuf_est = w.cbuf_est;
  a.cbuf_info = w.cbuf_info;
  a.cap = w.cbuf_per_q;
  a.overflow = w.overflow;
  a.cand = p.cand;
  a.allow = allow;
  a.allow_words = allow_words;
  a.allow_q = w.per_query_allow ? w.allow_q : nullptr;
  a.allow_wq = w.allow_wq;
  a.global = ix.global;
  static PerDeviceOnce attr;
  attr([] {
    cudaError_t e = cudaFuncSetAttribute(k_scan_seed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kMaxChunkBlocks * kKeyWordsPerBlock * 4));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_scan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(kMaxChunkBlocks * kKeyWordsPerBlock * 4));
    return e;
  });
  if (seed_blocks) k_scan_seed<<<nq, 256, seed_blocks * kKeyWordsPerBlock * 4, st>>>(a);
  if (chunk_blocks) k_scan<<<sms * ctas_per_sm, 256, chunk_blocks * kKeyWordsPerBlock * 4, st>>>(a);
}

// ---- stateless kernels for the parity tests ---------------------------------------------------
// lut::scan of whole blocks (G = 64 or 32 groups): one thread per block, all groups.
__global__ void k_lut_scan(uint32_t groups, const uint8_t* __restrict__ tables,
                           const uint8_t* __restrict__ blocks, uint64_t nblocks,
                           uint16_t* __restrict__ out) {
  const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const uint4* src = reinterpret_cast<const uint4*>(blocks + b * groups * 16);
  const uint4* tab = reinterpret_cast<const uint4*>(tables);
  uint32_t acc[16];
#pragma unroll
  for (int e = 0; e < 16; e++) acc[e] = 0;
  for (uint32_t g = 0; g < groups; g++) {
    uint4 code = src[g], t = tab[g];
    lut_word(code.x, t, acc + 0);
    lut_word(code.y, t, acc + 4);
    lut_word(code.z, t, acc + 8);
    lut_word(code.w, t, acc + 12);
  }
  uint16_t* o = out + b * SG_BLOCK;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    o[4 * j + 0] = (uint16_t)(acc[4 * j] & 0xFFFF);
    o[4 * j + 1] = (uint16_t)(acc[4 * j] >> 16);
    o[4 * j + 2] = (uint16_t)(acc[4 * j + 2] & 0xFFFF);
    o[4 * j + 3] = (uint16_t)(acc[4 * j + 2] >> 16);
    o[16 + 4 * j + 0] = (uint16_t)(acc[4 * j + 1] & 0xFFFF);
    o[16 + 4 * j + 1] = (uint16_t)(acc[4 * j + 1] >> 16);
    o[16 + 4 * j + 2] = (uint16_t)(acc[4 * j + 3] & 0xFFFF);
    o[16 + 4 * j + 3] = (uint16_t)(acc[4 * j + 3] >> 16);
  }
}

void launch_lut_scan(uint32_t groups, const uint8_t* tables, const uint8_t* blocks,
                     uint64_t nblocks, uint16_t* out, cudaStream_t st) {
  if (nblocks == 0) return;
  k_lut_scan<<<(unsigned)((nblocks + 127) / 128), 128, 0, st>>>(groups, tables, blocks, nblocks,
                                                                out);
}

}  // namespace sg
