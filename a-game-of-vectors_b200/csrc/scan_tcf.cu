// scan_tcf.cu — the batched scan's admission pass on the 5th-generation tensor cores: a rigorous
// upper bound of every (slot, query) estimate from a 256-wide binary dot product, and the exact
// LUT score only for the pairs the bound cannot reject.
//
// The exact score of a slot is s = sum_g T_g[n_g] over its 64 nibbles (src/lut.rs:58-60,
// :116-126), with T_g the query's u8 tables (src/lut.rs:33-55). T_g is, up to its per-entry
// rounding, linear in the four bits of the nibble: T_g[c] ~ T_g[0] + sum_{j in c} (T_g[1<<j] -
// T_g[0]). So for per-query integer weights w (s8, one per prefix dimension, from the singleton
// entries of the table, halved when they do not fit) and gamma in {1, 2}:
//   s = sum_g T_g[n_g] = gamma * D + sum_g (T_g[n_g] - gamma * L_g[n_g]),  D = sum_{k: bit k} w_k,
// where L_g[c] = sum_{j in c} w_{4g+j}. Each group's residual lies in [rlo_g, rhi_g], its minimum
// and maximum over the 16 nibbles, computed exactly from the tables. Hence
//   gamma * D + R_lo <= s <= gamma * D + R_hi,   R_lo = sum_g rlo_g, R_hi = sum_g rhi_g,
// all integers below 2^24, exact in f32. D is an exact s32 tensor-core product of the slot's 256
// code bits (u8 0/1, A in tensor memory) and the query's weights (s8, B in shared memory):
// tcgen05.mma.kind::i8 with K = 256, 8 instructions per 128-slot tile, where the exact one-hot
// contraction needs K = 1024 (32 instructions). The K order is free as long as A and B share it:
// byte 32i + 4s + j of a row is bit 8j + s of code word i, so each 4-byte column of A is one
// shift and one mask of a code word, and the weights are stored in that order.
//
// The estimate est = cent + mul * (a * s + b), rounded operation by operation (src/rabitq.rs:
// 127-130), is non-decreasing in s for mul >= 0 (a > 0) and non-increasing for mul < 0, and IEEE
// rounding is monotone. So the same expression evaluated at s_ub = gamma * D + R_hi (mul >= 0) or
// at gamma * D + R_lo (mul < 0) is an upper bound of the exact estimate, and a pair whose bound
// misses the query's admission threshold cannot be admitted. Pairs that pass reserve their entry
// in the query's candidate buffer (estimate field holding the slot's mul), and
// k_tc_recheck replaces it with the exact estimate from the exact LUT score. An entry whose exact
// estimate is below the threshold stays in the buffer with that estimate: the threshold is the
// cand-th estimate of entries already buffered, so such an entry is never among the best cand
// the cut keeps. Results are bit-identical to the exact scan.
//
// Warp roles of the persistent CTA (one per SM), as in the one-hot kernel of scan_tc.cu: a
// loader warp fills two item slots (B weights and per-query constants); four producer warps
// expand their slots' code bits into u8 A rows in tensor memory (one 64-column stage per tile,
// four stages), from the tile's codes that a copy warp streams into an eight-stage shared-memory
// ring with bulk async copies (a tile's 128 slots are 4 KB of contiguous codes); one MMA warp
// issues each tile's 8 MMAs from an elected lane into one of four
// accumulators; sixteen epilogue warps (four per TMEM lane quarter, one per accumulator) bound
// every (slot, query) pair and reserve buffer entries.
// Every mbarrier wait is bounded: a wait that runs out raises kStatusTimeout, every role stops,
// and the CTA frees its tensor memory and returns.
#include <climits>

#include "common.cuh"
#include "internal.hpp"
#include "tcgen05.cuh"

namespace sg {

constexpr int kFQG = 64;            // queries per work item (MMA N, padded to a multiple of 16)
constexpr int kFStages = 4;         // A stages: one tile (128 slots x 256 K bytes = 64 columns) each
constexpr uint32_t kFCols = 512;    // TMEM columns: 4 x 64 (A) + 4 x 64 (D)
constexpr uint32_t kFDCol = 256;    // first D column
constexpr int kFDBufs = 4;          // accumulators
constexpr int kFProducers = 4;      // warps 0-3 build A
constexpr int kFEpi = 4;            // warps 4-19 bound the pairs
constexpr int kFEpiWarps = 16;      // four per TMEM lane quarter, one per accumulator
constexpr int kFMma = 20;           // warp 20 issues the MMAs
constexpr int kFLoader = 21;        // warp 21 loads work items
constexpr int kFCopy = 22;          // warp 22 streams each tile's codes into shared memory
constexpr int kFThreads = 23 * 32;
constexpr float kMagic = 12582912.0f;     // 1.5 * 2^23: floats in [2^23, 2^24) step by 1
constexpr uint32_t kMagicBits = 0x4B400000u;
constexpr int kFCStages = 8;        // code stages: one tile's 128 slots x 32 B each
constexpr int kFCBytes = 4 * SG_BLOCK * 32;  // 4 KB
constexpr int kFBBytes = kFQG * SG_PDIM;  // B of one item slot: 64 queries x 256 s8 weights

// ---- per-query weights and residual bounds --------------------------------------------------
// One CTA of 64 threads per query; thread g owns group g (prefix dimensions 4g..4g+3).
__global__ void __launch_bounds__(64) k_filter_prep(const uint8_t* __restrict__ tables,
                                                    uint32_t* __restrict__ w8, float4* __restrict__ fq) {
  __shared__ int s_hi[2], s_lo[2];
  __shared__ uint32_t s_w[SG_GROUPS];
  const uint32_t q = blockIdx.x, g = threadIdx.x;
  const uint4 row = reinterpret_cast<const uint4*>(tables + (size_t)q * SG_GROUPS * 16)[g];
  int t[16];
  const uint32_t wd[4] = {row.x, row.y, row.z, row.w};
#pragma unroll
  for (int c = 0; c < 16; c++) t[c] = (int)((wd[c >> 2] >> (8 * (c & 3))) & 0xFFu);
  int w[4];
  bool big = false;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    w[j] = t[1 << j] - t[0];
    big |= w[j] > 127 || w[j] < -127;
  }
  const int gam = __syncthreads_or(big) ? 2 : 1;
#pragma unroll
  for (int j = 0; j < 4; j++) w[j] /= gam;  // |w| <= 127 (truncation: any integer keeps the bound)
  int rhi = INT_MIN, rlo = INT_MAX;
#pragma unroll
  for (int c = 0; c < 16; c++) {
    const int L = ((c & 1) ? w[0] : 0) + ((c & 2) ? w[1] : 0) + ((c & 4) ? w[2] : 0) + ((c & 8) ? w[3] : 0);
    const int v = t[c] - gam * L;
    rhi = max(rhi, v);
    rlo = min(rlo, v);
  }
  // The weights in the K order of the A rows: K byte 32i + 4s + j holds the weight of prefix
  // dimension 32i + 8j + s (A column 8i + s is bits s, s+8, s+16, s+24 of code word i). This
  // thread's dimension 4g + m is bit b = 4(g%8) + m of word g/8: j = b/8, s = b%8.
  uint8_t* sw = reinterpret_cast<uint8_t*>(s_w);
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const uint32_t b = 4 * (g & 7) + m;
    sw[32 * (g >> 3) + 4 * (b & 7) + (b >> 3)] = (uint8_t)(int8_t)w[m];
  }
  rhi = warp_sum_i(rhi);
  rlo = warp_sum_i(rlo);
  if ((g & 31) == 0) {
    s_hi[g >> 5] = rhi;
    s_lo[g >> 5] = rlo;
  }
  __syncthreads();
  w8[(size_t)q * SG_GROUPS + g] = s_w[g];
  if (g == 0) fq[q] = make_float4((float)gam, (float)(s_hi[0] + s_hi[1]), (float)(s_lo[0] + s_lo[1]), 0.0f);
}

// Instruction descriptor of kind::i8: u8 A, s8 B, both K-major, s32 accumulators, M = 128.
SG_DEV uint32_t idesc_u8s8(uint32_t n) { return (2u << 4) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24); }

struct TcfArgs {
  const uint4* codes;  // [nslots * 2] slot-major codes
  const float* mul;
  const uint32_t* ids;
  const uint32_t* block_off;
  const uint32_t* clen;
  const uint32_t* w8;   // [nq * 64] s8 weights, 4 per word
  const float4* fq;     // [nq] (gamma, R_hi, R_lo, -)
  const float4* qp;     // [nq] (scale, bias, a, b)
  const float* probe_sc;
  const uint32_t* probe_off;
  uint32_t P;
  const uint32_t* inv_off;
  const uint32_t* inv_list;
  const uint2* gitems;
  uint32_t* counters;  // [2] status, [4] items, [5] next item
  uint32_t* thr;
  uint32_t* ccount;
  uint32_t* cbuf_est;
  uint2* cbuf_info;
  uint32_t cap;
  uint8_t* overflow;
  const uint64_t* allow;
  uint64_t allow_words;
  const uint64_t* const* allow_q;
  const uint64_t* allow_wq;
  uint32_t global;  // global sign codes: centroid score 0, admission key = row
};


__global__ void __launch_bounds__(kFThreads, 1) k_scan_tcf(TcfArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];  // B of the two item slots
  __shared__ __align__(8) uint64_t bar_afull[kFStages], bar_aempty[kFStages], bar_dfull[kFDBufs],
      bar_dempty[kFDBufs], bar_ifull[2], bar_iempty[2], bar_cfull[kFCStages], bar_cempty[kFCStages];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ uint32_t s_meta[2][8];  // b0, nb, cl, ng, -, end
  __shared__ float4 s_qc[2][kFQG];   // cent, a, b, threshold key (as bits)
  __shared__ float4 s_qf[2][kFQG];   // gamma, R_hi, R_lo, threshold as an estimate
  __shared__ uint2 s_qk[2][kFQG];    // candidate order base, query
  __shared__ uint2 s_cb[kFEpiWarps][2][32];  // per column: reserved base, admitted lanes
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int* abort_flag = &s_abort;

  if (warp == kFMma) {
    tc_alloc(&s_tmem, kFCols);
    tc_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < kFStages; i++) {
      mbar_init(&bar_afull[i], kFProducers);
      mbar_init(&bar_aempty[i], 1);
    }
    for (int i = 0; i < kFDBufs; i++) {
      mbar_init(&bar_dfull[i], 1);
      mbar_init(&bar_dempty[i], 4);  // the epilogue warp of each lane quarter that reads buffer i
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(&bar_ifull[i], 1);
      mbar_init(&bar_iempty[i], kFProducers + kFEpiWarps + 2);  // + the MMA and copy warps
    }
    for (int i = 0; i < kFCStages; i++) {
      mbar_init(&bar_cfull[i], 1);
      mbar_init(&bar_cempty[i], kFProducers);
    }
    s_abort = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t bs_base = smem_addr(smem);
  const uint32_t cs_base = bs_base + 2 * kFBBytes;  // the code ring
  uint32_t c_issued = 0;  // the copy warp's tiles issued (lane 0), for the exit path's drain
  uint32_t* status = a.counters + 2;

  if (warp == kFLoader) {
    // ---- work items into the two item slots ------------------------------------------------
    const uint32_t nitems = a.counters[4];
    for (uint32_t it = 0;; it++) {
      const uint32_t slot = it & 1, use = it >> 1;
      if (!mbar_wait(&bar_iempty[slot], (use & 1) ^ 1, abort_flag)) break;
      uint32_t item = 0;
      if (lane == 0) item = atomicAdd(a.counters + 5, 1u);
      item = __shfl_sync(0xFFFFFFFFu, item, 0);
      if (item >= nitems) {
        if (lane == 0) {
          s_meta[slot][5] = 1;
          mbar_arrive(&bar_ifull[slot]);
        }
        break;
      }
      const uint2 gi = a.gitems[item];
      const uint32_t c = gi.x;
      const uint32_t l0 = a.inv_off[c] + gi.y * kFQG;
      const uint32_t ng = min((uint32_t)kFQG, a.inv_off[c + 1] - l0);
      const uint32_t b0 = a.block_off[c], nb = a.block_off[c + 1] - b0, cl = a.clen[c];
      const uint32_t N = (ng + 15) & ~15u;
      uint8_t* B = smem + slot * kFBBytes;
      if (nb > 0) {
        // query n's 16-byte K chunk g at (n/8)*2048 + g*128 + (n%8)*16 (K-major core matrices)
#pragma unroll 4
        for (uint32_t e = lane; e < N * 16; e += 32) {
          const uint32_t r = e & 7, g = (e >> 3) & 15, n = (e >> 7) * 8 + r;
          uint4 v = make_uint4(0, 0, 0, 0);
          if (n < ng) {
            const uint32_t q = a.inv_list[l0 + n] >> 12;
            v = reinterpret_cast<const uint4*>(a.w8 + (size_t)q * SG_GROUPS)[g];
          }
          *reinterpret_cast<uint4*>(B + (n >> 3) * 2048 + g * 128 + r * 16) = v;
        }
      }
      for (uint32_t qi = lane; qi < ng; qi += 32) {
        const uint32_t ent = a.inv_list[l0 + qi];
        const uint32_t q = ent >> 12, r = ent & 0xFFFu;
        const float4 p = a.qp[q];
        const float cent = a.global ? 0.0f : a.probe_sc[(size_t)q * a.P + r];
        const uint32_t thr = *(volatile const uint32_t*)(a.thr + q);
        s_qc[slot][qi] = make_float4(cent, p.z, p.w, __uint_as_float(thr));
        const float4 f = a.fq[q];
        // gamma as an integer; the residual bounds less 1.5 * 2^23 (exact: integers below 2^24)
        s_qf[slot][qi] = make_float4(__uint_as_float((uint32_t)f.x), __fsub_rn(f.y, kMagic),
                                     __fsub_rn(f.z, kMagic), thr ? unord(thr) : -INFINITY);
        s_qk[slot][qi] = make_uint2(a.probe_off[(size_t)q * a.P + r], q);
      }
      if (lane == 0) {
        s_meta[slot][0] = b0;
        s_meta[slot][1] = nb;
        s_meta[slot][2] = cl;
        s_meta[slot][3] = ng;
        s_meta[slot][5] = 0;
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_ifull[slot]);
    }
  } else {
    // ---- consumers: items in order, tiles numbered across items ------------------------------
    uint32_t ts = 0;  // tiles of earlier items
    for (uint32_t it = 0;; it++) {
      const uint32_t slot = it & 1, use = it >> 1;
      if (!mbar_wait(&bar_ifull[slot], use & 1, abort_flag)) break;
      if (s_meta[slot][5]) break;
      const uint32_t b0 = s_meta[slot][0], nb = s_meta[slot][1], cl = s_meta[slot][2], ng = s_meta[slot][3];
      const uint32_t N = (ng + 15) & ~15u, ntiles = (nb + 3) >> 2;
      bool ok = true;
      if (warp == kFCopy) {
        // the codes of tile t (blocks 4t..4t+3, contiguous) into ring stage (ts + t) % kFCStages
        for (uint32_t t = 0; t < ntiles; t++) {
          const uint32_t ds = ts + t, cs = ds % kFCStages, cu = ds / kFCStages;
          int r = 0;
          if (lane == 0) r = mbar_wait(&bar_cempty[cs], (cu & 1) ^ 1, abort_flag) ? 1 : 0;
          if (!__shfl_sync(0xFFFFFFFFu, r, 0)) {
            ok = false;
            break;
          }
          if (lane == 0) {
            const uint32_t bytes = min(4u, nb - 4 * t) * SG_BLOCK * 32;
            mbar_expect_tx(&bar_cfull[cs], bytes);
            bulk_load(cs_base + cs * kFCBytes,
                      reinterpret_cast<const uint8_t*>(a.codes) + (size_t)(b0 + 4 * t) * SG_BLOCK * 32, bytes,
                      &bar_cfull[cs]);
            c_issued = ds + 1;
          }
        }
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      } else if (warp < kFProducers) {
        // A: the code bits of block 4t + warp of the tile as u8 0/1, slot = lane, K = 256
        const uint32_t qd = warp;
        const uint32_t lane_base = (32u * qd) << 16;
        for (uint32_t t = 0; t < ntiles; t++) {
          const uint32_t ds = ts + t, st = ds & (kFStages - 1), su = ds / kFStages;
          const uint32_t cs = ds % kFCStages, cu = ds / kFCStages;
          if (!mbar_wait(&bar_aempty[st], (su & 1) ^ 1, abort_flag) ||
              !mbar_wait(&bar_cfull[cs], cu & 1, abort_flag)) {
            ok = false;
            break;
          }
          // this warp's block of the tile: slot `lane`'s 32 code bytes
          uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
          if (4 * t + qd < nb) {
            const uint4* src = reinterpret_cast<const uint4*>(smem + 2 * kFBBytes + cs * kFCBytes +
                                                              qd * (SG_BLOCK * 32) + lane * 32);
            lo = src[0];
            hi = src[1];
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&bar_cempty[cs]);
          // column 8i + s holds bits s, s+8, s+16, s+24 of code word i as bytes 0/1: prefix
          // dimensions 32i + s, +8, +16, +24 (k_filter_prep orders the weights the same way)
          const uint32_t wd[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
          for (int q4 = 0; q4 < 4; q4++) {  // 16 columns (two code words) per store
            uint32_t r[16];
#pragma unroll
            for (int c = 0; c < 16; c++) r[c] = (wd[2 * q4 + (c >> 3)] >> (c & 7)) & 0x01010101u;
            tc_st16(tmem + lane_base + st * 64 + 16 * q4, r);
          }
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&bar_afull[st]);
        }
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      } else if (warp == kFMma) {
        const uint32_t idesc = idesc_u8s8(N);
        // K step kk starts 256 B (two core matrices) further on: 16 in the 16-byte address field
        const uint64_t bdesc = smem_desc(bs_base + slot * kFBBytes, 128, 2048);
        for (uint32_t t = 0; t < ntiles && ok; t++) {
          const uint32_t ds = ts + t, dbuf = ds & (kFDBufs - 1), duse = ds / kFDBufs;
          const uint32_t st = ds & (kFStages - 1), su = ds / kFStages;
          if (!mbar_wait(&bar_dempty[dbuf], (duse & 1) ^ 1, abort_flag)) break;
          if (!mbar_wait(&bar_afull[st], su & 1, abort_flag)) break;
          tc_fence_after();
#pragma unroll
          for (uint32_t kk = 0; kk < 8; kk++)  // K bytes 32kk.. = prefix dimensions 32kk..32kk+31
            tc_mma_i8_elect(tmem + kFDCol + dbuf * kFQG, tmem + st * 64 + kk * 8, bdesc + (uint64_t)(kk * 16),
                            idesc, kk != 0);
          tc_commit_elect(&bar_aempty[st]);
          tc_commit_elect(&bar_dfull[dbuf]);
          __syncwarp();
        }
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      } else {
        // ---- epilogue: slot (4t + qd)*32 + lane of the tiles of this warp's parity ----------
        const uint32_t ew = warp - kFEpi, qd = ew & 3, par = ew >> 2;  // par: the accumulator it reads
        const uint32_t lane_base = (32u * qd) << 16;
        const uint32_t ncc = (N + 31) >> 5;
        uint2* cb = &s_cb[ew][0][0];
        const uint32_t lt = (1u << lane) - 1u;
        // A chunk's entries are written one chunk later, so the atomic that reserves their room
        // is in flight meanwhile: p_* is the pending chunk (its column ballots in buffer p_buf,
        // its reservation in p_base).
        bool p_on = false;
        // (p_gslot - b0 * SG_BLOCK is the pending slot's position within its cluster)
        uint32_t p_adm = 0, p_base = 0, p_gslot = 0, p_c0 = 0, p_buf = 0;
        float p_mv = 0.0f;
        auto flush = [&]() {
          if (!p_on) return;  // warp-uniform
          uint2* cbp = cb + p_buf * 32;
          cbp[lane].x = p_base;
          __syncwarp();
          for (uint32_t r = p_adm; r; r &= r - 1) {
            const uint32_t j = __ffs(r) - 1;
            const uint2 bc = cbp[j];
            const uint2 qk = s_qk[slot][p_c0 + j];
            const uint32_t pos = bc.x + (uint32_t)__popc(bc.y & lt);
            if (pos < a.cap) {
              // the slot's mul; k_tc_recheck turns it into the exact estimate
              a.cbuf_est[(size_t)qk.y * a.cap + pos] = __float_as_uint(p_mv);
              a.cbuf_info[(size_t)qk.y * a.cap + pos] =
                  make_uint2(a.global ? a.ids[p_gslot] : qk.x + (p_gslot - b0 * SG_BLOCK), p_gslot);
            } else {
              a.overflow[qk.y] = 1;
            }
          }
          __syncwarp();
          p_on = false;
        };
        auto tile_mul = [&](uint32_t t) {
          const uint32_t bl = 4 * t + qd;
          if (t >= ntiles || bl >= nb || bl * SG_BLOCK + lane >= cl) return 0.0f;
          return a.mul[(b0 + bl) * SG_BLOCK + lane];
        };
        const uint32_t t0 = (par + kFDBufs - (ts & (kFDBufs - 1))) & (kFDBufs - 1);  // first tile in its buffer
        float mv = tile_mul(t0);
        for (uint32_t t = t0; t < ntiles; t += kFDBufs) {
          const uint32_t ds = ts + t, dbuf = ds & (kFDBufs - 1), duse = ds / kFDBufs;
          const uint32_t bl = 4 * t + qd;
          const uint32_t loc = bl * SG_BLOCK + lane;
          const bool lane_ok = bl < nb && loc < cl;
          const uint32_t gslot = (b0 + bl) * SG_BLOCK + lane;
          const float nmv = tile_mul(t + kFDBufs);
          // the residual bound that gives an upper bound of the estimate for this slot's mul
          const bool neg = mv < 0.0f;
          const bool always = !isfinite(mv);  // no monotone bound: recheck every column
          if (!mbar_wait(&bar_dfull[dbuf], duse & 1, abort_flag)) break;
          tc_fence_after();
          for (uint32_t cc = 0; cc < ncc; cc++) {
            // 1. every column's bound of the estimate (the exact estimate's operations at the
            //    bound of the score) against the query's admission key, 16 columns at a time (a
            //    group of at most 16 queries fills only the first 16: MMA N = 16)
            const uint32_t cbuf = p_on ? (p_buf ^ 1) : 0;
            const uint32_t ncol = min(32u, ng - 32 * cc);
            uint32_t adm = 0;
            for (uint32_t h = 0; h < (ncol > 16 ? 2u : 1u); h++) {
              uint32_t v[16];
              tc_ld16(tmem + lane_base + kFDCol + dbuf * kFQG + 32 * cc + 16 * h, v);
              tc_wait_ld();
              // The score bound sb = gamma * D + R exactly: gamma * D + 1.5 * 2^23, written into
              // a float's bits, is that float for |gamma * D| < 2^22 (|D| <= 256 * 127), and
              // adding R - 1.5 * 2^23 meets an integer below 2^24. The threshold as an estimate
              // (ord is monotone, so est >= it exactly when ord(est) >= the key; a finite mul
              // gives a non-NaN est), -inf for the empty key.
#pragma unroll
              for (int j = 0; j < 16; j++) {
                const uint32_t col = 32 * cc + 16 * h + j;
                const float4 qc = s_qc[slot][col];
                const float4 qf = s_qf[slot][col];
                const float sb =
                    __fadd_rn(__uint_as_float(v[j] * __float_as_uint(qf.x) + kMagicBits), neg ? qf.z : qf.y);
                const float est = __fadd_rn(qc.x, __fmul_rn(mv, __fadd_rn(__fmul_rn(qc.y, sb), qc.z)));
                adm |= (always || est >= qf.w ? 1u : 0u) << (16 * h + j);
              }
            }
            adm &= lane_ok ? (ncol == 32 ? 0xFFFFFFFFu : (1u << ncol) - 1u) : 0u;
            if (adm && (a.allow || a.allow_q)) {  // allowlist filters (View::hidden)
              const uint32_t id = a.ids[gslot];
              for (uint32_t r = adm; r; r &= r - 1) {
                const uint32_t j = __ffs(r) - 1;
                const uint32_t q = s_qk[slot][32 * cc + j].y;
                const uint64_t* al = a.allow_q ? a.allow_q[q] : a.allow;
                const uint64_t aw = a.allow_q ? a.allow_wq[q] : a.allow_words;
                if (al && !allowed(al, aw, id)) adm &= ~(1u << j);
              }
            }
            if (!__any_sync(0xFFFFFFFFu, adm != 0)) continue;
            // 2. the 32 x 32 bit matrix (lane = slot, bit = column) transposed across the warp:
            //    lane j then holds column j's admitted lanes and reserves their room with one atomic
            uint32_t col = adm;
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) {
              const uint32_t lo = w == 16 ? 0x0000FFFFu : w == 8 ? 0x00FF00FFu : w == 4 ? 0x0F0F0F0Fu
                                  : w == 2 ? 0x33333333u : 0x55555555u;
              const uint32_t y = __shfl_xor_sync(0xFFFFFFFFu, col, w);
              col = (lane & w) ? ((col & ~lo) | ((y & ~lo) >> w)) : ((col & lo) | ((y & lo) << w));
            }
            uint32_t base = 0;
            if (col) base = atomicAdd(a.ccount + s_qk[slot][32 * cc + lane].y, (uint32_t)__popc(col));
            cb[cbuf * 32 + lane] = make_uint2(0, col);
            // 3. the previous pending chunk's entries, then this chunk becomes the pending one
            flush();
            p_on = true;
            p_adm = adm;
            p_base = base;
            p_gslot = gslot;
            p_mv = mv;
            p_c0 = 32 * cc;
            p_buf = cbuf;
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&bar_dempty[dbuf]);
          mv = nmv;
        }
        flush();
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      }
      ts += ntiles;
      if (*abort_flag) break;
    }
  }
  if (tid == 0 && *abort_flag) atomicOr(status, kStatusTimeout);
  // the copy warp's bulk copies in flight land before the CTA leaves (a no-op when every tile ran)
  if (warp == kFCopy && lane == 0 && *abort_flag)
    for (uint32_t back = 1; back <= (uint32_t)kFCStages && back <= c_issued; back++) {
      const uint32_t ds = c_issued - back;
      mbar_drain(&bar_cfull[ds % kFCStages], (ds / kFCStages) & 1);
    }
  tc_fence_before();
  __syncthreads();
  if (warp == kFMma) {
    tc_fence_after();
    tc_dealloc(tmem, kFCols);
  }
}

// The exact estimates of the entries the bound admitted: kRecheckSplit CTAs per query (the
// entries of one query can number hundreds of thousands, so one CTA per query left a long tail),
// each with the query's u8 tables in shared memory; per entry the 64 nibble lookups of its slot
// (src/lut.rs:116-126) and the estimate in the reference's operation order (src/rabitq.rs:127-130).
// The bound pass stored the slot's mul in the entry, and the probe's centroid score comes from
// the entry's admission key: probe r's slots hold keys probe_off[r] .. probe_off[r+1]-1, so r is
// the last probe whose offset is at most the key (the query's probe list sits in shared memory).
// Only the slot's 32-byte code is gathered. A thread takes two entries at a time so their loads
// are in flight together.
constexpr uint32_t kRecheckSplit = 8;
__global__ void __launch_bounds__(256) k_tc_recheck(const uint8_t* __restrict__ tables, const float4* __restrict__ qp,
                                                    const uint4* __restrict__ codes,
                                                    const uint32_t* __restrict__ probe_off,
                                                    const float* __restrict__ probe_sc,
                                                    const uint32_t* __restrict__ probe_n, uint32_t P,
                                                    uint32_t global, const uint32_t* __restrict__ tc_start,
                                                    const uint32_t* __restrict__ ccount, uint32_t cap,
                                                    uint64_t nslots, uint32_t* __restrict__ cbuf_est,
                                                    const uint2* __restrict__ cbuf_info) {
  __shared__ __align__(16) uint8_t T[SG_GROUPS * 16];
  extern __shared__ uint32_t s_po[];  // [np] probe offsets, then [np] centroid scores
  const uint32_t q = blockIdx.x;
  const uint32_t lo = tc_start[q], hi = min(ccount[q], cap);
  const uint32_t first = lo + blockIdx.y * blockDim.x + threadIdx.x, stride = gridDim.y * blockDim.x;
  if (lo + blockIdx.y * blockDim.x >= hi) return;  // uniform over the CTA
  reinterpret_cast<uint32_t*>(T)[threadIdx.x] =
      reinterpret_cast<const uint32_t*>(tables + (size_t)q * SG_GROUPS * 16)[threadIdx.x];
  const uint32_t np = global ? 0u : min(probe_n[q], P);  // global codes: centroid score 0
  float* s_ps = reinterpret_cast<float*>(s_po + np);
  for (uint32_t r = threadIdx.x; r < np; r += blockDim.x) {
    s_po[r] = probe_off[(size_t)q * P + r];
    s_ps[r] = probe_sc[(size_t)q * P + r];
  }
  __syncthreads();
  auto cent_of = [&](uint32_t key) {
    if (np == 0) return 0.0f;
    uint32_t rl = 0, rh = np;  // the first probe whose offset is above the key
    while (rl < rh) {
      const uint32_t mid = (rl + rh) >> 1;
      if (s_po[mid] <= key) rl = mid + 1;
      else rh = mid;
    }
    return s_ps[rl > 0 ? rl - 1 : 0];
  };
  const float4 p = qp[q];
  uint32_t* E = cbuf_est + (size_t)q * cap;
  const uint2* I = cbuf_info + (size_t)q * cap;
  auto score = [&](const uint4& c0, const uint4& c1) {
    const uint32_t wd[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
#pragma unroll
      for (int j = 0; j < 8; j++) s += T[(8 * k + j) * 16 + ((wd[k] >> (4 * j)) & 15u)];
    return s;
  };
  auto estimate = [&](float cent, float m, uint32_t s) {
    return __fadd_rn(cent, __fmul_rn(m, __fadd_rn(__fmul_rn(p.z, (float)s), p.w)));
  };
  for (uint32_t i = first; i < hi; i += 2 * stride) {
    const uint32_t i2 = i + stride;
    const bool two = i2 < hi;
    // only an aborted bound pass leaves an entry unwritten (slot >= nslots)
    const uint2 in = I[i], in2 = two ? I[i2] : make_uint2(0u, 0xFFFFFFFFu);
    const uint32_t gs = in.y, gs2 = in2.y;
    const bool ok = gs < nslots, ok2 = gs2 < nslots;
    uint4 a0 = make_uint4(0, 0, 0, 0), a1 = a0, b0 = a0, b1 = a0;
    float m = 0.0f, m2 = 0.0f, ce = 0.0f, ce2 = 0.0f;
    if (ok) {
      a0 = codes[2 * (size_t)gs];
      a1 = codes[2 * (size_t)gs + 1];
      m = __uint_as_float(E[i]);
      ce = cent_of(in.x);
    }
    if (ok2) {
      b0 = codes[2 * (size_t)gs2];
      b1 = codes[2 * (size_t)gs2 + 1];
      m2 = __uint_as_float(E[i2]);
      ce2 = cent_of(in2.x);
    }
    if (ok) E[i] = __float_as_uint(estimate(ce, m, score(a0, a1)));
    if (ok2) E[i2] = __float_as_uint(estimate(ce2, m2, score(b0, b1)));
  }
}

static int tcf_smem_bytes() { return 2 * kFBBytes + kFCStages * kFCBytes; }

// The tensor-core admission pass over the (cluster, query group) items launch_invert made:
// weights and residual bounds per query, the bound pass, then the exact estimates of what it
// admitted. Returns the kernels launched.
int launch_scan_tcf(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t P, const uint64_t* allow,
                    uint64_t allow_words, int sms, cudaStream_t st) {
  static PerDeviceOnce attr;
  attr([] {
    return cudaFuncSetAttribute(k_scan_tcf, cudaFuncAttributeMaxDynamicSharedMemorySize, tcf_smem_bytes());
  });
  TcfArgs a{};
  a.codes = reinterpret_cast<const uint4*>(ix.blocks_tc);
  a.mul = ix.mul;
  a.ids = ix.ids;
  a.block_off = ix.block_off;
  a.clen = ix.clen;
  a.w8 = w.w8;
  a.fq = w.fq;
  a.qp = w.qp;
  a.probe_sc = w.probe_sc;
  a.probe_off = w.probe_off;
  a.P = P;
  a.inv_off = w.inv_off;
  a.inv_list = w.inv_list;
  a.gitems = w.gitems;
  a.counters = w.counters;
  a.thr = w.thr;
  a.ccount = w.ccount;
  a.cbuf_est = w.cbuf_est;
  a.cbuf_info = w.cbuf_info;
  a.cap = w.cbuf_per_q;
  a.overflow = w.overflow;
  a.allow = allow;
  a.allow_words = allow_words;
  a.allow_q = w.per_query_allow ? w.allow_q : nullptr;
  a.allow_wq = w.allow_wq;
  a.global = ix.global;
  // entries from tc_start[q] on are the bound pass's (earlier ones are exact already)
  cudaMemcpyAsync(w.tc_start, w.ccount, (size_t)nq * 4, cudaMemcpyDeviceToDevice, st);
  k_scan_tcf<<<sms, kFThreads, tcf_smem_bytes(), st>>>(a);
  k_tc_recheck<<<dim3(nq, kRecheckSplit), 256, (size_t)(ix.global ? 0 : P) * 8, st>>>(
      w.tables, w.qp, reinterpret_cast<const uint4*>(ix.blocks_tc), w.probe_off, w.probe_sc, w.probe_n, P,
      ix.global, w.tc_start, w.ccount, w.cbuf_per_q, ix.nslots, w.cbuf_est, w.cbuf_info);
  return 2;
}

void launch_filter_prep(Workspace& w, uint32_t nq, cudaStream_t st) {
  k_filter_prep<<<nq, 64, 0, st>>>(w.tables, w.w8, w.fq);
}

}  // namespace sg
