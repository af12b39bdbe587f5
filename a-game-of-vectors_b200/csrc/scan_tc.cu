// scan_tc.cu — the batched LUT scan on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The LUT score of a slot is sum_g T_g[nibble_g] (src/lut.rs:58-60, :116-126). In the one-hot
// basis it is a dot product: the slot is a 1024-long 0/1 row (a 1 at g*16 + nibble_g for each of
// its 64 groups) and the query is its 1024 u8 table entries, stored group-major already. One
// cluster's slots times the tables of the queries that probe it is therefore a
// [slots x 1024] x [1024 x queries] u8 x u8 -> s32 product: exact integers.
//
// This kernel runs that product as tcgen05.mma.kind::i8 with M = 128 slots (a tile of 4 blocks),
// N = the item's queries (padded to 16, at most 64), K = 1024, in a persistent CTA per SM whose
// warps each keep one role:
//   - a loader warp takes (cluster, query group) work items from the queue and fills one of two
//     item slots in shared memory: B (the query tables as K-major core matrices, 8 queries x
//     16 B) and each query's constants, so an item's set-up overlaps the previous item's tiles;
//   - four producer warps build A (the one-hot slots) in registers and write it straight into
//     tensor memory with tcgen05.st: one-hot rows are 32x the size of the codes and never touch
//     shared memory or HBM. Warp w owns TMEM lanes 32*w.. (block w of the tile) and fills the
//     tile's four K chunks (16 groups = 256 one-hot bytes = 64 TMEM columns each);
//   - the MMA warp, converged, issues the 32 MMAs (K = 32) of a tile from one elected lane into
//     one of four TMEM accumulators and signals the A stages and the accumulator through
//     mbarriers (tcgen05.commit). Each MMA costs ~100 SM cycles whatever N up to 128, so a tile
//     costs ~3.2k cycles however many queries share the cluster: the per-cluster split sends
//     clusters that few queries probe to the ALU scan instead;
//   - eight epilogue warps (two per TMEM lane quarter, taking alternate tiles) read the s32
//     scores with tcgen05.ld (one slot per thread, one query per column) and form
//     est = cent + mul*(a*score + b) for every column in straight-line code, exactly as the ALU
//     scan does. The admitted (slot, query) bits are transposed across the warp so that each
//     column reserves room for its admitted slots with one atomic, all columns' atomics in
//     flight together, and the entries are written one chunk later, when the reservations have
//     returned.
// Every mbarrier wait is bounded: a wait that runs out raises kStatusTimeout, every role stops,
// and the kernel frees its tensor memory and returns.
//
// A raw form of the same pipeline (kRaw) writes the u16 scores of every (query, slot) pair: it
// is the batched lut::scan behind sg_lut_scan_batch and pins the contraction bit for bit.
#include "common.cuh"
#include "internal.hpp"
#include "tcgen05.cuh"

namespace sg {

constexpr int kTcQG = 64;           // queries per work item (MMA N, padded to a multiple of 16)
constexpr int kTcChunks = 4;        // K chunks per tile: 16 groups = 256 one-hot bytes each
constexpr uint32_t kTcCols = 512;   // TMEM columns: 4 x 64 (A stages) + 4 x 64 (D)
constexpr uint32_t kTcDCol = 256;   // first D column
constexpr int kTcDBufs = 4;         // accumulators
constexpr int kTcProducers = 4;     // warps 0-3 build A
constexpr int kTcEpi = 4;           // warps 4-11 drain D
constexpr int kTcEpiWarps = 8;
constexpr int kTcMma = 12;          // warp 12 issues the MMAs
constexpr int kTcLoader = 13;       // warp 13 loads work items
constexpr int kTcThreads = 14 * 32;
constexpr int kTcBBytes = kTcQG * 1024;  // B of one item slot
constexpr int kTcVStride = 68;      // words per lane row of the epilogue's spills (2 x 32 + pad)
constexpr int kTcVBytes = kTcEpiWarps * 32 * kTcVStride * 4;  // the epilogue warps' spills

// ---- slot-major codes ----------------------------------------------------------------------
// Slot s's 64 nibbles in 8 words (32 B): group g at word g/8, bits 4*(g%8). Source: blocks.bin,
// where group g's byte k holds the nibble of slot k (low) and of slot k+16 (high).
__global__ void k_transcode_tc(const uint8_t* __restrict__ blocks, uint64_t nblocks,
                               uint32_t* __restrict__ out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nblocks * 256) return;
  const uint64_t b = t >> 8;
  const uint32_t s = (uint32_t)(t >> 3) & 31, j = (uint32_t)t & 7;
  const uint8_t* src = blocks + b * SG_BLOCK_BYTES + (s & 15);
  const uint32_t sh = (s >> 4) * 4;
  uint32_t w = 0;
#pragma unroll
  for (int p = 0; p < 8; p++) w |= (uint32_t)((src[(8 * j + p) * 16] >> sh) & 15u) << (4 * p);
  out[t] = w;
}

void transcode_tc(const uint8_t* blocks, uint64_t nblocks, uint32_t* out, cudaStream_t st) {
  if (nblocks == 0) return;
  const uint64_t n = nblocks * 256;
  k_transcode_tc<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(blocks, nblocks, out);
}

// Instruction descriptor of kind::i8: u8 A and B, both K-major, s32 accumulators, M = 128.
SG_DEV uint32_t idesc_u8(uint32_t n) { return (2u << 4) | ((n >> 3) << 17) | ((128u >> 4) << 24); }

SG_DEV uint32_t shl_sat(uint32_t x, uint32_t s) {
  uint32_t d;  // PTX shl clamps shift amounts above 31 to 32: the result is then 0
  asm("shl.b32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(s));
  return d;
}
// One-hot of 8 groups (the 8 nibbles of w): group p's 16 bytes are 4 TMEM columns, the byte of
// its nibble n set to 1 (column 4p + n/4, byte n%4).
SG_DEV void onehot8(uint32_t w, uint32_t* r) {
#pragma unroll
  for (int p = 0; p < 8; p++) {
    const uint32_t n8 = ((w >> (4 * p)) & 15u) << 3;
    r[4 * p + 0] = shl_sat(1u, n8);
    r[4 * p + 1] = shl_sat(1u, n8 - 32u);
    r[4 * p + 2] = shl_sat(1u, n8 - 64u);
    r[4 * p + 3] = shl_sat(1u, n8 - 96u);
  }
}


struct TcArgs {
  const uint4* codes;  // [nslots * 2] slot-major codes
  // admission form
  const float* mul;
  const uint32_t* ids;
  const uint32_t* block_off;
  const uint32_t* clen;
  const uint8_t* tables;
  const float4* qp;
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
  // raw form: items are (query group, chunk of raw_chunk blocks); counters [0] status, [1] next
  uint32_t nq;
  uint64_t nblocks;
  uint32_t raw_chunk;
  uint16_t* out;  // [nq][nblocks * 32]
};

template <bool kRaw>
__global__ void __launch_bounds__(kTcThreads, 1) k_scan_tc(TcArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];  // B of the two item slots
  __shared__ __align__(8) uint64_t bar_afull[kTcChunks], bar_aempty[kTcChunks], bar_dfull[kTcDBufs],
      bar_dempty[kTcDBufs], bar_ifull[2], bar_iempty[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ uint32_t s_meta[2][8];  // b0, nb, cl, ng, qbase, end
  __shared__ float4 s_qc[2][kTcQG];  // cent, a, b, threshold key (as bits)
  __shared__ uint2 s_qk[2][kTcQG];   // candidate order base, query
  __shared__ uint2 s_cb[kTcEpiWarps][2][32];               // per column: reserved base, admitted lanes
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int* abort_flag = &s_abort;

  if (warp == kTcMma) {
    tc_alloc(&s_tmem, kTcCols);
    tc_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < kTcChunks; i++) {
      mbar_init(&bar_afull[i], 4);  // the four producer warps (lane quarters) of the chunk
      mbar_init(&bar_aempty[i], 1);
    }
    for (int i = 0; i < kTcDBufs; i++) {
      mbar_init(&bar_dfull[i], 1);
      mbar_init(&bar_dempty[i], 4);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(&bar_ifull[i], 1);
      mbar_init(&bar_iempty[i], kTcProducers + kTcEpiWarps + 1);
    }
    s_abort = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t bs_base = smem_addr(smem);
  uint32_t* status = kRaw ? a.counters : a.counters + 2;

  if (warp == kTcLoader) {
    // ---- work items into the two item slots ------------------------------------------------
    uint32_t nitems, nchunks = 0;
    if (kRaw) {
      nchunks = (uint32_t)((a.nblocks + a.raw_chunk - 1) / a.raw_chunk);
      nitems = ((a.nq + kTcQG - 1) / kTcQG) * nchunks;
    } else {
      nitems = a.counters[4];
    }
    uint32_t* next_item = kRaw ? a.counters + 1 : a.counters + 5;
    for (uint32_t it = 0;; it++) {
      const uint32_t slot = it & 1, use = it >> 1;
      if (!mbar_wait(&bar_iempty[slot], (use & 1) ^ 1, abort_flag)) break;
      uint32_t item = 0;
      if (lane == 0) item = atomicAdd(next_item, 1u);
      item = __shfl_sync(0xFFFFFFFFu, item, 0);
      if (item >= nitems) {
        if (lane == 0) {
          s_meta[slot][5] = 1;
          mbar_arrive(&bar_ifull[slot]);
        }
        break;
      }
      uint32_t b0, nb, ng, cl, l0 = 0, qbase = 0, c = 0;
      if (kRaw) {
        const uint32_t qg = item / nchunks, ch = item % nchunks;
        qbase = qg * kTcQG;
        ng = min((uint32_t)kTcQG, a.nq - qbase);
        b0 = ch * a.raw_chunk;
        nb = (uint32_t)min((uint64_t)a.raw_chunk, a.nblocks - b0);
        cl = nb * SG_BLOCK;
      } else {
        const uint2 gi = a.gitems[item];
        c = gi.x;
        l0 = a.inv_off[c] + gi.y * kTcQG;
        ng = min((uint32_t)kTcQG, a.inv_off[c + 1] - l0);
        b0 = a.block_off[c];
        nb = a.block_off[c + 1] - b0;
        cl = a.clen[c];
      }
      const uint32_t N = (ng + 15) & ~15u;
      uint8_t* B = smem + slot * kTcBBytes;
      if (nb > 0) {
        // query n's table chunk g (16 B) at (n/8)*8192 + g*128 + (n%8)*16
#pragma unroll 4
        for (uint32_t e = lane; e < N * 64; e += 32) {
          const uint32_t r = e & 7, g = (e >> 3) & 63, n = (e >> 9) * 8 + r;
          uint4 v = make_uint4(0, 0, 0, 0);
          if (n < ng) {
            const uint32_t q = kRaw ? qbase + n : a.inv_list[l0 + n] >> 12;
            v = reinterpret_cast<const uint4*>(a.tables + (size_t)q * SG_GROUPS * 16)[g];
          }
          *reinterpret_cast<uint4*>(B + (n >> 3) * 8192 + g * 128 + r * 16) = v;
        }
      }
      if (!kRaw) {
        for (uint32_t qi = lane; qi < ng; qi += 32) {
          const uint32_t ent = a.inv_list[l0 + qi];
          const uint32_t q = ent >> 12, r = ent & 0xFFFu;
          const float4 p = a.qp[q];
          const float cent = a.probe_sc[(size_t)q * a.P + r];
          const uint32_t thr = *(volatile const uint32_t*)(a.thr + q);
          s_qc[slot][qi] = make_float4(cent, p.z, p.w, __uint_as_float(thr));
          s_qk[slot][qi] = make_uint2(a.probe_off[(size_t)q * a.P + r], q);
        }
      }
      if (lane == 0) {
        s_meta[slot][0] = b0;
        s_meta[slot][1] = nb;
        s_meta[slot][2] = cl;
        s_meta[slot][3] = ng;
        s_meta[slot][4] = qbase;
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
      const uint32_t qbase = s_meta[slot][4];
      const uint32_t N = (ng + 15) & ~15u, ntiles = (nb + 3) >> 2;
      bool ok = true;
      if (warp < kTcProducers) {
        // one-hot A: block 4t + warp of the tile, slot = lane, all four K chunks
        const uint32_t qd = warp;
        const uint32_t lane_base = (32u * qd) << 16;
        auto codes_of = [&](uint32_t t, uint4& lo, uint4& hi) {
          const uint32_t bl = 4 * t + qd;
          lo = hi = make_uint4(0, 0, 0, 0);
          if (t < ntiles && bl < nb) {
            const uint64_t gs = (uint64_t)(b0 + bl) * SG_BLOCK + lane;
            lo = a.codes[2 * gs];
            hi = a.codes[2 * gs + 1];
          }
        };
        uint4 lo, hi, nlo, nhi;
        codes_of(0, lo, hi);
        for (uint32_t t = 0; t < ntiles && ok; t++) {
          codes_of(t + 1, nlo, nhi);
          const uint32_t tp = (ts + t) & 1;
          for (uint32_t ch = 0; ch < kTcChunks; ch++) {
            if (!mbar_wait(&bar_aempty[ch], tp ^ 1, abort_flag)) {
              ok = false;
              break;
            }
            const uint4 cw = ch < 2 ? lo : hi;
            uint32_t r[32];
            onehot8((ch & 1) ? cw.z : cw.x, r);
            tc_st32(tmem + lane_base + ch * 64, r);
            onehot8((ch & 1) ? cw.w : cw.y, r);
            tc_st32(tmem + lane_base + ch * 64 + 32, r);
            tc_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_afull[ch]);
          }
          lo = nlo;
          hi = nhi;
        }
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      } else if (warp == kTcMma) {
        const uint32_t idesc = idesc_u8(N);
        // K step s starts 256 B (two core matrices) further on: 16 in the 16-byte address field
        const uint64_t bdesc = smem_desc(bs_base + slot * kTcBBytes, 128, 8192);
        for (uint32_t t = 0; t < ntiles && ok; t++) {
          const uint32_t ds = ts + t, dbuf = ds & (kTcDBufs - 1), duse = ds / kTcDBufs;
          if (!mbar_wait(&bar_dempty[dbuf], (duse & 1) ^ 1, abort_flag)) break;
          tc_fence_after();
          for (uint32_t ch = 0; ch < kTcChunks; ch++) {
            if (!mbar_wait(&bar_afull[ch], ds & 1, abort_flag)) {
              ok = false;
              break;
            }
            tc_fence_after();
#pragma unroll
            for (uint32_t kk = 0; kk < 8; kk++)  // K bytes 32*(8ch + kk).. = groups 2*(8ch + kk), +1
              tc_mma_i8_elect(tmem + kTcDCol + dbuf * kTcQG, tmem + ch * 64 + kk * 8,
                              bdesc + (uint64_t)((ch * 8 + kk) * 16), idesc, (ch | kk) != 0);
            tc_commit_elect(&bar_aempty[ch]);
            if (ch == kTcChunks - 1) tc_commit_elect(&bar_dfull[dbuf]);
            __syncwarp();
          }
        }
        if (lane == 0) mbar_arrive(&bar_iempty[slot]);
      } else {
        // ---- epilogue: slot (4t + qd)*32 + lane of the tiles of this warp's parity ----------
        const uint32_t ew = warp - kTcEpi, qd = ew & 3, par = ew >> 2;
        const uint32_t lane_base = (32u * qd) << 16;
        const uint32_t ncc = (N + 31) >> 5;
        uint2* cb = &s_cb[ew][0][0];
        uint32_t* vrow = reinterpret_cast<uint32_t*>(smem + 2 * kTcBBytes) + (ew * 32 + lane) * kTcVStride;
        const uint32_t lt = (1u << lane) - 1u;
        // A chunk's entries are written one chunk later, so the atomic that reserves their room
        // is in flight meanwhile: p_* is the pending chunk (its spill row and column ballots in
        // buffer p_buf, its reservation in p_base).
        bool p_on = false;
        uint32_t p_adm = 0, p_base = 0, p_loc = 0, p_gslot = 0, p_c0 = 0, p_buf = 0;
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
              a.cbuf_est[(size_t)qk.y * a.cap + pos] = vrow[p_buf * 32 + j];
              a.cbuf_info[(size_t)qk.y * a.cap + pos] = make_uint2(qk.x + p_loc, p_gslot);
            } else {
              a.overflow[qk.y] = 1;
            }
          }
          __syncwarp();
          p_on = false;
        };
        // the warp's next tile's mul values are loaded one tile ahead
        auto tile_mul = [&](uint32_t t) {
          const uint32_t bl = 4 * t + qd;
          if (kRaw || t >= ntiles || bl >= nb || bl * SG_BLOCK + lane >= cl) return 0.0f;
          return a.mul[(b0 + bl) * SG_BLOCK + lane];
        };
        const uint32_t t0 = ((ts & 1) == par) ? 0 : 1;  // first tile of this warp's parity
        float mv = tile_mul(t0);
        for (uint32_t t = t0; t < ntiles; t += 2) {
          const uint32_t ds = ts + t, dbuf = ds & (kTcDBufs - 1), duse = ds / kTcDBufs;
          const uint32_t bl = 4 * t + qd;
          const uint32_t loc = bl * SG_BLOCK + lane;
          const bool lane_ok = bl < nb && loc < cl;
          const uint32_t gslot = (b0 + bl) * SG_BLOCK + lane;
          const float nmv = tile_mul(t + 2);
          if (!mbar_wait(&bar_dfull[dbuf], duse & 1, abort_flag)) break;
          tc_fence_after();
          for (uint32_t cc = 0; cc < ncc; cc++) {
            uint32_t v[32];
            tc_ld32(tmem + lane_base + kTcDCol + dbuf * kTcQG + 32 * cc, v);
            tc_wait_ld();
            if (kRaw) {
              if (lane_ok) {
#pragma unroll
                for (int j = 0; j < 32; j++)
                  if (32 * cc + j < ng) a.out[(size_t)(qbase + 32 * cc + j) * (a.nblocks * SG_BLOCK) + gslot] = (uint16_t)v[j];
              }
              continue;
            }
            // 1. every column's estimate, exactly as the ALU scan forms it (the score is exact in
            //    f32 through the 2^23 bias trick), and its admission test against the query's key
            const uint32_t cbuf = p_on ? (p_buf ^ 1) : 0;
            uint32_t* vr = vrow + cbuf * 32;
            const uint32_t ncol = min(32u, ng - 32 * cc);
            uint32_t adm = 0;
#pragma unroll
            for (int j4 = 0; j4 < 8; j4++) {
              uint32_t e4[4];
#pragma unroll
              for (int e = 0; e < 4; e++) {
                const int j = 4 * j4 + e;
                const float4 qc = s_qc[slot][32 * cc + j];
                const float sf = __fsub_rn(__uint_as_float(v[j] | 0x4B000000u), 8388608.0f);
                const float est = __fadd_rn(qc.x, __fmul_rn(mv, __fadd_rn(__fmul_rn(qc.y, sf), qc.z)));
                e4[e] = __float_as_uint(est);
                adm |= (ord(est) >= __float_as_uint(qc.w) ? 1u : 0u) << j;
              }
              *reinterpret_cast<uint4*>(vr + 4 * j4) = make_uint4(e4[0], e4[1], e4[2], e4[3]);
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
            p_loc = loc;
            p_gslot = gslot;
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
  tc_fence_before();
  __syncthreads();
  if (warp == kTcMma) {
    tc_fence_after();
    tc_dealloc(tmem, kTcCols);
  }
}

static int tc_smem_bytes() { return 2 * kTcBBytes + kTcVBytes; }

template <bool kRaw>
static void tc_set_attr() {
  static PerDeviceOnce attr;
  attr([] {
    return cudaFuncSetAttribute(k_scan_tc<kRaw>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes());
  });
}

// A query's threshold raised to the cand-th largest estimate key its candidate buffer holds.
// Every buffered entry is a scanned slot that stays in the buffer, and the cut takes the best
// cand entries before the SOAR dedup (src/ivf.rs:698-726), so the final cand-th estimate is at
// least this value: slots below it can never be among the candidates.
__global__ void __launch_bounds__(1024) k_raise_thr(const uint32_t* __restrict__ cbuf_est, uint32_t cap,
                                                    const uint32_t* __restrict__ ccount,
                                                    const uint8_t* __restrict__ overflow, uint32_t cand,
                                                    uint32_t* __restrict__ thr) {
  __shared__ uint32_t hist[2048];
  __shared__ uint32_t tmp[32];
  const uint32_t q = blockIdx.x;
  const uint32_t M = min(ccount[q], cap);
  if (overflow[q] || cand == 0 || M < cand) return;
  const uint32_t* E = cbuf_est + (size_t)q * cap;
  const uint32_t T = block_select_nth_u32r([&](uint32_t i) { return ord(__uint_as_float(E[i])); }, M, cand, hist, tmp);
  if (threadIdx.x == 0 && T > thr[q]) thr[q] = T;
}

int launch_scan_tc(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p, const uint64_t* allow,
                   uint64_t allow_words, int sms, const Config& cfg, uint32_t chunk_blocks, cudaStream_t st) {
  const uint32_t P = probe_stride(ix, p.nprobe);
  const uint32_t split = cfg.tc_split, tmin = std::max<uint32_t>(cfg.tc_min_queries, 1);
  TcArgs a{};
  a.codes = reinterpret_cast<const uint4*>(ix.blocks_tc);
  a.mul = ix.mul;
  a.ids = ix.ids;
  a.block_off = ix.block_off;
  a.clen = ix.clen;
  a.tables = w.tables;
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
  tc_set_attr<false>();
  int launches = 0;
  // the ALU chunk pass: the routing kernel's rank-0 chunks past the seed, then the chunks of
  // the pairs whose clusters too few queries probe (appended by k_alu_split)
  auto alu_pass = [&]() {
    launch_scan(ix, w, nq, p, allow, allow_words, sms, chunk_blocks, 0, (int)cfg.scan_ctas_per_sm, st);
    // a later round's ALU pass starts where this one's queue ended
    cudaMemcpyAsync(w.counters + 1, w.counters, 4, cudaMemcpyDeviceToDevice, st);
  };
  // one tensor-core round: the bound pass with its exact recheck (default), or the exact one-hot
  // contraction (SIEVE_GPU_TC=2, kept for comparison)
  const bool bound = cfg.tc != 2;
  const uint32_t qg = kTcQG;
  auto tc_round = [&]() {
    if (bound) return launch_scan_tcf(ix, w, nq, P, allow, allow_words, sms, st);
    k_scan_tc<false><<<sms, kTcThreads, tc_smem_bytes(), st>>>(a);
    return 1;
  };
  if (bound) {
    launch_filter_prep(w, nq, st);
    launches++;
  }
  if (split > 1 && split < P) {
    launch_invert(ix, w, nq, P, qg, 1, split, st, tmin, chunk_blocks);
    alu_pass();
    launches += tc_round();
    k_raise_thr<<<nq, 1024, 0, st>>>(w.cbuf_est, w.cbuf_per_q, w.ccount, w.overflow, p.cand, w.thr);
    launches += 6;
  }
  launch_invert(ix, w, nq, P, qg, split > 1 && split < P ? split : 1, P, st, tmin, chunk_blocks);
  alu_pass();
  launches += tc_round();
  return launches + 5;
}

// Raw scores of nq query tables against nblocks blocks (slot-major codes already on the device);
// counters: 2 words on the device, zeroed by the caller ([0] status, [1] next item).
void launch_lut_scan_tc(uint32_t nq, const uint8_t* tables, const uint32_t* codes, uint64_t nblocks,
                        uint16_t* out, uint32_t* counters, int sms, cudaStream_t st) {
  TcArgs a{};
  a.codes = reinterpret_cast<const uint4*>(codes);
  a.tables = tables;
  a.counters = counters;
  a.nq = nq;
  a.nblocks = nblocks;
  a.raw_chunk = 64;
  a.out = out;
  tc_set_attr<true>();
  const uint64_t items = (uint64_t)((nq + kTcQG - 1) / kTcQG) * ((nblocks + 63) / 64);
  const unsigned grid = (unsigned)std::min<uint64_t>(items, (uint64_t)sms);
  k_scan_tc<true><<<grid, kTcThreads, tc_smem_bytes(), st>>>(a);
}

}  // namespace sg
