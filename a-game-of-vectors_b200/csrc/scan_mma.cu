// scan_mma.cu — the batched LUT scan on the tensor cores.
//
// The LUT score of a slot is sum_g T_g[nibble_g] (src/lut.rs:58-60, :116-126). Written over a
// one-hot basis it is a dot product: the slot is a 1024-long 0/1 vector (a 1 at g*16 + nibble_g
// for each of its 64 groups) and the query is its 1024 u8 table entries (the tables are already
// stored group-major, g*16 + c). For a batch, many queries probe the same cluster, so one
// cluster's slots times the tables of the queries probing it is a [slots x 1024] x [1024 x queries]
// u8 x u8 -> s32 matrix product: exact integers, on the tensor pipe, with the cluster's codes read
// once for all of those queries.
//
// Work: after routing, the (query, probe rank >= 1) pairs are inverted into per-cluster query
// lists (count, scan, fill), cut into groups of up to 64 queries. A persistent grid drains the
// (cluster, group) items. One CTA stages the group's 64 tables in shared memory as the B operand
// (column stride 1040 B so ldmatrix rows hit distinct banks); each warp takes one 32-slot block
// at a time, builds the one-hot A fragments in registers straight from the codes, and runs
// mma.sync.m16n8k32 u8 over 32 k-steps for 2 m-tiles x up to 8 n-tiles. The epilogue forms
// est = cent + mul*(a*score + b) exactly as the ALU scan does and appends every eligible slot
// at or above the query's threshold (set by the seed pass) to the query's candidate buffer.
// The probes the seed pass covered (scan.cu) are left out, so every (query, probe) pair is
// scanned once.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

constexpr int kQG = 64;           // queries per group: 8 n-tiles of 8
constexpr int kBStride = 1040;    // bytes per query column of B in shared memory

// Device layout for the MMA scan: word (b, kk, g) holds the four code bytes thread row g needs
// at k-step kk: byte g and byte g+8 of group 2kk, then of group 2kk+1 (blocks.bin layout:
// group G's byte j = nibble of slot j | nibble of slot j+16 << 4).
__global__ void k_transcode_mma(const uint8_t* __restrict__ blocks, uint64_t nblocks,
                                uint32_t* __restrict__ out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nblocks * 256) return;
  const uint64_t b = t >> 8;
  const uint32_t kk = (uint32_t)(t >> 3) & 31, g = (uint32_t)t & 7;
  const uint8_t* src = blocks + b * SG_BLOCK_BYTES;
  const uint32_t g0 = 2 * kk * 16, g1 = (2 * kk + 1) * 16;
  out[t] = (uint32_t)src[g0 + g] | ((uint32_t)src[g0 + g + 8] << 8) | ((uint32_t)src[g1 + g] << 16) |
           ((uint32_t)src[g1 + g + 8] << 24);
}

int transcode_mma(const uint8_t* blocks, uint64_t nblocks, uint32_t* out) {
  if (nblocks == 0) return 0;
  const uint64_t n = nblocks * 256;
  k_transcode_mma<<<(unsigned)((n + 255) / 256), 256>>>(blocks, nblocks, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---- inversion of the probe lists ----------------------------------------------------------
// Probes the seed covered (seed_items[q].y) are not scanned again.
__global__ void k_inv_count(const uint32_t* __restrict__ probe_cl, const uint32_t* __restrict__ probe_n,
                            const uint4* __restrict__ seed, uint32_t P, uint32_t nq, uint32_t rlo, uint32_t rhi,
                            uint32_t* __restrict__ cnt) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (uint64_t)nq * P) return;
  const uint32_t q = (uint32_t)(t / P), r = (uint32_t)(t % P);
  if (r < seed[q].y || r >= probe_n[q] || r < rlo || r >= rhi) return;
  atomicAdd(cnt + probe_cl[t], 1u);
}

// One CTA: exclusive scan of the per-cluster counts, and the (cluster, group) items of the
// clusters probed by at least tmin queries (the others go to the ALU scan, k_alu_split).
__global__ void __launch_bounds__(1024) k_inv_scan(const uint32_t* __restrict__ cnt, uint32_t K, uint32_t qg,
                                                   uint32_t tmin, uint32_t* __restrict__ off,
                                                   uint2* __restrict__ gitems, uint64_t gcap,
                                                   uint32_t* __restrict__ counters) {
  __shared__ uint32_t tmp[32];
  const uint32_t per = (K + blockDim.x - 1) / blockDim.x;
  const uint32_t c0 = threadIdx.x * per, c1 = min(K, c0 + per);
  uint32_t s = 0, gsum = 0;
  for (uint32_t c = c0; c < c1; c++) {
    s += cnt[c];
    gsum += cnt[c] >= tmin ? (cnt[c] + qg - 1) / qg : 0;
  }
  uint32_t tot, gtot;
  uint32_t base = block_exclusive_scan(s, tmp, &tot);
  uint32_t gbase = block_exclusive_scan(gsum, tmp, &gtot);
  for (uint32_t c = c0; c < c1; c++) {
    off[c] = base;
    const uint32_t ng = cnt[c] >= tmin ? (cnt[c] + qg - 1) / qg : 0;
    for (uint32_t j = 0; j < ng; j++)
      if (gbase + j < gcap) gitems[gbase + j] = make_uint2(c, j);
    base += cnt[c];
    gbase += ng;
  }
  if (threadIdx.x == 0) {
    off[K] = tot;
    counters[4] = (uint32_t)min((uint64_t)gtot, gcap);
    counters[5] = 0;
  }
}

__global__ void k_inv_fill(const uint32_t* __restrict__ probe_cl, const uint32_t* __restrict__ probe_n,
                           const uint4* __restrict__ seed, uint32_t P, uint32_t nq, uint32_t rlo, uint32_t rhi,
                           const uint32_t* __restrict__ off, uint32_t* __restrict__ fill,
                           uint32_t* __restrict__ list) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (uint64_t)nq * P) return;
  const uint32_t q = (uint32_t)(t / P), r = (uint32_t)(t % P);
  if (r < seed[q].y || r >= probe_n[q] || r < rlo || r >= rhi) return;
  const uint32_t c = probe_cl[t];
  list[off[c] + atomicAdd(fill + c, 1u)] = (q << 12) | r;
}

// ---- the MMA scan --------------------------------------------------------------------------
SG_DEV uint32_t shl_clamp(uint32_t x, uint32_t s) {
  uint32_t d;  // PTX shl clamps shift amounts above 31 to 32: the result is then 0
  asm("shl.b32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(s));
  return d;
}

// Smallest LUT score `acc` at which some slot of a cluster whose mul values lie in [lo, hi] can
// reach the admission key `thr` of a query (cent, a, b): est = cent + mul*(a*acc + b) rounded
// operation by operation as the epilogue forms it. With a >= 0 and 0 <= lo <= hi, the bound
// U(acc) = cent + m*(a*acc + b), m = hi where a*acc + b >= 0 and lo below, is at least every
// slot's estimate (rounding is monotone in each operand) and is itself non-decreasing in acc,
// so every slot with a score below the returned floor has ord(est) < thr and is rejected
// without forming its estimate. Returns 0 where the bound does not apply, kMaxLutScore + 1
// where no score can reach thr.
constexpr uint32_t kMaxLutScore = SG_GROUPS * 255;

SG_DEV uint32_t score_floor(float cent, float a, float b, float lo, float hi, uint32_t thr) {
  if (thr == 0) return 0;
  const float xmax = __fadd_rn(__fmul_rn(a, (float)kMaxLutScore), b);
  if (!(lo >= 0.0f) || !(hi >= lo) || !(a >= 0.0f) || !isfinite(xmax) || !isfinite(b) ||
      !isfinite(cent) || !isfinite(__fmul_rn(hi, xmax)) || !isfinite(__fmul_rn(hi, b)))
    return 0;
  auto U = [&](uint32_t acc) {
    const float x = __fadd_rn(__fmul_rn(a, (float)acc), b);
    return ord(__fadd_rn(cent, __fmul_rn(x >= 0.0f ? hi : lo, x)));
  };
  if (U(0) >= thr) return 0;
  if (U(kMaxLutScore) < thr) return kMaxLutScore + 1;
  uint32_t l = 0, h = kMaxLutScore;  // U(l) < thr <= U(h)
  while (h - l > 1) {
    const uint32_t m = (l + h) >> 1;
    if (U(m) >= thr) h = m;
    else l = m;
  }
  return h;
}

SG_DEV void mma_u8(int* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

SG_DEV void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g));
}
SG_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
SG_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

SG_DEV void ldsm_x4(uint32_t* r, uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}

struct MmaArgs {
  const uint32_t* bmma;
  const float* mul;
  const uint32_t* ids;
  const uint32_t* block_off;
  const uint32_t* clen;
  const float2* mul_rng;
  const uint8_t* tables;
  const float4* qp;
  const float* probe_sc;
  const uint32_t* probe_off;
  uint32_t P;
  const uint32_t* inv_off;
  const uint32_t* inv_list;
  const uint2* gitems;
  uint32_t* counters;
  uint32_t* thr;
  uint32_t* ccount;
  uint32_t* cbuf_est;
  uint2* cbuf_info;
  uint32_t cap;
  uint8_t* overflow;
  const uint64_t* allow;
  uint64_t allow_words;
  const uint64_t* const* allow_q;  // per-query allow bitsets (null entries: no filter), or null
  const uint64_t* allow_wq;
};

// Per warp, two shared-memory stages of one block each: its 256 code words (1 KB) and its 32
// `mul` factors (128 B). A warp copies its next block in with cp.async while it computes the
// current one, so the L2/HBM latency of a block is hidden behind a whole block of MMAs.
constexpr int kStageWords = 256 + 32;

__global__ void __launch_bounds__(256, 2) k_scan_mma(MmaArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint8_t* Bs = smem;                                                     // [kQG][kBStride]
  uint32_t* stage = reinterpret_cast<uint32_t*>(smem + kQG * kBStride);  // [8 warps][2][kStageWords]
  __shared__ float s_cent[kQG], s_a[kQG], s_b[kQG];
  __shared__ uint32_t s_thr[kQG], s_kb[kQG], s_q[kQG];
  __shared__ __align__(8) int s_floor[kQG];  // score floor per query column (INT_MAX: empty column)
  __shared__ uint32_t s_item;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int nwarps = blockDim.x >> 5;
  const uint32_t bs_base = (uint32_t)__cvta_generic_to_shared(Bs);
  uint32_t* my_stage = stage + warp * 2 * kStageWords;
  const uint32_t my_stage_s = (uint32_t)__cvta_generic_to_shared(my_stage);
  // ldmatrix.x4 row address of this lane for n-tile pair 0, k-step 0: matrix m = lane/8 covers
  // (n-tile m/2, k-half m%2); its row r = lane%8 is query column 8*(m/2) + r.
  const uint32_t lm = lane >> 3, lrow = lane & 7;
  const uint32_t lane_off = ((lm >> 1) * 8 + lrow) * kBStride + (lm & 1) * 16;
  const uint32_t ngroups = a.counters[4];
  // issue the copies of block b into stage buffer `buf` (1152 B: 72 x 16 B, <= 3 per lane)
  auto prefetch = [&](uint32_t b, int buf) {
    const uint8_t* src_w = reinterpret_cast<const uint8_t*>(a.bmma + (size_t)b * 256);
    const uint8_t* src_m = reinterpret_cast<const uint8_t*>(a.mul + (size_t)b * SG_BLOCK);
    const uint32_t dst = my_stage_s + buf * kStageWords * 4;
    for (int c = lane; c < 72; c += 32) {
      if (c < 64) cp_async16(dst + c * 16, src_w + c * 16);
      else cp_async16(dst + 1024 + (c - 64) * 16, src_m + (c - 64) * 16);
    }
    cp_async_commit();
  };
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&a.counters[5], 1u);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= ngroups) break;
    const uint2 gi = a.gitems[item];
    const uint32_t c = gi.x;
    const uint32_t l0 = a.inv_off[c] + gi.y * kQG;
    const uint32_t ng = min((uint32_t)kQG, a.inv_off[c + 1] - l0);
    const uint32_t cb0 = a.block_off[c], nb = a.block_off[c + 1] - cb0, cl = a.clen[c];
    if ((uint32_t)warp < nb) prefetch(cb0 + warp, 0);
    for (int e = threadIdx.x; e < kQG * 64; e += blockDim.x) {
      const int qi = e >> 6, part = e & 63;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (qi < (int)ng) {
        const uint32_t q = a.inv_list[l0 + qi] >> 12;
        v = reinterpret_cast<const uint4*>(a.tables + (size_t)q * SG_GROUPS * 16)[part];
      }
      *reinterpret_cast<uint4*>(Bs + qi * kBStride + part * 16) = v;
    }
    if (threadIdx.x < kQG) {
      const int qi = threadIdx.x;
      int fl = 0x7FFFFFFF;
      if (qi < (int)ng) {
        const uint32_t ent = a.inv_list[l0 + qi];
        const uint32_t q = ent >> 12, r = ent & 0xFFFu;
        const float4 p = a.qp[q];
        const float cent = a.probe_sc[(size_t)q * a.P + r];
        const uint32_t thr = *(volatile const uint32_t*)(a.thr + q);
        const float2 mr = a.mul_rng[c];
        s_cent[qi] = cent;
        s_a[qi] = p.z;
        s_b[qi] = p.w;
        s_thr[qi] = thr;
        s_kb[qi] = a.probe_off[(size_t)q * a.P + r];
        s_q[qi] = q;
        fl = (int)score_floor(cent, p.z, p.w, mr.x, mr.y, thr);
      }
      s_floor[qi] = fl;
    }
    __syncthreads();
    const int ntiles = (int)((ng + 7) >> 3);
    int it = 0;
    for (uint32_t bl = warp; bl < nb; bl += nwarps, it++) {
      const uint32_t b = cb0 + bl;
      const int buf = it & 1;
      if (bl + nwarps < nb) {
        prefetch(b + nwarps, buf ^ 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const uint32_t* W = my_stage + buf * kStageWords;
      int acc[2][8][4];
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
          for (int e = 0; e < 4; e++) acc[i][j][e] = 0;
#pragma unroll 2
      for (int kk = 0; kk < 32; kk++) {
        const uint32_t w = W[kk * 8 + g];
        uint32_t A0[4], A1[4];
#pragma unroll
        for (int p = 0; p < 8; p++) {
          const uint32_t n8 = p == 0 ? ((w << 3) & 0x78u) : ((w >> (4 * p - 3)) & 0x78u);
          const uint32_t v = shl_clamp(1u, n8 - 32u * (uint32_t)tig);
          if (p & 1) A1[p >> 1] = v;
          else A0[p >> 1] = v;
        }
#pragma unroll
        for (int jp = 0; jp < 4; jp++) {
          if (2 * jp < ntiles) {
            uint32_t bf[4];
            ldsm_x4(bf, bs_base + lane_off + jp * 16 * kBStride + kk * 32);
            mma_u8(acc[0][2 * jp], A0, bf[0], bf[1]);
            mma_u8(acc[1][2 * jp], A1, bf[0], bf[1]);
            if (2 * jp + 1 < ntiles) {
              mma_u8(acc[0][2 * jp + 1], A0, bf[2], bf[3]);
              mma_u8(acc[1][2 * jp + 1], A1, bf[2], bf[3]);
            }
          }
        }
      }
      // epilogue: rows (slots) 16i + g + 8h, columns (queries) 8j + 2tig + (e & 1)
      const uint32_t loc = bl * SG_BLOCK;
      const float* M = reinterpret_cast<const float*>(W + 256);
      float mv[2][2];
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int h = 0; h < 2; h++) mv[i][h] = M[16 * i + g + 8 * h];
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (j >= ntiles) break;
        const int2 fl = *reinterpret_cast<const int2*>(s_floor + 8 * j + 2 * tig);
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int e = 0; e < 4; e++) {
            if (acc[i][j][e] < ((e & 1) ? fl.y : fl.x)) continue;  // below the cluster's floor
            const uint32_t slot = 16 * i + g + 8 * (e >> 1);
            const uint32_t qi = 8 * j + 2 * tig + (e & 1);
            if (qi < ng && loc + slot < cl) {
              const float est = __fadd_rn(
                  s_cent[qi],
                  __fmul_rn(mv[i][e >> 1], __fadd_rn(__fmul_rn(s_a[qi], (float)acc[i][j][e]), s_b[qi])));
              const uint32_t key = ord(est);
              if (key >= s_thr[qi]) {
                const uint32_t gslot = b * SG_BLOCK + slot;
                const uint32_t q = s_q[qi];
                const uint64_t* al = a.allow_q ? a.allow_q[q] : a.allow;
                const uint64_t aw = a.allow_q ? a.allow_wq[q] : a.allow_words;
                if (!al || allowed(al, aw, a.ids[gslot])) {
                  const uint32_t pos = atomicAdd(a.ccount + q, 1u);
                  if (pos < a.cap) {
                    a.cbuf_est[(size_t)q * a.cap + pos] = __float_as_uint(est);
                    a.cbuf_info[(size_t)q * a.cap + pos] = make_uint2(s_kb[qi] + loc + slot, gslot);
                  } else {
                    a.overflow[q] = 1;
                  }
                }
              }
            }
          }
      }
    }
    __syncthreads();
  }
}

// The (query, probe) pairs left to the ALU scan by the split: every pair of rank in [rlo, rhi)
// past the seed whose cluster fewer than tmin queries probe becomes chunk items (q, rank, b,
// b + chunk) appended to the ALU work queue (counters[0]) after the routing kernel's own items.
__global__ void __launch_bounds__(256) k_alu_split(const uint32_t* __restrict__ probe_cl,
                                                   const uint32_t* __restrict__ probe_n,
                                                   const uint4* __restrict__ seed,
                                                   const uint32_t* __restrict__ block_off,
                                                   const uint32_t* __restrict__ cnt, uint32_t P, uint32_t nq,
                                                   uint32_t rlo, uint32_t rhi, uint32_t tmin, uint32_t chunk,
                                                   uint4* __restrict__ items, uint64_t item_cap,
                                                   uint32_t* __restrict__ counters) {
  __shared__ uint32_t tmp[32], s_base;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t q = 0, r = 0, c = 0, nch = 0;
  if (t < (uint64_t)nq * P) {
    q = (uint32_t)(t / P);
    r = (uint32_t)(t % P);
    if (r >= seed[q].y && r < probe_n[q] && r >= rlo && r < rhi) {
      c = probe_cl[t];
      if (cnt[c] < tmin) nch = (block_off[c + 1] - block_off[c] + chunk - 1) / chunk;
    }
  }
  uint32_t tot;
  const uint32_t off = block_exclusive_scan(nch, tmp, &tot);
  if (threadIdx.x == 0) {
    s_base = tot ? atomicAdd(&counters[0], tot) : 0;
    if ((uint64_t)s_base + tot > item_cap) atomicOr(&counters[2], kStatusOverflow);
  }
  __syncthreads();
  if (!nch) return;
  const uint32_t b0 = block_off[c], b1 = block_off[c + 1];
  uint64_t pos = (uint64_t)s_base + off;
  for (uint32_t b = b0; b < b1; b += chunk, pos++)
    if (pos < item_cap) items[pos] = make_uint4(q, r, b, min(b1, b + chunk));
}

// Per-cluster query lists of the (query, probe) pairs the seed left with probe rank in
// [rlo, rhi), cut into (cluster, group) work items of up to qg queries for the clusters that at
// least tmin queries probe (counters[4] items, counters[5] the next one to take). With
// alu_chunk > 0 the pairs of the other clusters become ALU chunk items (k_alu_split).
void launch_invert(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t P, uint32_t qg, uint32_t rlo,
                   uint32_t rhi, cudaStream_t st, uint32_t tmin, uint32_t alu_chunk) {
  const uint64_t pairs = (uint64_t)nq * P;
  cudaMemsetAsync(w.inv_cnt, 0, (size_t)ix.k * 4, st);
  cudaMemsetAsync(w.inv_fill, 0, (size_t)ix.k * 4, st);
  const unsigned grid = (unsigned)((pairs + 255) / 256);
  k_inv_count<<<grid, 256, 0, st>>>(w.probe_cl, w.probe_n, w.seed_items, P, nq, rlo, rhi, w.inv_cnt);
  k_inv_scan<<<1, 1024, 0, st>>>(w.inv_cnt, ix.k, qg, tmin, w.inv_off, w.gitems, w.gitems_cap, w.counters);
  k_inv_fill<<<grid, 256, 0, st>>>(w.probe_cl, w.probe_n, w.seed_items, P, nq, rlo, rhi, w.inv_off, w.inv_fill,
                                   w.inv_list);
  if (alu_chunk && tmin > 1)
    k_alu_split<<<grid, 256, 0, st>>>(w.probe_cl, w.probe_n, w.seed_items, ix.block_off, w.inv_cnt, P, nq, rlo,
                                      rhi, tmin, alu_chunk, w.items, w.item_cap, w.counters);
}

int launch_scan_mma(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                    const uint64_t* allow, uint64_t allow_words, int sms, cudaStream_t st) {
  const uint32_t P = p.nprobe < ix.k ? p.nprobe : ix.k;
  launch_invert(ix, w, nq, P, kQG, 0, P, st);
  MmaArgs a;
  a.bmma = ix.blocks_mma;
  a.mul = ix.mul;
  a.ids = ix.ids;
  a.block_off = ix.block_off;
  a.clen = ix.clen;
  a.mul_rng = ix.mul_rng;
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
  static PerDeviceOnce attr;
  const int smem = kQG * kBStride + 8 * 2 * kStageWords * 4;
  attr([&] { return cudaFuncSetAttribute(k_scan_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); });
  k_scan_mma<<<sms * 2, 256, smem, st>>>(a);
  return 4;
}

}  // namespace sg
