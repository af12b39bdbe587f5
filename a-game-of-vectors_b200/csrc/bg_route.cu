// bg_route.cu — bigann routing (bigann::Index::route, src/bigann.rs:660-678) on the tcgen05
// tensor cores, with the probe lists of the reference's exact FP32 routing.
//
// The reference scores every leaf c by s(c) = 2 <q, c> - |c|^2 (a sequential f32 dot of the
// int8 query with the f32 leaf, src/bigann.rs:664-670) and keeps TopK(nprobe). Here:
//
//   1. Every leaf is stored as two bf16 rows, hi = bf16(c) and lo = bf16(c - hi), side by side in
//      one [K x 208] matrix (100 + 4 zero columns each), and every int8 query as [q, 0, q, 0] in
//      bf16 (exact). One kind::f16 MMA chain over K = 208 gives <q, hi> + <q, lo> with exact
//      products and FP32 accumulation: the approximate score s~ = 2 acc - |c|^2.
//   2. |s~ - s| <= delta(q) = 5e-4 |q| cmax + 2^-22 cmax^2, cmax the largest leaf norm:
//        c - hi - lo is at most 2^-16 |c| per coordinate (two bf16 roundings, unit roundoff 2^-8);
//        the FP32 accumulation of 208 exact products is allowed 208 * 2^-20 of sum|q_i c_i| (four
//        times the IEEE bound, so a truncating accumulator is covered); the reference's own
//        sequential sum differs from the real dot by <= 100 * 2^-24 * sum|q_i c_i|; the two final
//        f32 operations (2 acc - |c|^2) round by <= 2^-24 of their operands on each side. With
//        sum|q_i c_i| <= |q| |c| the sum of the terms is below delta.
//   3. A threshold from a subset: the same GEMM over every 16th leaf writes its s~, and the
//      nprobe-th best of those, t, bounds the exact nprobe-th best score from below up to delta
//      (a subset's nprobe-th best never exceeds the whole set's). Every leaf of the exact top
//      nprobe therefore has s~ >= t - 2 delta.
//   4. The full GEMM's epilogue emits (leaf, s~) only where s~ >= t - 2 delta, into a per-query
//      list (capacity `cap`).
//   5. Per query: the nprobe-th best s~ of the list, s~P; every listed leaf with
//      s~ >= s~P - 2 delta (which holds every exact top-nprobe leaf, ties included) is rescored with
//      the reference's sequential FP32 dot, and TopK(nprobe) by (score desc, leaf asc) is taken
//      over the rescored window. The margin rule and the exact <q, c> of each kept leaf follow as in
//      the FP32 path. A list that overflowed `cap`, or a window wider than its buffer, falls back to
//      exact FP32 scoring of every leaf in that query's CTA (kStatusWindow is raised).
//
// The GEMM kernel is persistent: one CTA per SM walks a contiguous range of (query group, leaf
// tile) jobs. Warp 0 loads tiles by TMA (no multicast) in the 128-byte swizzle, one copy per
// 64-element k-block (four per tile, the last one zero-filled past column 208): the query group's
// B once per group, each 128-leaf A tile into one of two stages. Warp 1 issues the 13 MMAs of a
// job into one of two TMEM accumulators (M = 128 leaves, N = 64/128/192 queries). Eight epilogue
// warps read the accumulators (two per TMEM lane quarter, one half of the columns each) and emit
// the passing (leaf, score) pairs with one atomic per query and 32 leaves, so the epilogue of one
// job overlaps the loads and MMAs of the next. Every wait is bounded (2 s); a wait that runs out
// raises kStatusTimeout and the CTA stops after its copies in flight have landed.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <float.h>

#include "common.cuh"
#include "internal.hpp"
#include "tcgen05.cuh"

namespace sg {

constexpr uint32_t kHlCols = 208;  // [hi 100, 0 x 4, lo 100, 0 x 4]
constexpr uint32_t kHlLo = 104;    // first column of lo
constexpr uint32_t kBrM = 128;     // leaves per tile (TMEM lanes)
constexpr uint32_t kBrRowBytes = kHlCols * 2;       // 416 B per row in HBM
constexpr uint32_t kBrAtoms = 4;                    // 64-element k-blocks (the last one 16 real)
constexpr uint32_t kBrABytes = kBrAtoms * kBrM * 128;  // 64 KB per A stage (128-byte swizzle)
constexpr uint32_t kBrSteps = kHlCols / 16;         // 13 MMAs of K = 16
constexpr int kBrProducer = 0, kBrMma = 1, kBrEpi0 = 2, kBrEpiWarps = 8;
constexpr int kBrThreads = 32 * (kBrEpi0 + kBrEpiWarps);  // 320
constexpr uint32_t kBrWin = 4096;  // rescoring window of one query (u64 keys in shared memory)
constexpr uint32_t kBrSelThreads = 256;

// The [K x 208] bf16 hi/lo matrix of the leaves, one element per thread.
__global__ void k_bg_leaf_hl(const float* __restrict__ leaves, uint32_t K, __nv_bfloat16* __restrict__ hl) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * kHlCols) return;
  const uint32_t c = (uint32_t)(i / kHlCols), j = (uint32_t)(i % kHlCols);
  float v = 0.0f;
  if (j < SG_BG_DIM) {
    v = __bfloat162float(__float2bfloat16_rn(leaves[(size_t)c * SG_BG_DIM + j]));
  } else if (j >= kHlLo && j < kHlLo + SG_BG_DIM) {
    const float x = leaves[(size_t)c * SG_BG_DIM + (j - kHlLo)];
    const float hi = __bfloat162float(__float2bfloat16_rn(x));
    v = __bfloat162float(__float2bfloat16_rn(__fsub_rn(x, hi)));  // x - hi is exact in f32
  }
  hl[i] = __float2bfloat16_rn(v);
}

// The queries as [q, 0 x 4, q, 0 x 4] bf16 rows (int8 values are exact in bf16).
__global__ void k_bg_q_hl(const int8_t* __restrict__ q, uint32_t nq, __nv_bfloat16* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)nq * kHlCols) return;
  const uint32_t r = (uint32_t)(i / kHlCols), j = (uint32_t)(i % kHlCols);
  float v = 0.0f;
  if (j < SG_BG_DIM) v = (float)q[(size_t)r * SG_BG_DIM + j];
  else if (j >= kHlLo && j < kHlLo + SG_BG_DIM) v = (float)q[(size_t)r * SG_BG_DIM + (j - kHlLo)];
  out[i] = __float2bfloat16_rn(v);
}

struct BrArgs {
  uint32_t K;         // rows of the leaf matrix the map covers
  uint32_t row_step;  // leaf number of matrix row r: r * row_step
  uint32_t nq, N;     // queries; queries per job (64, 128 or 192)
  uint32_t ntiles;    // 128-row tiles of the leaf matrix
  uint64_t njobs;     // ceil(nq / N) * ntiles
  const float* ln;    // |c|^2 per leaf
  uint32_t mode;      // 0: write every s~ to scores [nq x K]; 1: emit s~ >= lim[q] to ent
  float* scores;
  const float* lim;
  uint2* ent;  // [nq x cap] (leaf, s~ bits)
  uint32_t cap;
  uint32_t* cnt;  // per query: entries passed (may exceed cap)
  uint32_t* status;
};

__global__ void __launch_bounds__(kBrThreads, 1) k_bg_route_tc(const __grid_constant__ CUtensorMap map_l,
                                                               const __grid_constant__ CUtensorMap map_q,
                                                               BrArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];  // B [N rows], then the two A stages
  __shared__ __align__(8) uint64_t bar_afull[2], bar_aempty[2], bar_dfull[2], bar_dempty[2], bar_bfull;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int* abort_flag = &s_abort;
  const uint64_t j0 = a.njobs * blockIdx.x / gridDim.x, j1 = a.njobs * (blockIdx.x + 1) / gridDim.x;
  const uint32_t N = a.N, ncols = N <= 64 ? 128 : N <= 128 ? 256 : 512;  // 2N, rounded to a power of two

  if (warp == kBrMma) {
    tc_alloc(&s_tmem, ncols);
    tc_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&bar_afull[i], 1);
      mbar_init(&bar_aempty[i], 1);
      mbar_init(&bar_dfull[i], 1);
      mbar_init(&bar_dempty[i], kBrEpiWarps);
    }
    mbar_init(&bar_bfull, 1);
    s_abort = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t bsm = smem_addr(smem), asm0 = bsm + kBrAtoms * N * 128;
  // one lane waits, the warp follows its verdict (keeps the warp converged for .sync.aligned ops)
  auto wait1 = [&](uint64_t* b, uint32_t par) {
    int r = 0;
    if (lane == 0) r = mbar_wait(b, par, abort_flag) ? 1 : 0;
    return __shfl_sync(0xFFFFFFFFu, r, 0) != 0;
  };

  if (warp == kBrProducer) {
    if (lane == 0) {
      uint32_t cur_qg = 0xFFFFFFFFu, nb = 0;
      uint64_t t = 0;
      for (uint64_t j = j0; j < j1; j++, t++) {
        const uint32_t s = (uint32_t)(t & 1), u = (uint32_t)(t >> 1);
        if (!mbar_wait(&bar_aempty[s], (u & 1) ^ 1, abort_flag)) break;
        const uint32_t qg = (uint32_t)(j / a.ntiles), tile = (uint32_t)(j % a.ntiles);
        if (qg != cur_qg) {
          // B is read by every MMA issued so far: wait for the last job's (its commit tracks all)
          if (t > 0 && !mbar_wait(&bar_aempty[(t - 1) & 1], (uint32_t)(((t - 1) >> 1) & 1), abort_flag)) break;
          mbar_expect_tx(&bar_bfull, kBrAtoms * N * 128);
          for (uint32_t kb = 0; kb < kBrAtoms; kb++)
            tma_load_2d(bsm + kb * N * 128, &map_q, (int32_t)(64 * kb), (int32_t)(qg * N), &bar_bfull);
          cur_qg = qg;
          nb++;
        }
        mbar_expect_tx(&bar_afull[s], kBrABytes);
        for (uint32_t kb = 0; kb < kBrAtoms; kb++)
          tma_load_2d(asm0 + s * kBrABytes + kb * kBrM * 128, &map_l, (int32_t)(64 * kb), (int32_t)(tile * kBrM),
                      &bar_afull[s]);
      }
      // copies in flight land before the CTA leaves (a no-op when every job ran)
      if (*abort_flag) {
        for (uint64_t back = 1; back <= 2 && back <= t; back++) {
          const uint64_t tt = t - back;
          mbar_drain(&bar_afull[tt & 1], (uint32_t)((tt >> 1) & 1));
        }
        if (nb) mbar_drain(&bar_bfull, (nb - 1) & 1);
      }
    }
  } else if (warp == kBrMma) {
    // kind::f16: F32 accumulators, BF16 A and B, both K-major, M = 128, N
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((kBrM >> 4) << 24);
    uint32_t cur_qg = 0xFFFFFFFFu, nb = 0;
    uint64_t t = 0;
    for (uint64_t j = j0; j < j1; j++, t++) {
      const uint32_t s = (uint32_t)(t & 1), u = (uint32_t)(t >> 1);
      const uint32_t qg = (uint32_t)(j / a.ntiles);
      if (qg != cur_qg) {
        if (!wait1(&bar_bfull, nb & 1)) break;
        cur_qg = qg;
        nb++;
      }
      if (!wait1(&bar_dempty[s], (u & 1) ^ 1)) break;
      if (!wait1(&bar_afull[s], u & 1)) break;
      tc_fence_after();
      const uint32_t as = asm0 + s * kBrABytes;
      // K step k: k-block k/4 (rows * 128 B further on), then 32 B into its rows
#pragma unroll
      for (uint32_t k = 0; k < kBrSteps; k++)
        tc_mma_bf16_ss_elect(tmem + s * N, smem_desc_sw128(as + (k >> 2) * (kBrM * 128) + (k & 3) * 32),
                             smem_desc_sw128(bsm + (k >> 2) * (N * 128) + (k & 3) * 32), idesc, k != 0);
      tc_commit_elect(&bar_aempty[s]);
      tc_commit_elect(&bar_dfull[s]);
      __syncwarp();
    }
  } else {
    const uint32_t quarter = warp & 3, half = (warp - kBrEpi0) >> 2;
    uint64_t t = 0;
    for (uint64_t j = j0; j < j1; j++, t++) {
      const uint32_t s = (uint32_t)(t & 1), u = (uint32_t)(t >> 1);
      if (!wait1(&bar_dfull[s], u & 1)) break;
      tc_fence_after();
      const uint32_t qg = (uint32_t)(j / a.ntiles), tile = (uint32_t)(j % a.ntiles);
      const uint32_t row = tile * kBrM + 32 * quarter + lane;
      const bool valid = row < a.K;
      const uint32_t leaf = row * a.row_step;
      const float lnc = valid ? __ldg(a.ln + leaf) : 0.0f;
      for (uint32_t i = 0; i < N / 64; i++) {
        const uint32_t col = half * (N / 2) + 32 * i;
        uint32_t r[32];
        tc_ld32(tmem + ((32u * quarter) << 16) + s * N + col, r);
        tc_wait_ld();
        const uint32_t q0 = qg * N + col;
        if (a.mode == 0) {
#pragma unroll
          for (uint32_t jj = 0; jj < 32; jj++)
            if (valid && q0 + jj < a.nq)
              a.scores[(size_t)(q0 + jj) * a.K + row] = __fsub_rn(__fmul_rn(2.0f, __uint_as_float(r[jj])), lnc);
        } else {
          // 1. every column's passing leaves as a ballot; lane j keeps column j's
          const bool q_on = q0 + lane < a.nq;
          const float my_lim = q_on ? a.lim[q0 + lane] : 0.0f;
          uint32_t mine = 0;
#pragma unroll
          for (uint32_t jj = 0; jj < 32; jj++) {
            const float v = __fsub_rn(__fmul_rn(2.0f, __uint_as_float(r[jj])), lnc);
            r[jj] = __float_as_uint(v);
            const float lj = __shfl_sync(0xFFFFFFFFu, my_lim, jj);
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, valid && v >= lj);
            if (lane == jj) mine = m;
          }
          if (!q_on) mine = 0;
          // 2. one atomic per column with entries, all columns at once (lane j for query q0 + j)
          uint32_t base = 0;
          if (mine) base = atomicAdd(a.cnt + q0 + lane, (uint32_t)__popc(mine));
          // 3. the entries, column by column over the columns that have any
          const uint32_t lt = (1u << lane) - 1u;
          for (uint32_t cols = __ballot_sync(0xFFFFFFFFu, mine != 0); cols; cols &= cols - 1) {
            const uint32_t jj = __ffs(cols) - 1;
            const uint32_t m = __shfl_sync(0xFFFFFFFFu, mine, jj);
            const uint32_t b = __shfl_sync(0xFFFFFFFFu, base, jj);
            float v = 0.0f;
#pragma unroll
            for (uint32_t k = 0; k < 32; k++)
              if (k == jj) v = __uint_as_float(r[k]);
            if ((m >> lane) & 1u) {
              const uint32_t idx = b + (uint32_t)__popc(m & lt);
              if (idx < a.cap) a.ent[(size_t)(q0 + jj) * a.cap + idx] = make_uint2(leaf, __float_as_uint(v));
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_dempty[s]);
    }
  }
  if (tid == 0 && *abort_flag) atomicOr(a.status, kStatusTimeout);
  tc_fence_before();
  __syncthreads();
  if (warp == kBrMma) {
    tc_fence_after();
    tc_dealloc(tmem, ncols);
  }
}

// delta(q) of the header: the bound on |s~ - s| for every leaf.
SG_DEV float route_delta(float qq, float cmax, float cmax2) {
  return __fadd_ru(__fmul_ru(__fmul_ru(5e-4f, __fsqrt_ru(qq)), cmax), __fmul_ru(2.384185791015625e-07f, cmax2));
}

// Per query: lim = (nprobe-th best s~ of the subset) - 2 delta, or -inf without a subset; the
// emission counters start at zero.
__global__ void __launch_bounds__(256) k_bg_route_thr(const float* __restrict__ sub, uint32_t ks, uint32_t P,
                                                      const float* __restrict__ qq, float cmax, float cmax2,
                                                      float* __restrict__ lim, uint32_t* __restrict__ cnt) {
  __shared__ uint32_t hist[2048], tmp[32];
  const uint32_t q = blockIdx.x;
  float l = -INFINITY;
  if (ks >= P && P > 0) {
    const float* row = sub + (size_t)q * ks;
    const uint32_t T = block_select_nth_u32r([&](uint32_t i) { return ord(row[i]); }, ks, P, hist, tmp);
    const float d = route_delta(qq[q], cmax, cmax2);
    l = __fsub_rd(unord(T), __fmul_ru(2.0f, d));
    if (!(l == l)) l = -INFINITY;  // a NaN score: emit everything (the list then overflows to the exact path)
  }
  if (threadIdx.x == 0) {
    lim[q] = l;
    cnt[q] = 0;
  }
}

// The reference's route score of leaf c: 2 <q, c> - |c|^2, the dot a sequential f32 sum from
// -0.0 (src/bigann.rs:664-670, blas::gemm_abt portable).
SG_DEV float bg_exact_score(const float* qf, const float* __restrict__ leaves, const float* __restrict__ ln,
                            uint32_t c, float* dot_out) {
  float d = -0.0f;
  const float* y = leaves + (size_t)c * SG_BG_DIM;
#pragma unroll 4
  for (int i = 0; i < SG_BG_DIM; i++) d = __fadd_rn(d, __fmul_rn(qf[i], __ldg(y + i)));
  if (dot_out) *dot_out = d;
  return __fsub_rn(__fmul_rn(2.0f, d), ln[c]);
}

// Sorts keys[0..P) best first, applies the margin rule on |q - c|^2 = |q|^2 - s (src/bigann.rs:
// 671-677) and writes the kept leaves with their exact dots <q, c>.
SG_DEV void bg_emit_probes(uint64_t* keys, uint32_t P, float margin, float Q, const float* qf,
                           const float* __restrict__ leaves, const float* __restrict__ ln, uint32_t q,
                           uint32_t* __restrict__ probe, float* __restrict__ probe_cent,
                           uint32_t* __restrict__ probe_n) {
  __shared__ uint32_t s_m;
  const uint32_t n2 = next_pow2(P);
  for (uint32_t i = P + threadIdx.x; i < n2; i += blockDim.x) keys[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc(keys, n2);
  if (threadIdx.x == 0) {
    uint32_t m = P;
    if (margin > 0.0f) {
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
    float d;
    bg_exact_score(qf, leaves, ln, c, &d);
    probe[(size_t)q * P + r] = c;
    probe_cent[(size_t)q * P + r] = d;
  }
}

// Step 5 of the header: one CTA (256 threads) per query.
__global__ void __launch_bounds__(kBrSelThreads) k_bg_select_tc(const uint2* __restrict__ ent, const uint32_t* __restrict__ cnt,
                                                       uint32_t cap, uint32_t K, uint32_t P, float margin,
                                                       const float* __restrict__ qq, float cmax, float cmax2,
                                                       const int8_t* __restrict__ qin, const float* __restrict__ leaves,
                                                       const float* __restrict__ ln, uint32_t* __restrict__ probe,
                                                       float* __restrict__ probe_cent, uint32_t* __restrict__ probe_n,
                                                       uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw);  // [kBrWin]
  __shared__ uint32_t hist[2048], tmp[32], s_nw, s_m;
  __shared__ float qf[SG_BG_DIM];
  const uint32_t q = blockIdx.x;
  if (P == 0) {
    if (threadIdx.x == 0) probe_n[q] = 0;
    return;
  }
  if (threadIdx.x < SG_BG_DIM) qf[threadIdx.x] = (float)qin[(size_t)q * SG_BG_DIM + threadIdx.x];
  if (threadIdx.x == 0) s_nw = 0;
  __syncthreads();
  const uint32_t n = cnt[q];
  bool exact_all = n > cap || n < P;
  if (!exact_all) {
    const uint2* E = ent + (size_t)q * cap;
    const uint32_t T = block_select_nth_u32r([&](uint32_t i) { return ord(__uint_as_float(E[i].y)); }, n, P,
                                             hist, tmp);
    const float d = route_delta(qq[q], cmax, cmax2);
    const float lim = __fsub_rd(unord(T), __fmul_ru(2.0f, d));
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint2 e = E[i];
      if (__uint_as_float(e.y) >= lim) {
        const uint32_t slot = atomicAdd(&s_nw, 1u);
        if (slot < kBrWin) keys[slot] = e.x;
      }
    }
    __syncthreads();
    const uint32_t nw = s_nw;
    if (nw < P || nw > kBrWin) {
      exact_all = true;
    } else {
      for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) {
        const uint32_t c = (uint32_t)keys[i];
        keys[i] = rank_key(bg_exact_score(qf, leaves, ln, c, nullptr), c);
      }
      __syncthreads();
      const uint64_t T2 = block_select_nth_u64([&](uint32_t i) { return keys[i]; }, nw, P, hist, tmp);
      uint64_t mine[kBrWin / kBrSelThreads];
      uint32_t nm = 0;
      for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x)
        if (keys[i] >= T2) mine[nm++] = keys[i];
      if (threadIdx.x == 0) s_m = 0;
      __syncthreads();
      for (uint32_t i = 0; i < nm; i++) keys[atomicAdd(&s_m, 1u)] = mine[i];
      __syncthreads();
    }
  }
  if (exact_all) {
    if (threadIdx.x == 0) atomicOr(status, kStatusWindow);
    block_top_keys([&](uint32_t i) { return bg_exact_score(qf, leaves, ln, i, nullptr); }, K, P, keys, hist, tmp);
  }
  bg_emit_probes(keys, P, margin, qq[q], qf, leaves, ln, q, probe, probe_cent, probe_n);
}

// ---- host side ---------------------------------------------------------------------------------
int bg_route_tc_prepare(const float* d_leaves, uint32_t K, __nv_bfloat16* d_hl, cudaStream_t st) {
  const uint64_t n = (uint64_t)K * kHlCols;
  k_bg_leaf_hl<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_leaves, K, d_hl);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

size_t bg_route_tc_hl_elems(uint32_t rows) { return (size_t)rows * kHlCols; }

BgRoutePlan bg_route_plan(uint32_t K, uint32_t P) {
  BgRoutePlan pl;
  pl.ksub = (K + kBgSubStep - 1) / kBgSubStep;
  pl.cap = K;
  pl.subset = false;
  if (P > 0 && K > 8192 && pl.ksub >= 2 * P) {
    const uint64_t cap = std::max<uint64_t>(8192, 32ull * P);
    if (cap < K) {
      pl.cap = (uint32_t)cap;
      pl.subset = true;
    }
  }
  return pl;
}

// Queries per job: B (4 x N x 128 B) and the two A stages (2 x 64 KB) fit in shared memory up to
// N = 192.
static uint32_t queries_per_job(uint32_t nq) { return nq <= 64 ? 64 : nq <= 128 ? 128 : 192; }

cudaError_t launch_bg_route_tc(const BgRouteTc& r, cudaStream_t st) {
  static PerDeviceOnce attr;
  const int gemm_smem_max = (int)(kBrAtoms * 192 * 128 + 2 * kBrABytes);
  attr([&] {
    cudaError_t e = cudaFuncSetAttribute(k_bg_route_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem_max);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_bg_select_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(kBrWin * sizeof(uint64_t)));
    return e;
  });
  const uint32_t nq = r.nq, N = queries_per_job(nq);
  const BgRoutePlan pl = bg_route_plan(r.K, r.P);
  const uint64_t nel = (uint64_t)nq * kHlCols;
  k_bg_q_hl<<<(unsigned)((nel + 255) / 256), 256, 0, st>>>(r.q, nq, r.qhl);
  CUtensorMap map_q, map_full, map_sub;
  if (!encode_bf16_rows(&map_q, r.qhl, kHlCols, nq, kBrRowBytes, N, true) ||
      !encode_bf16_rows(&map_full, r.hl, kHlCols, r.K, kBrRowBytes, kBrM, true) ||
      (pl.subset && !encode_bf16_rows(&map_sub, r.hl, kHlCols, pl.ksub, (uint64_t)kBgSubStep * kBrRowBytes, kBrM, true)))
    return cudaErrorInvalidValue;
  const size_t smem = (size_t)kBrAtoms * N * 128 + 2 * kBrABytes;
  const uint32_t nqg = (nq + N - 1) / N;
  BrArgs a{};
  a.nq = nq;
  a.N = N;
  a.ln = r.ln;
  a.status = r.status;
  if (pl.subset) {
    a.K = pl.ksub;
    a.row_step = kBgSubStep;
    a.ntiles = (pl.ksub + kBrM - 1) / kBrM;
    a.njobs = (uint64_t)nqg * a.ntiles;
    a.mode = 0;
    a.scores = r.sub_scores;
    k_bg_route_tc<<<(unsigned)std::min<uint64_t>(a.njobs, (uint64_t)r.sms), kBrThreads, smem, st>>>(map_sub, map_q, a);
  }
  k_bg_route_thr<<<nq, 256, 0, st>>>(r.sub_scores, pl.subset ? pl.ksub : 0, r.P, r.qq, r.cmax, r.cmax2, r.lim, r.cnt);
  a.K = r.K;
  a.row_step = 1;
  a.ntiles = (r.K + kBrM - 1) / kBrM;
  a.njobs = (uint64_t)nqg * a.ntiles;
  a.mode = 1;
  a.lim = r.lim;
  a.ent = r.ent;
  a.cap = pl.cap;
  a.cnt = r.cnt;
  k_bg_route_tc<<<(unsigned)std::min<uint64_t>(a.njobs, (uint64_t)r.sms), kBrThreads, smem, st>>>(map_full, map_q, a);
  k_bg_select_tc<<<nq, kBrSelThreads, kBrWin * sizeof(uint64_t), st>>>(r.ent, r.cnt, pl.cap, r.K, r.P, r.margin, r.qq, r.cmax,
                                                               r.cmax2, r.q, r.leaves, r.ln, r.probe, r.probe_cent,
                                                               r.probe_n, r.status);
  return cudaGetLastError();
}

}  // namespace sg
