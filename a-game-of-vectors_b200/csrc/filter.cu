// filter.cu — metadata filters of filter::search (src/filter.rs): Filter::new on the device and the
// Brute plan's exact int8 scoring of every allowed row.
//
//   Filter::new (src/filter.rs:27-38): rows = the set bits of the allow bitset, ascending;
//     per_cluster[c] = slots of cluster c whose row is allowed (PAD never is).
//   Plan::Brute (src/filter.rs:95-105): score = (dot_i8i8(wq, row) as f32) * inv for every allowed
//     row, TopK(k) in (score desc, row asc) order.
// Bits at rows >= n are ignored (they name no row of the corpus).
#include "common.cuh"
#include "internal.hpp"

namespace sg {

constexpr uint32_t kWordsPerThread = 8;
constexpr uint32_t kTileWords = 256 * kWordsPerThread;  // words per CTA of the row kernels

SG_DEV uint64_t word_masked(const uint64_t* allow, uint64_t w, uint64_t words, uint64_t n) {
  if (w >= words || w * 64 >= n) return 0;
  const uint64_t v = allow[w];
  const uint64_t valid = n - w * 64;
  return valid >= 64 ? v : v & ((1ull << valid) - 1);
}

// allowed rows per tile of kTileWords words
__global__ void __launch_bounds__(256) k_filter_tile_counts(const uint64_t* __restrict__ allow,
                                                            uint64_t words, uint64_t n,
                                                            uint32_t* __restrict__ tile_cnt) {
  __shared__ uint32_t tmp[32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kTileWords + threadIdx.x * kWordsPerThread;
  uint32_t c = 0;
  for (uint32_t i = 0; i < kWordsPerThread; i++) c += __popcll(word_masked(allow, w0 + i, words, n));
  const uint32_t total = block_sum(c, tmp);
  if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

// exclusive scan of the tile counts in one CTA (tile_off[ntiles] = total)
__global__ void __launch_bounds__(1024) k_filter_tile_scan(const uint32_t* __restrict__ tile_cnt,
                                                           uint32_t ntiles,
                                                           uint32_t* __restrict__ tile_off) {
  __shared__ uint32_t tmp[32];
  uint32_t carry = 0;
  for (uint32_t b = 0; b < ntiles; b += blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    uint32_t total;
    const uint32_t off = block_exclusive_scan(i < ntiles ? tile_cnt[i] : 0u, tmp, &total);
    if (i < ntiles) tile_off[i] = carry + off;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_off[ntiles] = carry;
}

__global__ void __launch_bounds__(256) k_filter_rows(const uint64_t* __restrict__ allow,
                                                     uint64_t words, uint64_t n,
                                                     const uint32_t* __restrict__ tile_off,
                                                     uint32_t* __restrict__ rows) {
  __shared__ uint32_t tmp[32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kTileWords + threadIdx.x * kWordsPerThread;
  uint64_t v[kWordsPerThread];
  uint32_t c = 0;
  for (uint32_t i = 0; i < kWordsPerThread; i++) {
    v[i] = word_masked(allow, w0 + i, words, n);
    c += __popcll(v[i]);
  }
  uint32_t total;
  uint32_t o = tile_off[blockIdx.x] + block_exclusive_scan(c, tmp, &total);
  for (uint32_t i = 0; i < kWordsPerThread; i++)
    for (uint64_t b = v[i]; b; b &= b - 1) rows[o++] = (uint32_t)((w0 + i) * 64 + __ffsll(b) - 1);
}

__global__ void __launch_bounds__(256) k_filter_per_cluster(const uint32_t* __restrict__ block_off,
                                                            const uint32_t* __restrict__ ids,
                                                            const uint64_t* __restrict__ allow,
                                                            uint64_t words, uint64_t n,
                                                            uint32_t* __restrict__ per_cluster) {
  __shared__ uint32_t tmp[32];
  const uint32_t c = blockIdx.x;
  const uint64_t s0 = (uint64_t)block_off[c] * SG_BLOCK, s1 = (uint64_t)block_off[c + 1] * SG_BLOCK;
  uint32_t cnt = 0;
  for (uint64_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
    const uint32_t id = ids[s];
    cnt += id != SG_PAD && id < n && allowed(allow, words, id);
  }
  const uint32_t total = block_sum(cnt, tmp);
  if (threadIdx.x == 0) per_cluster[c] = total;
}

int filter_build(const DevIndex& ix, const uint64_t* allow, uint64_t words, uint32_t** rows,
                 uint64_t* nrows, uint32_t* per_cluster, cudaStream_t st) {
  *rows = nullptr;
  *nrows = 0;
  const uint64_t used = std::min<uint64_t>(words, (ix.n + 63) / 64);
  const uint32_t ntiles = (uint32_t)((used + kTileWords - 1) / kTileWords);
  uint32_t* tiles = nullptr;
  cudaError_t e = cudaMallocAsync(&tiles, ((size_t)2 * ntiles + 2) * sizeof(uint32_t), st);
  if (e != cudaSuccess) return fail(SG_ERR_OOM, "filter scratch");
  uint32_t* tile_cnt = tiles;
  uint32_t* tile_off = tiles + ntiles + 1;
  uint32_t total = 0;
  if (ntiles) {
    k_filter_tile_counts<<<ntiles, 256, 0, st>>>(allow, used, ix.n, tile_cnt);
    k_filter_tile_scan<<<1, 1024, 0, st>>>(tile_cnt, ntiles, tile_off);
    e = cudaMemcpyAsync(&total, tile_off + ntiles, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e == cudaSuccess && total) {
    e = cudaMalloc(rows, (size_t)total * sizeof(uint32_t));
    if (e == cudaSuccess) k_filter_rows<<<ntiles, 256, 0, st>>>(allow, used, ix.n, tile_off, *rows);
  }
  if (e == cudaSuccess && ix.k) {
    k_filter_per_cluster<<<ix.k, 256, 0, st>>>(ix.block_off, ix.ids, allow, used, ix.n, per_cluster);
    e = cudaGetLastError();
  }
  cudaFreeAsync(tiles, st);
  if (e != cudaSuccess) {
    if (*rows) cudaFree(*rows);
    *rows = nullptr;
    return fail(SG_ERR_DEVICE, std::string("filter build: ") + cudaGetErrorString(e));
  }
  *nrows = total;
  return SG_OK;
}

// ---- Brute: exact int8 scores of a shared row list -------------------------------------------
// One CTA scores 32 rows (8 warps x 4 rows, held in registers) against kBruteQ queries (their
// int8 weights in shared memory), so each row is read once per kBruteQ queries.
constexpr uint32_t kBruteQ = 8;

__global__ void __launch_bounds__(256) k_brute_scores(const int8_t* __restrict__ corpus,
                                                      const int8_t* __restrict__ wq_all,
                                                      const float* __restrict__ inv_all,
                                                      uint32_t nq, const uint32_t* __restrict__ rows,
                                                      uint32_t nrows, float* __restrict__ scores) {
  __shared__ __align__(16) int8_t wq[kBruteQ][SG_DIM];
  const uint32_t qb = blockIdx.y * kBruteQ;
  const uint32_t nqb = min(kBruteQ, nq - qb);
  for (uint32_t i = threadIdx.x; i < nqb * (SG_DIM / 16); i += blockDim.x)
    reinterpret_cast<int4*>(&wq[0][0])[i] =
        reinterpret_cast<const int4*>(wq_all + (size_t)qb * SG_DIM)[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t j0 = blockIdx.x * 32 + warp * 4;
  int4 x[4][2];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint32_t j = j0 + r;
    const int4* src =
        reinterpret_cast<const int4*>(corpus + (size_t)(j < nrows ? rows[j] : 0) * SG_DIM);
    x[r][0] = j < nrows ? __ldg(src + lane) : make_int4(0, 0, 0, 0);
    x[r][1] = (j < nrows && lane < 16) ? __ldg(src + lane + 32) : make_int4(0, 0, 0, 0);
  }
  for (uint32_t qi = 0; qi < nqb; qi++) {
    const int4 w0 = reinterpret_cast<const int4*>(wq[qi])[lane];
    const int4 w1 = lane < 16 ? reinterpret_cast<const int4*>(wq[qi])[lane + 32] : make_int4(0, 0, 0, 0);
    const float inv = inv_all[qb + qi];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      int s = 0;
      s = __dp4a(x[r][0].x, w0.x, s);
      s = __dp4a(x[r][0].y, w0.y, s);
      s = __dp4a(x[r][0].z, w0.z, s);
      s = __dp4a(x[r][0].w, w0.w, s);
      s = __dp4a(x[r][1].x, w1.x, s);
      s = __dp4a(x[r][1].y, w1.y, s);
      s = __dp4a(x[r][1].z, w1.z, s);
      s = __dp4a(x[r][1].w, w1.w, s);
      s = warp_sum_i(s);
      const uint32_t j = j0 + r;
      if (lane == 0 && j < nrows) scores[(size_t)(qb + qi) * nrows + j] = __fmul_rn((float)s, inv);
    }
  }
}

__global__ void k_fill_u32(uint32_t* p, uint32_t n, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

int launch_brute(const DevIndex& ix, Workspace& w, uint32_t nq, const uint32_t* rows,
                 uint32_t nrows, uint32_t k, float* scores, cudaStream_t st) {
  if (nrows == 0 || k == 0) {
    cudaMemsetAsync(w.out_n, 0, nq * sizeof(uint32_t), st);
    return 1;
  }
  dim3 grid((nrows + 31) / 32, (nq + kBruteQ - 1) / kBruteQ);
  k_brute_scores<<<grid, 256, 0, st>>>(ix.rerank, w.wq, w.winv, nq, rows, nrows, scores);
  k_fill_u32<<<(nq + 255) / 256, 256, 0, st>>>(w.ln, nq, nrows);
  launch_top_list(scores, rows, w.ln, nrows, 0, k, w.out_sc, w.out_id, w.out_n, k, nq, st);
  return 3;
}

}  // namespace sg
