// invert.cu — the batched path's per-cluster work lists.
//
// After routing, the (query, probe rank) pairs not covered by each query's seed are inverted into
// per-cluster query lists (count, scan, fill), so the tensor-core pass reads each probed cluster
// once for every query that probes it: (cluster, group of up to qg queries) work items. Clusters
// that fewer than tmin queries probe give their pairs back to the ALU chunk scan instead.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

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

}  // namespace sg
