// cut.cu — the candidate cut and SOAR dedup of ivf::Index::candidates (src/ivf.rs:698-726).
//
// One CTA per query takes the best `cand` entries of the query's candidate buffer by
// (estimate desc, admission order asc) — cand.into_sorted() — then reads each slot's row id and
// error half-width and keeps, per row, the entry that comes first in (row asc, estimate desc,
// admission asc): sort_unstable_by(id, est total_cmp) + dedup_by_key(id). Output in row order.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

struct CutArgs {
  const uint4* cbuf;
  uint32_t cap;
  const uint32_t* ccount;
  const uint8_t* overflow;
  const uint32_t* ids;
  const float* err;
  uint32_t cand;
  float* cest;
  uint32_t* cid;
  float* cerr;
  uint32_t* cn;
};

__global__ void __launch_bounds__(1024) k_cut(CutArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* key = reinterpret_cast<uint64_t*>(smem_raw);           // [kMaxCand]
  uint32_t* pay = reinterpret_cast<uint32_t*>(key + kMaxCand);     // [kMaxCand]
  float* sest = reinterpret_cast<float*>(pay + kMaxCand);          // [kMaxCand]
  float* serr = sest + kMaxCand;                                   // [kMaxCand]
  uint32_t* sid = reinterpret_cast<uint32_t*>(serr + kMaxCand);    // [kMaxCand]
  __shared__ uint32_t hist[256], tmp[32], s_n;
  const uint32_t q = blockIdx.x;
  const uint32_t cand = a.cand;
  if (a.overflow[q]) {
    if (threadIdx.x == 0) a.cn[q] = 0;
    return;
  }
  const uint4* E = a.cbuf + (size_t)q * a.cap;
  const uint32_t M = min(a.ccount[q], a.cap);
  auto ordk = [&](uint32_t i) { return ord(__uint_as_float(E[i].x)); };
  uint32_t T = 0, Kt = 0;
  bool cut = M > cand;
  if (cut) {
    T = block_select_nth_u32(ordk, M, cand, hist);
    uint32_t gt = 0, eq = 0;
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
      uint32_t o = ordk(i);
      gt += o > T;
      eq += o == T;
    }
    uint32_t n_gt = block_sum(gt, tmp), n_eq = block_sum(eq, tmp);
    uint32_t need = cand - n_gt;
    if (n_eq > need) {
      // ties at the cut: the `need` earliest admitted of them
      Kt = block_select_nth_u32(
          [&](uint32_t i) { return ordk(i) == T ? 0xFFFFFFFFu - E[i].y : 0u; }, M, need, hist);
    } else {
      Kt = 0;
    }
  }
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
    uint4 e = E[i];
    uint32_t o = ord(__uint_as_float(e.x));
    bool sel = !cut || o > T || (o == T && 0xFFFFFFFFu - e.y >= Kt);
    if (sel) {
      uint32_t s = atomicAdd(&s_n, 1u);
      key[s] = ((uint64_t)o << 32) | (0xFFFFFFFFu - e.y);
      pay[s] = i;
    }
  }
  __syncthreads();
  const uint32_t n = s_n;
  const uint32_t n2 = next_pow2(n > 0 ? n : 1);
  for (uint32_t i = n + threadIdx.x; i < n2; i += blockDim.x) {
    key[i] = 0;
    pay[i] = 0;
  }
  __syncthreads();
  block_bitonic_sort_desc_kv(key, pay, n2);
  // rank p in (est desc, admission asc); now fetch row id and error of each slot
  for (uint32_t p = threadIdx.x; p < n; p += blockDim.x) {
    uint4 e = E[pay[p]];
    uint32_t id = a.ids[e.z];
    sest[p] = __uint_as_float(e.x);
    serr[p] = a.err[e.z];
    sid[p] = id;
    // ascending (id, p) as a descending sort of the complement
    key[p] = ~(((uint64_t)id << 32) | p);
    pay[p] = p;
  }
  for (uint32_t i = n + threadIdx.x; i < n2; i += blockDim.x) key[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc_kv(key, pay, n2);
  // keep the first entry of every row id (contiguous ranges per thread keep the order)
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t i0 = threadIdx.x * per, i1 = min(n, i0 + per);
  uint32_t keep = 0;
  for (uint32_t i = i0; i < i1; i++) {
    uint32_t id = (uint32_t)(~key[i] >> 32);
    uint32_t prev = i > 0 ? (uint32_t)(~key[i - 1] >> 32) : 0xFFFFFFFFu;
    keep += (i == 0 || id != prev);
  }
  uint32_t total;
  uint32_t off = block_exclusive_scan(keep, tmp, &total);
  for (uint32_t i = i0; i < i1; i++) {
    uint32_t id = (uint32_t)(~key[i] >> 32);
    uint32_t prev = i > 0 ? (uint32_t)(~key[i - 1] >> 32) : 0xFFFFFFFFu;
    if (i == 0 || id != prev) {
      uint32_t p = pay[i];
      size_t o = (size_t)q * cand + off++;
      a.cest[o] = sest[p];
      a.cid[o] = sid[p];
      a.cerr[o] = serr[p];
    }
  }
  if (threadIdx.x == 0) a.cn[q] = total;
}

void launch_cut(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                cudaStream_t st) {
  CutArgs a;
  a.cbuf = w.cbuf;
  a.cap = w.cbuf_per_q;
  a.ccount = w.ccount;
  a.overflow = w.overflow;
  a.ids = ix.ids;
  a.err = ix.err;
  a.cand = p.cand;
  a.cest = w.cest;
  a.cid = w.cid;
  a.cerr = w.cerr;
  a.cn = w.cn;
  static bool attr = false;
  size_t smem = (size_t)kMaxCand * (8 + 4 + 4 + 4 + 4);
  if (!attr) {
    cudaFuncSetAttribute(k_cut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  k_cut<<<nq, 1024, smem, st>>>(a);
}

}  // namespace sg
