// cut.cu — the candidate cut and SOAR dedup of ivf::Index::candidates (src/ivf.rs:698-726).
//
// One CTA per query takes the best `cand` entries of the query's candidate buffer by
// (estimate desc, admission order asc) — the set cand.into_sorted() keeps — then reads each
// slot's row id and keeps, per row, the entry first in (estimate desc, admission asc): the entry
// sort_unstable_by(id, est) + dedup_by_key(id) keeps. The list is left in an unspecified order
// (everything downstream is order-free); sg_candidates sorts it by row as the reference returns it.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

struct CutArgs {
  const uint32_t* cbuf_est;
  const uint2* cbuf_info;
  uint32_t cap;
  const uint32_t* ccount;
  const uint8_t* overflow;
  const uint32_t* ids;
  const float* err;
  uint32_t cand;
  const float4* qp;  // (scale, bias, a, b): global codes report lut.to_float(score)
  uint32_t global;   // global sign codes: the admission key is the row, copies differ by slot
  float* cest;
  uint32_t* cid;
  float* cerr;
  uint32_t* cn;
};

// Shared memory of one cut CTA (sized so two 1024-thread CTAs fit on an SM):
//   region K: the buffer's ordered estimates for the radix passes (buffers of up to kCutSmemKeys
//             entries; larger ones are read from global memory), later reused as the dedup
//             hash table (kHash row ids + kHash packed (estimate, admission) winners);
//   region S: the radix histogram (2048 words), later the selected entries' buffer indices.
constexpr uint32_t kHash = 8192;  // >= 2 x kMaxCand
constexpr uint32_t kCutSmemKeys = kHash * 3;  // 96 KB, the size of the hash table
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

SG_DEV uint32_t hash_row(uint32_t id) { return (id * 0x9E3779B1u) >> 19; }  // 13 bits = kHash

__global__ void __launch_bounds__(1024, 2) k_cut(CutArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* sk = reinterpret_cast<uint32_t*>(smem_raw);                 // region K: [kCutSmemKeys]
  uint32_t* h_id = reinterpret_cast<uint32_t*>(smem_raw);               // region K: [kHash]
  uint64_t* h_best = reinterpret_cast<uint64_t*>(h_id + kHash);         // region K: [kHash]
  uint32_t* hist = reinterpret_cast<uint32_t*>(smem_raw + kHash * 12);  // region S: [2048]
  uint32_t* sel = hist;                                                 // region S: [kMaxCand]
  __shared__ uint32_t tmp[32], s_n;
  const uint32_t q = blockIdx.x;
  const uint32_t cand = a.cand;
  if (a.overflow[q]) {
    if (threadIdx.x == 0) a.cn[q] = 0;
    return;
  }
  const uint32_t* Ee = a.cbuf_est + (size_t)q * a.cap;  // 16-byte aligned: cap % 4 == 0
  const uint2* Ei = a.cbuf_info + (size_t)q * a.cap;
  const uint32_t M = min(a.ccount[q], a.cap);
  const bool cut = M > cand;
  const bool in_smem = M <= kCutSmemKeys;
  if (cut && in_smem) {
    const uint4* E4 = reinterpret_cast<const uint4*>(Ee);
    for (uint32_t j = threadIdx.x; j < (M + 3) / 4; j += blockDim.x) {
      const uint4 v = __ldg(E4 + j);
      sk[4 * j] = ord(__uint_as_float(v.x));
      if (4 * j + 1 < M) sk[4 * j + 1] = ord(__uint_as_float(v.y));
      if (4 * j + 2 < M) sk[4 * j + 2] = ord(__uint_as_float(v.z));
      if (4 * j + 3 < M) sk[4 * j + 3] = ord(__uint_as_float(v.w));
    }
    __syncthreads();
  }
  auto ordk = [&](uint32_t i) { return in_smem ? sk[i] : ord(__uint_as_float(Ee[i])); };
  // ---- the best `cand` by (estimate desc, admission asc): threshold T, and among entries at T
  //      the admission keys up to ~Kt
  uint32_t T = 0, Kt = 0;
  if (cut) {
    T = block_select_nth_u32r(ordk, M, cand, hist, tmp);
    uint32_t gt = 0, eq = 0;
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
      const uint32_t o = ordk(i);
      gt += o > T;
      eq += o == T;
    }
    const uint32_t n_gt = block_sum(gt, tmp), n_eq = block_sum(eq, tmp);
    const uint32_t need = cand - n_gt;
    if (n_eq > need)
      Kt = block_select_nth_u32r(
          [&](uint32_t i) { return ordk(i) == T ? 0xFFFFFFFFu - Ei[i].x : 0u; }, M, need, hist, tmp);
  }
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
    bool take = true;
    if (cut) {
      const uint32_t o = ordk(i);
      take = o > T || (o == T && 0xFFFFFFFFu - Ei[i].x >= Kt);
    }
    if (take) sel[atomicAdd(&s_n, 1u)] = i;
  }
  __syncthreads();
  const uint32_t n = s_n;  // = min(M, cand)
  // ---- SOAR dedup: per row id keep the entry first in (estimate desc, admission asc) ---------
  for (uint32_t h = threadIdx.x; h < kHash; h += blockDim.x) {
    h_id[h] = kEmpty;
    h_best[h] = 0;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t i = sel[j];
    const uint2 info = Ei[i];
    const uint32_t id = a.ids[info.y];
    const uint64_t pack = ((uint64_t)ord(__uint_as_float(Ee[i])) << 32) |
                          (0xFFFFFFFFu - (a.global ? info.y : info.x));
    uint32_t h = hash_row(id);
    for (uint32_t probe = 0; probe < kHash; probe++) {
      const uint32_t prev = atomicCAS(&h_id[h], kEmpty, id);
      if (prev == kEmpty || prev == id) break;
      h = (h + 1) & (kHash - 1);
    }
    atomicMax(reinterpret_cast<unsigned long long*>(&h_best[h]), (unsigned long long)pack);
  }
  __syncthreads();
  // keep the winners, in contiguous ranges of j per thread (stable compaction)
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t j0 = threadIdx.x * per, j1 = min(n, j0 + per);
  uint32_t keep = 0;
  auto winner = [&](uint32_t j, uint32_t* id_out, uint32_t* slot_out) {
    const uint32_t i = sel[j];
    const uint2 info = Ei[i];
    const uint32_t id = a.ids[info.y];
    const uint64_t pack = ((uint64_t)ord(__uint_as_float(Ee[i])) << 32) |
                          (0xFFFFFFFFu - (a.global ? info.y : info.x));
    uint32_t h = hash_row(id);
    for (uint32_t probe = 0; probe < kHash && h_id[h] != id; probe++) h = (h + 1) & (kHash - 1);
    *id_out = id;
    *slot_out = info.y;
    return h_id[h] == id && h_best[h] == pack;
  };
  for (uint32_t j = j0; j < j1; j++) {
    uint32_t id, slot;
    keep += winner(j, &id, &slot);
  }
  uint32_t total;
  uint32_t off = block_exclusive_scan(keep, tmp, &total);
  for (uint32_t j = j0; j < j1; j++) {
    uint32_t id, slot;
    if (winner(j, &id, &slot)) {
      const size_t o = (size_t)q * cand + off++;
      const float e = __uint_as_float(Ee[sel[j]]);
      // Lut::to_float (src/lut.rs:62-64) of a global code's score
      a.cest[o] = a.global ? __fadd_rn(__fdiv_rn(e, a.qp[q].x), a.qp[q].y) : e;
      a.cid[o] = id;
      a.cerr[o] = a.err[slot];
    }
  }
  if (threadIdx.x == 0) a.cn[q] = total;
}

void launch_cut(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                cudaStream_t st) {
  CutArgs a;
  a.cbuf_est = w.cbuf_est;
  a.cbuf_info = w.cbuf_info;
  a.cap = w.cbuf_per_q;
  a.ccount = w.ccount;
  a.overflow = w.overflow;
  a.ids = ix.ids;
  a.err = ix.err;
  a.cand = p.cand;
  a.qp = w.qp;
  a.global = ix.global;
  a.cest = w.cest;
  a.cid = w.cid;
  a.cerr = w.cerr;
  a.cn = w.cn;
  static PerDeviceOnce attr;
  const size_t smem = (size_t)kHash * 12 + (size_t)kMaxCand * 4;
  attr([&] { return cudaFuncSetAttribute(k_cut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); });
  k_cut<<<nq, 1024, smem, st>>>(a);
}

}  // namespace sg
