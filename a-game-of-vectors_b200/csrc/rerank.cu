// rerank.cu — bound pruning, the 2-bit tier, the int8 rerank and the final top-k of
// ivf::Index::rerank (src/ivf.rs:734-832).
//
//   prune:   tau = m-th largest (est - w*err) by total_cmp; keep est + w*err >= tau (src/ivf.rs:543-550,
//            :736-739).
//   Full:    score = (dot_i8i8(wq, row) as f32) * inv over every candidate (src/ivf.rs:752-762).
//   Ssd(r):  best r by estimate, then Full over them (src/ivf.rs:763-768).
//   Tiered(r) with tier2: 2-bit table score (tier2::score, src/tier2.rs:69-75) of every candidate,
//            best r, then Full (src/ivf.rs:769-784, :819-832).
//   Prefix / Tiered without tier2: (dot256 as f32) * inv / norm256 of every candidate; Prefix
//            returns the best k, Tiered(r) takes the best r to Full (src/ivf.rs:785-811).
// Every top-n is the reference TopK order (score desc, id asc). Integer dots use dp4a and are
// exact; the float steps repeat the reference's operations.
#include "common.cuh"
#include "internal.hpp"

namespace sg {

// ---- prune: one CTA per query -------------------------------------------------------------
__global__ void __launch_bounds__(256) k_prune(const float* __restrict__ cest,
                                               const uint32_t* __restrict__ cid,
                                               const float* __restrict__ cerr,
                                               const uint32_t* __restrict__ cn, uint32_t cand,
                                               uint32_t has_prune, uint32_t m, float w,
                                               uint32_t* __restrict__ lid, float* __restrict__ lsc,
                                               uint32_t* __restrict__ ln) {
  __shared__ uint32_t hist[256], tmp[32];
  const uint32_t q = blockIdx.x, n = cn[q];
  const size_t o = (size_t)q * cand;
  float tau = -INFINITY;
  if (has_prune && m > 0 && n >= m) {
    uint32_t t = block_select_nth_u32(
        [&](uint32_t i) { return ord_total(__fsub_rn(cest[o + i], __fmul_rn(w, cerr[o + i]))); },
        n, m, hist);
    tau = unord(t);
    // ord_total keeps -0.0 apart from +0.0; unord gives back the exact f32 bits
  }
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t i0 = threadIdx.x * per, i1 = min(n, i0 + per);
  uint32_t keep = 0;
  for (uint32_t i = i0; i < i1; i++)
    keep += !has_prune || __fadd_rn(cest[o + i], __fmul_rn(w, cerr[o + i])) >= tau;
  uint32_t total;
  uint32_t off = block_exclusive_scan(keep, tmp, &total);
  for (uint32_t i = i0; i < i1; i++)
    if (!has_prune || __fadd_rn(cest[o + i], __fmul_rn(w, cerr[o + i])) >= tau) {
      lid[o + off] = cid[o + i];
      lsc[o + off] = cest[o + i];
      off++;
    }
  if (threadIdx.x == 0) ln[q] = total;
}

// ---- int8 dot scores of a list: 8 warps x 4 rows per CTA, dp4a ---------------------------
// mode 0: Full (768-d):  (dot as f32) * inv
// mode 1: Prefix (256-d): (dot as f32) * inv / norm256[id]
template <int MODE>
__global__ void __launch_bounds__(256) k_dot_list(const int8_t* __restrict__ rows,
                                                  const int8_t* __restrict__ wq_all,
                                                  const float* __restrict__ inv_all,
                                                  const float* __restrict__ norm256,
                                                  const uint32_t* __restrict__ lid,
                                                  const uint32_t* __restrict__ ln, uint32_t stride,
                                                  float* __restrict__ lsc) {
  constexpr int D = MODE == 0 ? SG_DIM : SG_PDIM;
  __shared__ __align__(16) int8_t wq[D];
  const uint32_t q = blockIdx.y, n = ln[q];
  const uint32_t j0 = blockIdx.x * 32;
  if (j0 >= n) return;
  for (int i = threadIdx.x; i < D / 16; i += blockDim.x)
    reinterpret_cast<int4*>(wq)[i] = reinterpret_cast<const int4*>(wq_all + (size_t)q * D)[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float inv = inv_all[q];
  // D/16 16-byte pieces per row: 48 (768) or 16 (256); lanes take pieces lane and lane+32
  int4 x[4][2];
  uint32_t id[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint32_t j = j0 + warp * 4 + r;
    id[r] = j < n ? lid[(size_t)q * stride + j] : 0xFFFFFFFFu;
    const int4* src = reinterpret_cast<const int4*>(rows + (size_t)(j < n ? id[r] : 0) * SG_DIM);
    x[r][0] = (j < n && lane < D / 16) ? __ldg(src + lane) : make_int4(0, 0, 0, 0);
    x[r][1] = (j < n && lane + 32 < D / 16) ? __ldg(src + lane + 32) : make_int4(0, 0, 0, 0);
  }
  const int4 w0 = lane < D / 16 ? reinterpret_cast<const int4*>(wq)[lane] : make_int4(0, 0, 0, 0);
  const int4 w1 =
      lane + 32 < D / 16 ? reinterpret_cast<const int4*>(wq)[lane + 32] : make_int4(0, 0, 0, 0);
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
    const uint32_t j = j0 + warp * 4 + r;
    if (lane == 0 && j < n) {
      float v = __fmul_rn((float)s, inv);
      if (MODE == 1) v = __fdiv_rn(v, norm256[id[r]]);
      lsc[(size_t)q * stride + j] = v;
    }
  }
}

// ---- 2-bit tier scores: tables in shared memory (64 x 256 f32), 128 candidates per CTA ------
__global__ void __launch_bounds__(256) k_tier2_list(const float* __restrict__ q256,
                                                    const float* __restrict__ sigma,
                                                    const uint8_t* __restrict__ codes,
                                                    const float* __restrict__ norms,
                                                    const uint32_t* __restrict__ lid,
                                                    const uint32_t* __restrict__ ln,
                                                    uint32_t stride, float* __restrict__ lsc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* tab = reinterpret_cast<float*>(smem_raw);   // [64][256]
  __shared__ float half[SG_TIER2_BYTES][2][16];
  const uint32_t q = blockIdx.y, n = ln[q];
  const uint32_t j0 = blockIdx.x * 128;
  if (j0 >= n) return;
  const float L[4] = {-1.510f, -0.4528f, 0.4528f, 1.510f};
  const float* qv = q256 + (size_t)q * SG_PDIM;
  for (int e = threadIdx.x; e < SG_TIER2_BYTES * 32; e += blockDim.x) {
    int g = e >> 5, h = (e >> 4) & 1, b = e & 15;
    int i0 = 4 * g + 2 * h, i1 = i0 + 1;
    float t0 = __fmul_rn(__fmul_rn(qv[i0], L[b & 3]), sigma[i0]);
    float t1 = __fmul_rn(__fmul_rn(qv[i1], L[(b >> 2) & 3]), sigma[i1]);
    half[g][h][b] = __fadd_rn(__fadd_rn(-0.0f, t0), t1);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < SG_TIER2_BYTES * 256; e += blockDim.x) {
    int g = e >> 8, b = e & 255;
    tab[e] = __fadd_rn(half[g][0][b & 15], half[g][1][b >> 4]);
  }
  __syncthreads();
  for (uint32_t j = j0 + threadIdx.x; j < min(n, j0 + 128); j += blockDim.x) {
    const uint32_t id = lid[(size_t)q * stride + j];
    const uint4* src = reinterpret_cast<const uint4*>(codes + (size_t)id * SG_TIER2_BYTES);
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int p = 0; p < 4; p++) {
      uint4 v = __ldg(src + p);
      uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int by = 0; by < 4; by++) {
          const int g = p * 16 + u * 4 + by;
          acc[g & 3] = __fadd_rn(acc[g & 3], tab[g * 256 + ((wv[u] >> (8 * by)) & 255)]);
        }
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[1]), acc[2]), acc[3]);
    lsc[(size_t)q * stride + j] = __fdiv_rn(s, norms[id]);
  }
}

// ---- top-n of a scored list by (score desc, id asc), sorted; one CTA per query ------------
__global__ void __launch_bounds__(1024) k_top_list(const float* __restrict__ sc,
                                                   const uint32_t* __restrict__ id,
                                                   const uint32_t* __restrict__ n_in,
                                                   uint64_t stride_in, uint64_t id_stride,
                                                   uint32_t nsel,
                                                   float* __restrict__ out_sc,
                                                   uint32_t* __restrict__ out_id,
                                                   uint32_t* __restrict__ n_out,
                                                   uint32_t stride_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* key = reinterpret_cast<uint64_t*>(smem_raw);  // [kMaxCand]
  __shared__ uint32_t hist[256], tmp[32], s_n;
  const uint32_t q = blockIdx.x, M = n_in[q];
  const float* S = sc + (size_t)q * stride_in;
  const uint32_t* I = id + (size_t)q * id_stride;
  uint64_t T = 0;
  const bool cut = M > nsel;
  if (cut && nsel > 0) {
    T = block_select_nth_u64([&](uint32_t i) { return rank_key(S[i], I[i]); }, M, nsel, hist, tmp);
  }
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  if (nsel > 0)
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
      uint64_t k = rank_key(S[i], I[i]);
      if (!cut || k >= T) key[atomicAdd(&s_n, 1u)] = k;
    }
  __syncthreads();
  const uint32_t n = s_n;
  const uint32_t n2 = next_pow2(n > 0 ? n : 1);
  for (uint32_t i = n + threadIdx.x; i < n2; i += blockDim.x) key[i] = 0;
  __syncthreads();
  block_bitonic_sort_desc(key, n2);
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    out_sc[(size_t)q * stride_out + i] = key_score(key[i]);
    out_id[(size_t)q * stride_out + i] = key_id(key[i]);
  }
  if (threadIdx.x == 0) n_out[q] = n;
}

void launch_top_list(const float* sc, const uint32_t* id, const uint32_t* n_in, uint64_t sc_stride,
                     uint64_t id_stride, uint32_t nsel, float* out_sc, uint32_t* out_id,
                     uint32_t* n_out, uint32_t stride_out, uint32_t nq, cudaStream_t st) {
  static PerDeviceOnce attr;
  const size_t smem = (size_t)kMaxCand * 8;
  attr([&] { return cudaFuncSetAttribute(k_top_list, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); });
  k_top_list<<<nq, 1024, smem, st>>>(sc, id, n_in, sc_stride, id_stride, nsel, out_sc, out_id,
                                     n_out, stride_out);
}

static void top_list(const float* sc, const uint32_t* id, const uint32_t* n_in, uint32_t stride_in,
                     uint32_t nsel, float* out_sc, uint32_t* out_id, uint32_t* n_out,
                     uint32_t stride_out, uint32_t nq, cudaStream_t st) {
  launch_top_list(sc, id, n_in, stride_in, stride_in, nsel, out_sc, out_id, n_out, stride_out, nq,
                  st);
}

static void dot_list(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t stride, bool prefix,
                     cudaStream_t st) {
  dim3 grid((stride + 31) / 32, nq);
  if (prefix)
    k_dot_list<1><<<grid, 256, 0, st>>>(ix.rerank, w.wq256, w.winv256, ix.norm256, w.lid, w.ln,
                                        stride, w.lsc);
  else
    k_dot_list<0><<<grid, 256, 0, st>>>(ix.rerank, w.wq, w.winv, ix.norm256, w.lid, w.ln, stride,
                                        w.lsc);
}

int launch_rerank(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                  cudaStream_t st, cudaEvent_t ev_t2_begin, cudaEvent_t ev_t2_end) {
  const uint32_t stride = p.cand;
  int launches = 0;
  k_prune<<<nq, 256, 0, st>>>(w.cest, w.cid, w.cerr, w.cn, stride, p.has_prune, p.prune_m,
                              p.prune_w, w.lid, w.lsc, w.ln);
  launches++;
  int kind = (int)p.rerank_kind;
  if (ev_t2_begin) cudaEventRecord(ev_t2_begin, st);
  if (kind == SG_RERANK_NONE) {
    // estimates are the scores
  } else if (kind == SG_RERANK_FULL) {
    dot_list(ix, w, nq, stride, false, st);
    launches++;
  } else if (kind == SG_RERANK_SSD) {
    top_list(w.lsc, w.lid, w.ln, stride, p.rerank_r, w.lsc, w.lid, w.ln, stride, nq, st);
    dot_list(ix, w, nq, stride, false, st);
    launches += 2;
  } else if (kind == SG_RERANK_TIERED && ix.has_t2) {
    static PerDeviceOnce attr;
    const size_t smem = (size_t)SG_TIER2_BYTES * 256 * sizeof(float);
    attr([&] {
      return cudaFuncSetAttribute(k_tier2_list, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    dim3 grid((stride + 127) / 128, nq);
    k_tier2_list<<<grid, 256, smem, st>>>(w.q256, ix.t2_sigma, ix.t2_codes, ix.t2_norm, w.lid,
                                          w.ln, stride, w.lsc);
    top_list(w.lsc, w.lid, w.ln, stride, p.rerank_r, w.lsc, w.lid, w.ln, stride, nq, st);
    if (ev_t2_end) cudaEventRecord(ev_t2_end, st);
    dot_list(ix, w, nq, stride, false, st);
    launches += 3;
  } else {  // Prefix, or Tiered without a tier-2 file
    dot_list(ix, w, nq, stride, true, st);
    launches++;
    if (kind == SG_RERANK_TIERED) {
      top_list(w.lsc, w.lid, w.ln, stride, p.rerank_r, w.lsc, w.lid, w.ln, stride, nq, st);
      if (ev_t2_end) cudaEventRecord(ev_t2_end, st);
      dot_list(ix, w, nq, stride, false, st);
      launches += 2;
    }
  }
  if (ev_t2_end && kind != SG_RERANK_TIERED) cudaEventRecord(ev_t2_end, st);
  top_list(w.lsc, w.lid, w.ln, stride, p.k, w.out_sc, w.out_id, w.out_n, p.k, nq, st);
  return launches + 1;
}

// ---- stateless int8 dots for the parity tests --------------------------------------------------
__global__ void k_dot_rows(const int8_t* __restrict__ q, const int8_t* __restrict__ rows,
                           uint64_t nrows, uint32_t dim, int32_t* __restrict__ out) {
  const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nrows) return;
  const int8_t* x = rows + r * dim;
  int s = 0;
  for (uint32_t i = 4 * lane; i < dim; i += 128) {
    int a = *reinterpret_cast<const int*>(q + i);
    int b = *reinterpret_cast<const int*>(x + i);
    s = __dp4a(a, b, s);
  }
  s = warp_sum_i(s);
  if (lane == 0) out[r] = s;
}

void launch_dot_i8i8(const int8_t* q, const int8_t* rows, uint64_t nrows, uint32_t dim,
                     int32_t* out, cudaStream_t st) {
  if (nrows == 0) return;
  k_dot_rows<<<(unsigned)((nrows * 32 + 255) / 256), 256, 0, st>>>(q, rows, nrows, dim, out);
}

}  // namespace sg
