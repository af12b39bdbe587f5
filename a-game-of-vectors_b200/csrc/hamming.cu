// hamming.cu — the flat Hamming baseline of the reference's search binary
// (flat_hamming_rerank, src/bin/search.rs:251-269): no index, every row's global sign code
// (codes.bin) scored against the query's sign code by 256 - Hamming distance (lut::hamming,
// src/lut.rs:156-165), the best `cand` rows kept (TopK by (score desc, row asc)), then reranked
// by the float-weight int8 dot quant::dot_i8 (src/quant.rs:72-84) with the query weights
// Int8Quantizer::query_weights (src/quant.rs:64-67) into the top k.
//
// One CTA per query (1024 threads) scans every code twice: a 257-bin histogram of the scores
// gives the cand-th score T and how many rows tied at T fit; the second pass keeps every row
// above T and the lowest-numbered rows at T (a block-wide scan over rows in ascending order),
// so the kept set is exactly the first `cand` rows in (score desc, row asc).
#include "common.cuh"
#include "internal.hpp"

namespace sg {

__global__ void __launch_bounds__(1024) k_hamming_select(const uint4* __restrict__ codes, uint64_t n,
                                                         const float* __restrict__ q256, uint32_t cand,
                                                         uint32_t* __restrict__ lid, uint32_t* __restrict__ ln,
                                                         uint32_t stride) {
  __shared__ uint32_t qc[8];
  __shared__ uint32_t hist[SG_PDIM + 1];
  __shared__ uint32_t tmp[32], s_T, s_need, s_n;
  const uint32_t q = blockIdx.x, tid = threadIdx.x;
  // sign_code (src/quant.rs:24-32): bit i set where the prefix is positive
  if (tid < 8) qc[tid] = 0;
  for (uint32_t i = tid; i <= SG_PDIM; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  if (tid < SG_PDIM && q256[(size_t)q * SG_PDIM + tid] > 0.0f) atomicOr(&qc[tid >> 5], 1u << (tid & 31));
  __syncthreads();
  const uint32_t c0 = qc[0], c1 = qc[1], c2 = qc[2], c3 = qc[3], c4 = qc[4], c5 = qc[5], c6 = qc[6], c7 = qc[7];
  auto score = [&](uint64_t r) {
    const uint4 a = __ldg(codes + 2 * r), b = __ldg(codes + 2 * r + 1);
    const uint32_t d = __popc(a.x ^ c0) + __popc(a.y ^ c1) + __popc(a.z ^ c2) + __popc(a.w ^ c3) +
                       __popc(b.x ^ c4) + __popc(b.y ^ c5) + __popc(b.z ^ c6) + __popc(b.w ^ c7);
    return (uint32_t)SG_PDIM - d;
  };
  for (uint64_t r = tid; r < n; r += blockDim.x) atomicAdd(&hist[score(r)], 1u);
  __syncthreads();
  if (tid == 0) {
    uint32_t cum = 0, T = 0, need = 0;
    bool found = false;
    for (int s = SG_PDIM; s >= 0 && !found; s--) {
      if (cum + hist[s] >= cand) {
        T = (uint32_t)s;
        need = cand - cum;
        found = true;
      } else {
        cum += hist[s];
      }
    }
    if (!found) {  // fewer rows than cand: every row
      T = 0;
      need = hist[0];
    }
    s_T = T;
    s_need = need;
    s_n = 0;
  }
  __syncthreads();
  const uint32_t T = s_T, need = s_need;
  uint32_t* out = lid + (size_t)q * stride;
  uint32_t ties_before = 0;  // rows at T in earlier tiles
  for (uint64_t base = 0; base < n; base += blockDim.x) {
    const uint64_t r = base + tid;
    uint32_t s = 0;
    if (r < n) s = score(r);
    const uint32_t eq = r < n && s == T;
    uint32_t tot;
    const uint32_t rank = ties_before + block_exclusive_scan(eq, tmp, &tot);
    if (r < n && (s > T || (eq && rank < need))) out[atomicAdd(&s_n, 1u)] = (uint32_t)r;
    ties_before += tot;
  }
  __syncthreads();
  if (tid == 0) ln[q] = s_n;
}

// quant::dot_i8 of each kept row with w = q768 / quant_scale: sixteen running sums over the
// 16-wide chunks, added in order from -0.0 (src/quant.rs:72-84); one thread per row.
__global__ void __launch_bounds__(256) k_dot_i8_weights(const int8_t* __restrict__ rows,
                                                        const float* __restrict__ q768,
                                                        const float* __restrict__ qscale,
                                                        const uint32_t* __restrict__ lid,
                                                        const uint32_t* __restrict__ ln, uint32_t stride,
                                                        float* __restrict__ lsc) {
  __shared__ float w[SG_DIM];
  const uint32_t q = blockIdx.x;
  for (uint32_t i = threadIdx.x; i < SG_DIM; i += blockDim.x)
    w[i] = __fdiv_rn(q768[(size_t)q * SG_DIM + i], qscale[i]);
  __syncthreads();
  const uint32_t n = ln[q];
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint4* x = reinterpret_cast<const uint4*>(rows + (size_t)lid[(size_t)q * stride + j] * SG_DIM);
    float acc[16];
#pragma unroll
    for (int i = 0; i < 16; i++) acc[i] = 0.0f;
    for (int c = 0; c < SG_DIM / 16; c++) {
      const uint4 v = __ldg(x + c);
      const uint32_t wd[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const float xi = (float)(int8_t)((wd[i >> 2] >> (8 * (i & 3))) & 0xFFu);
        acc[i] = __fadd_rn(acc[i], __fmul_rn(w[16 * c + i], xi));
      }
    }
    float s = -0.0f;
#pragma unroll
    for (int i = 0; i < 16; i++) s = __fadd_rn(s, acc[i]);
    lsc[(size_t)q * stride + j] = __fadd_rn(s, -0.0f);  // + the empty tail (768 = 48 x 16)
  }
}

// The baseline for the nq queries staged in w (q768, q256): the kept rows in w.lid / w.ln
// (stride cand), their dot scores in w.lsc, the top k in w.out_* (stride k). Returns the
// kernels launched.
int launch_flat_hamming(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t cand, uint32_t k,
                        cudaStream_t st) {
  k_hamming_select<<<nq, 1024, 0, st>>>(reinterpret_cast<const uint4*>(ix.codes), ix.n, w.q256, cand, w.lid,
                                        w.ln, cand);
  k_dot_i8_weights<<<nq, 256, 0, st>>>(ix.rerank, w.q768, ix.qscale, w.lid, w.ln, cand, w.lsc);
  launch_top_list(w.lsc, w.lid, w.ln, cand, cand, k, w.out_sc, w.out_id, w.out_n, k, nq, st);
  return 3;
}

}  // namespace sg
