// prep.cu — per-query preparation, one CTA per query (built with -fmad=false).
//
// rabitq::Query::new (src/rabitq.rs:119-125): rotate q256 (3 rounds of sign flips + FWHT, then
// d^-1.5; src/rabitq.rs:60-84), Lut::new over the rotated vector (src/lut.rs:33-55), then
// a = 2/scale and b = 2*bias - sum(qr). Also the rerank weights of query_i8 (src/quant.rs:104-110)
// over w = q/scale for the full 768-d query (Rerank::Full, src/ivf.rs:753-755) and the 256-d
// prefix (Rerank::Prefix, src/ivf.rs:786-788). Every float operation is the reference's, in the
// reference's order: sequential sums run in one thread from -0.0, products are rounded before
// they are added (no FMA), divisions are IEEE.
#include <float.h>

#include "internal.hpp"

namespace sg {

__global__ void __launch_bounds__(256) k_prep(const float* __restrict__ q256,
                                              const float* __restrict__ q768,
                                              const float* __restrict__ signs, float rot_norm,
                                              const float* __restrict__ qscale,
                                              uint8_t* __restrict__ tables, float4* __restrict__ qp,
                                              float* __restrict__ qnorm, int8_t* __restrict__ wq,
                                              float* __restrict__ winv, int8_t* __restrict__ wq256,
                                              float* __restrict__ winv256) {
  __shared__ float v[SG_PDIM];
  __shared__ float f[SG_GROUPS * 16];
  __shared__ float mins[SG_GROUPS], maxs[SG_GROUPS];
  __shared__ float red[32];
  __shared__ float s_scale;
  const int q = blockIdx.x, t = threadIdx.x;
  const float* x = q256 + (size_t)q * SG_PDIM;
  v[t] = x[t];
  __syncthreads();
  // ||q256|| (any order): the routing error window scales with it.
  if (t < 32) {
    float s = 0.0f;
    for (int i = t; i < SG_PDIM; i += 32) s = __fadd_rn(s, __fmul_rn(v[i], v[i]));
    for (int o = 16; o > 0; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xFFFFFFFFu, s, o));
    if (t == 0) qnorm[q] = sqrtf(s);
  }
  // Rotation::apply: three rounds of sign flip + FWHT, then the d^-1.5 scale. Global sign codes
  // (no rotation) take the LUT of the prefix itself (src/ivf.rs:701).
  for (int r = 0; signs && r < 3; r++) {
    v[t] = __fmul_rn(v[t], signs[r * SG_PDIM + t]);
    __syncthreads();
    for (int h = 1; h < SG_PDIM; h *= 2) {
      if (t < SG_PDIM / 2) {
        int blk = t / h, i = t % h;
        int a = blk * 2 * h + i, b = a + h;
        float xa = v[a], yb = v[b];
        v[a] = __fadd_rn(xa, yb);
        v[b] = __fsub_rn(xa, yb);
      }
      __syncthreads();
    }
  }
  if (signs) v[t] = __fmul_rn(v[t], rot_norm);
  __syncthreads();
  // Lut::new: entry (g, c) sums q[4g + j] over the set bits j of c, ascending, from -0.0.
  for (int e = t; e < SG_GROUPS * 16; e += blockDim.x) {
    int g = e >> 4, c = e & 15;
    float s = -0.0f;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if ((c >> j) & 1) s = __fadd_rn(s, v[4 * g + j]);
    f[e] = s;
  }
  __syncthreads();
  if (t < SG_GROUPS) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int c = 0; c < 16; c++) {
      mn = fminf(mn, f[t * 16 + c]);
      mx = fmaxf(mx, f[t * 16 + c]);
    }
    mins[t] = mn;
    maxs[t] = mx;
  }
  __syncthreads();
  if (t == 0) {
    float max_range = 0.0f;
    for (int g = 0; g < SG_GROUPS; g++) max_range = fmaxf(max_range, __fsub_rn(maxs[g], mins[g]));
    float scale = max_range > 0.0f ? __fdiv_rn(255.0f, max_range) : 1.0f;
    float bias = -0.0f;
    for (int g = 0; g < SG_GROUPS; g++) bias = __fadd_rn(bias, mins[g]);
    float sum = -0.0f;
    for (int i = 0; i < SG_PDIM; i++) sum = __fadd_rn(sum, v[i]);
    float a = __fdiv_rn(2.0f, scale);
    float b = __fsub_rn(__fmul_rn(2.0f, bias), sum);
    // global sign codes rank by the LUT score itself: est = 0 + 1 * (1 * s + 0) = s exactly
    if (!signs) {
      a = 1.0f;
      b = 0.0f;
    }
    qp[q] = make_float4(scale, bias, a, b);
    s_scale = scale;
  }
  __syncthreads();
  const float scale = s_scale;
  uint8_t* tq = tables + (size_t)q * SG_GROUPS * 16;
  for (int e = t; e < SG_GROUPS * 16; e += blockDim.x) {
    float r = roundf(__fmul_rn(__fsub_rn(f[e], mins[e >> 4]), scale));
    r = fminf(fmaxf(r, 0.0f), 255.0f);
    tq[e] = (uint8_t)r;
  }
  // query_i8 over w = q / quant_scale: full 768-d query, then the 256-d prefix.
  const float* y = q768 + (size_t)q * SG_DIM;
  for (int pass = 0; pass < 2; pass++) {
    const int n = pass == 0 ? SG_DIM : SG_PDIM;
    const float* src = pass == 0 ? y : x;
    float m = 1e-12f;
    for (int i = t; i < n; i += blockDim.x) m = fmaxf(m, fabsf(__fdiv_rn(src[i], qscale[i])));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((t & 31) == 0) red[t >> 5] = m;
    __syncthreads();
    if (t == 0) {
      float mm = 1e-12f;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) mm = fmaxf(mm, red[i]);
      red[31] = mm;
    }
    __syncthreads();
    const float s = __fdiv_rn(127.0f, red[31]);
    int8_t* out = pass == 0 ? wq + (size_t)q * SG_DIM : wq256 + (size_t)q * SG_PDIM;
    for (int i = t; i < n; i += blockDim.x) {
      float r = roundf(__fmul_rn(__fdiv_rn(src[i], qscale[i]), s));
      r = fminf(fmaxf(r, -128.0f), 127.0f);  // Rust `as i8` saturates
      out[i] = (int8_t)(int)r;
    }
    if (t == 0) (pass == 0 ? winv : winv256)[q] = __fdiv_rn(1.0f, s);
    __syncthreads();
  }
}

// quant::prefix (src/quant.rs:17-20) for queries given without q256: copy the first 256 dims
// of the unit 768-d query and normalize (sequential sum of squares from -0.0, then * 1/n).
__global__ void k_prefix(const float* __restrict__ q768, float* __restrict__ q256) {
  __shared__ float s_inv;
  const int q = blockIdx.x, t = threadIdx.x;
  const float* x = q768 + (size_t)q * SG_DIM;
  if (t == 0) {
    float s = -0.0f;
    for (int i = 0; i < SG_PDIM; i++) s = __fadd_rn(s, __fmul_rn(x[i], x[i]));
    float n = sqrtf(s);
    s_inv = n > 0.0f ? __fdiv_rn(1.0f, n) : 1.0f;
  }
  __syncthreads();
  q256[(size_t)q * SG_PDIM + t] = __fmul_rn(x[t], s_inv);
}

void launch_prep(const DevIndex& ix, Workspace& w, uint32_t nq, cudaStream_t st) {
  k_prep<<<nq, 256, 0, st>>>(w.q256, w.q768, ix.rot, ix.rot_norm, ix.qscale, w.tables, w.qp,
                             w.qnorm, w.wq, w.winv, w.wq256, w.winv256);
}

void launch_prefix(Workspace& w, uint32_t nq, cudaStream_t st) {
  k_prefix<<<nq, SG_PDIM, 0, st>>>(w.q768, w.q256);
}

}  // namespace sg
