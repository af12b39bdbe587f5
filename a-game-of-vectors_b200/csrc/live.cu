// live.cu — inserts, deletes and upserts over an index on the GPU (ivf live updates,
// src/live.rs), without a rebuild.
//
// The built index stays as it is in HBM. An inserted row is encoded on the device exactly as
// Live::apply_insert encodes it (src/live.rs:318-350): the int8 rerank row, its prefix norm, the
// normalised prefix of the int8 row, its nearest centroid and (with SOAR) its secondary among the
// 16 nearest, RaBitQ residual codes of the rotated prefix against each rotated centroid, and the
// 2-bit tier code. Its rerank row and tier code are written at row id n + j of the index's row
// arrays (grown at open), so the rerank reads delta rows where it reads corpus rows. Its slots go
// to per-centroid delta lists in the base block layout (DeltaList, src/live.rs:39-66): cluster
// kc + c of the live index is centroid c's delta list, and routing scans it right after c's base
// list (route.cu, expand_delta), as Index::candidates scans a view's delta list after each base
// list (src/ivf.rs:682-684). Delta lists are repacked into the index's spare blocks after every
// insert call. Deletes set tombstones: the search's allow bitset is every live row, so a deleted
// row is skipped at admission (View::hidden, src/ivf.rs:474-483). Results carry external ids:
// a corpus row's is its row, a delta row's the id it was inserted under; inserting an id that is
// live replaces it (an upsert tombstones the old row).
//
// The write-ahead log, its replay and compaction (src/live.rs:131-249, :398-468) are host file
// I/O of the reference's server and are not part of the device path.
#include <cfloat>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace sg {

constexpr float kT2T = 0.9816f;  // tier2: T (src/tier2.rs:9-11)
__constant__ float kT2Levels[4] = {-1.510f, -0.4528f, 0.4528f, 1.510f};

// Rotation::apply (src/rabitq.rs:60-69) of v[256] in shared memory by all 256 threads.
SG_DEV void rotate256(float* v, const float* __restrict__ signs, float norm) {
  const int t = threadIdx.x;
  for (int r = 0; r < 3; r++) {
    v[t] = __fmul_rn(v[t], signs[r * SG_PDIM + t]);
    __syncthreads();
    for (int h = 1; h < SG_PDIM; h *= 2) {
      if (t < SG_PDIM / 2) {
        const int blk = t / h, i = t % h;
        const int a = blk * 2 * h + i, b = a + h;
        const float x = v[a], y = v[b];
        v[a] = __fadd_rn(x, y);
        v[b] = __fsub_rn(x, y);
      }
      __syncthreads();
    }
  }
  v[t] = __fmul_rn(v[t], norm);
  __syncthreads();
}

// quant::dot_f32 (src/quant.rs:86-100): sixteen running sums over 16-wide chunks, added in order.
SG_DEV float dot16(const float* a, const float* __restrict__ b) {
  float acc[16];
#pragma unroll
  for (int i = 0; i < 16; i++) acc[i] = 0.0f;
  for (int c = 0; c < SG_PDIM; c += 16)
#pragma unroll
    for (int i = 0; i < 16; i++) acc[i] = __fadd_rn(acc[i], __fmul_rn(a[c + i], b[c + i]));
  float s = -0.0f;
#pragma unroll
  for (int i = 0; i < 16; i++) s = __fadd_rn(s, acc[i]);
  return __fadd_rn(s, -0.0f);
}

// The reference's sequential f32 dot (blas::gemm_abt portable, src/blas.rs:46-52).
SG_DEV float seq_dot(const float* a, const float* __restrict__ b) {
  float s = -0.0f;
  for (int i = 0; i < SG_PDIM; i++) s = __fadd_rn(s, __fmul_rn(a[i], b[i]));
  return s;
}

__global__ void __launch_bounds__(256) k_rotate_rows(const float* __restrict__ in, const float* __restrict__ signs,
                                                     float norm, float* __restrict__ out) {
  __shared__ float v[SG_PDIM];
  const size_t r = blockIdx.x;
  v[threadIdx.x] = in[r * SG_PDIM + threadIdx.x];
  __syncthreads();
  rotate256(v, signs, norm);
  out[r * SG_PDIM + threadIdx.x] = v[threadIdx.x];
}

struct EncodeArgs {
  const float* vecs;  // [m * 768] unit vectors
  const float* qscale;
  const float* cent;  // [kc * 256]
  const float* cents_rot;
  uint32_t kc;
  const float* signs;
  float rot_norm;
  const float* t2_sigma;  // null: no 2-bit tier
  int soar;
  float lambda;
  float* scores;          // [m * kc] scratch
  int8_t* rows;           // rerank rows of the new ids [m * 768]
  float* norm256;         // [m] (null: the index keeps none)
  uint8_t* t2;            // [m * 64]
  float* t2_norm;         // [m]
  uint32_t* pair;         // [m * 2]
  uint8_t* codes;         // [m * 2 * 32]
  float* factors;         // [m * 2 * 2]
};

// One CTA of 256 threads per inserted row.
__global__ void __launch_bounds__(256) k_live_encode(EncodeArgs a) {
  __shared__ float v[SG_DIM];
  __shared__ float x[SG_PDIM], xr[SG_PDIM];
  __shared__ uint64_t keys[16];
  __shared__ uint32_t hist[256], tmp[32], s_m;
  __shared__ float s_loss[16], s_xc1, s_r2, s_rx;
  __shared__ uint32_t s_pair[2];
  const uint32_t j = blockIdx.x, t = threadIdx.x;
  for (uint32_t i = t; i < SG_DIM; i += blockDim.x) v[i] = a.vecs[(size_t)j * SG_DIM + i];
  __syncthreads();
  // Int8Quantizer::encode (src/quant.rs:52-56), and the row's prefix over its scale
  for (uint32_t i = t; i < SG_DIM; i += blockDim.x) {
    const float r = fminf(fmaxf(roundf(__fmul_rn(v[i], a.qscale[i])), -127.0f), 127.0f);
    a.rows[(size_t)j * SG_DIM + i] = (int8_t)(int)r;
    if (i < SG_PDIM) x[i] = __fdiv_rn(r, a.qscale[i]);
  }
  __syncthreads();
  if (t == 0) {
    // the prefix norm of the unit vector (src/live.rs:280), then quant::normalize of the prefix
    float nn = -0.0f;
    for (int i = 0; i < SG_PDIM; i++) nn = __fadd_rn(nn, __fmul_rn(v[i], v[i]));
    if (a.norm256) a.norm256[j] = sqrtf(nn);
    float s = -0.0f;
    for (int i = 0; i < SG_PDIM; i++) s = __fadd_rn(s, __fmul_rn(x[i], x[i]));
    const float n = sqrtf(s);
    s_m = 0;
    s_xc1 = n > 0.0f ? __fdiv_rn(1.0f, n) : 0.0f;
    s_rx = n > 0.0f ? 1.0f : 0.0f;
  }
  __syncthreads();
  if (s_rx != 0.0f) x[t] = __fmul_rn(x[t], s_xc1);
  __syncthreads();
  // assign_top (src/ivf.rs:138-158): the centroid scores, then TopK(16) or the first maximum
  float* row = a.scores + (size_t)j * a.kc;
  for (uint32_t c = t; c < a.kc; c += blockDim.x) row[c] = seq_dot(x, a.cent + (size_t)c * SG_PDIM);
  __syncthreads();
  const uint32_t m = a.soar ? min(16u, a.kc) : 1u;
  const uint64_t T = block_select_nth_u64([&](uint32_t c) { return rank_key(row[c], c); }, a.kc, m, hist, tmp);
  for (uint32_t c = t; c < a.kc; c += blockDim.x) {
    const uint64_t k = rank_key(row[c], c);
    if (k >= T) keys[atomicAdd(&s_m, 1u)] = k;
  }
  __syncthreads();
  if (t == 0) {  // the m winners best first (insertion sort of at most 16)
    for (uint32_t i = 1; i < m; i++) {
      const uint64_t k = keys[i];
      uint32_t p = i;
      while (p > 0 && keys[p - 1] < k) {
        keys[p] = keys[p - 1];
        p--;
      }
      keys[p] = k;
    }
    for (uint32_t i = m; i < 16; i++) keys[i] = rank_key(0.0f, 0);  // cluster 0, as assign_top leaves
    s_pair[0] = key_id(keys[0]);
    s_pair[1] = SG_PAD;
  }
  __syncthreads();
  if (a.soar) {
    // soar_secondary (src/ivf.rs:168-186) over candidates 1..15
    const float* c1 = a.cent + (size_t)key_id(keys[0]) * SG_PDIM;
    if (t == 0) {
      s_xc1 = dot16(x, c1);
      s_r2 = fmaxf(__fsub_rn(2.0f, __fmul_rn(2.0f, s_xc1)), 1e-12f);
      s_rx = __fsub_rn(1.0f, s_xc1);
    }
    __syncthreads();
    if (t >= 1 && t < 16) {
      const float* cv = a.cent + (size_t)key_id(keys[t]) * SG_PDIM;
      const float x_c = dot16(x, cv);
      const float r_c = __fsub_rn(x_c, dot16(c1, cv));
      const float along = __fsub_rn(s_rx, r_c);
      s_loss[t] = __fadd_rn(__fsub_rn(2.0f, __fmul_rn(2.0f, x_c)),
                            __fdiv_rn(__fmul_rn(__fmul_rn(a.lambda, along), along), s_r2));
    }
    __syncthreads();
    if (t == 0) {
      float best = FLT_MAX;
      uint32_t best_c = key_id(keys[1]);
      for (int i = 1; i < 16; i++)
        if (s_loss[i] < best) {
          best = s_loss[i];
          best_c = key_id(keys[i]);
        }
      s_pair[1] = best_c;
    }
    __syncthreads();
  }
  // the rotated prefix, and rabitq::encode against each assigned centroid (src/rabitq.rs:88-108)
  xr[t] = x[t];
  __syncthreads();
  rotate256(xr, a.signs, a.rot_norm);
  if (t < 2) {
    const uint32_t c = s_pair[t];
    uint8_t* code = a.codes + ((size_t)j * 2 + t) * SG_CODE_BYTES;
    float* f = a.factors + ((size_t)j * 2 + t) * 2;
    a.pair[(size_t)j * 2 + t] = c;
    uint8_t bytes[SG_CODE_BYTES];
    for (int i = 0; i < SG_CODE_BYTES; i++) bytes[i] = 0;
    float nr2 = 0.0f, l1 = 0.0f;
    if (c != SG_PAD) {
      const float* cr = a.cents_rot + (size_t)c * SG_PDIM;
      for (int i = 0; i < SG_PDIM; i++) {
        const float r = __fsub_rn(xr[i], cr[i]);
        nr2 = __fadd_rn(nr2, __fmul_rn(r, r));
        l1 = __fadd_rn(l1, fabsf(r));
        if (r > 0.0f) bytes[i >> 3] |= (uint8_t)(1u << (i & 7));
      }
    }
    for (int i = 0; i < SG_CODE_BYTES; i++) code[i] = bytes[i];
    if (c == SG_PAD || l1 < 1e-12f) {
      f[0] = 0.0f;
      f[1] = 0.0f;
    } else {
      const float df = (float)SG_PDIM;
      const float nr = sqrtf(nr2);
      const float od = __fdiv_rn(l1, __fmul_rn(nr, sqrtf(df)));
      const float od2 = __fmul_rn(od, od);
      const float inner = __fdiv_rn(__fsub_rn(1.0f, od2), __fmul_rn(od2, __fsub_rn(df, 1.0f)));
      f[0] = __fdiv_rn(nr2, l1);
      f[1] = __fmul_rn(__fmul_rn(nr, 1.9f), sqrtf(fmaxf(inner, 0.0f)));
    }
  } else if (t == 2 && a.t2_sigma) {
    // Tier2::encode (src/tier2.rs:42-48)
    uint8_t* out = a.t2 + (size_t)j * SG_TIER2_BYTES;
    float nn = 0.0f;
    uint8_t cur = 0;
    for (int i = 0; i < SG_PDIM; i++) {
      const float s = a.t2_sigma[i], th = __fmul_rn(kT2T, s), xi = x[i];
      const uint32_t l = xi < -th ? 0u : xi < 0.0f ? 1u : xi < th ? 2u : 3u;
      cur |= (uint8_t)(l << ((i & 3) * 2));
      if ((i & 3) == 3) {
        out[i >> 2] = cur;
        cur = 0;
      }
      const float lv = __fmul_rn(kT2Levels[l], s);
      nn = __fadd_rn(nn, __fmul_rn(lv, lv));
    }
    a.t2_norm[j] = sqrtf(nn);
  }
}

}  // namespace sg

using sg::fail;

// A live index: the device side lives in the index (its delta clusters, rows and spare blocks);
// this is the host bookkeeping of Live (src/live.rs:151-163).
struct sg_live {
  struct Slot {
    uint8_t code[SG_CODE_BYTES];
    float mul, err;
    uint32_t id;
  };
  sg_index* h = nullptr;
  uint64_t n = 0;         // corpus rows (the first delta row's id)
  uint64_t max_rows = 0;  // delta rows the index has room for
  uint64_t rows = 0;      // delta rows inserted
  uint64_t block_cap = 0;
  bool soar = false;
  float lambda = 0.0f;
  float* cents_rot = nullptr;  // [kc * 256] device
  uint64_t* alive = nullptr;   // device bitset over n + max_rows rows: live rows
  uint64_t words = 0;
  std::vector<std::vector<Slot>> lists;  // per centroid: its delta list
  std::vector<uint64_t> deleted;         // tombstones over row ids
  std::vector<uint32_t> ext;             // external id of each delta row
  std::unordered_map<uint32_t, uint32_t> by_ext;  // external id -> row, for live delta rows
  std::mutex mu;                                   // one writer or reader at a time

  bool is_deleted(uint64_t id) const { return (deleted[id >> 6] >> (id & 63)) & 1; }
  void set_deleted(uint64_t id) { deleted[id >> 6] |= 1ull << (id & 63); }
  // Live::current (src/live.rs:259-265): the row an external id resolves to, or -1
  int64_t current(uint32_t e) const {
    auto it = by_ext.find(e);
    if (it != by_ext.end()) return it->second;
    return (e < n && !is_deleted(e)) ? (int64_t)e : -1;
  }
  int upload_alive() {
    std::vector<uint64_t> a(words, 0);
    const uint64_t rows_now = n + rows;
    for (uint64_t w = 0; w < words; w++) {
      uint64_t bits = ~deleted[w];
      const uint64_t lo = w * 64;
      if (lo >= rows_now) bits = 0;
      else if (rows_now - lo < 64) bits &= (1ull << (rows_now - lo)) - 1;
      a[w] = bits;
    }
    cudaError_t e = cudaMemcpy(alive, a.data(), words * 8, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? SG_OK : fail(SG_ERR_DEVICE, std::string("live tombstones: ") + cudaGetErrorString(e));
  }
};

namespace {

// pack_block (src/lut.rs:72-82) of up to 32 raw codes into one block (group g's byte k: the
// nibble of code k, high nibble that of code k + 16).
void pack_block(const sg_live::Slot* s, uint32_t n, uint8_t* out) {
  memset(out, 0, SG_BLOCK_BYTES);
  for (uint32_t k = 0; k < n; k++)
    for (uint32_t g = 0; g < SG_GROUPS; g++) {
      const uint32_t nib = (s[k].code[g >> 1] >> ((g & 1) * 4)) & 15u;
      out[g * 16 + (k & 15)] |= (uint8_t)(nib << ((k >> 4) * 4));
    }
}

// Every delta list into blocks, in cluster order, and into the index's spare blocks.
int repack(sg_live* L) {
  const uint32_t kc = L->h->ix.kc;
  std::vector<uint32_t> nb(kc), cl(kc);
  uint64_t total = 0;
  for (uint32_t c = 0; c < kc; c++) {
    cl[c] = (uint32_t)L->lists[c].size();
    nb[c] = (cl[c] + SG_BLOCK - 1) / SG_BLOCK;
    total += nb[c];
  }
  if (total > L->block_cap) return fail(SG_ERR_OOM, "the live index's delta lists are full");
  std::vector<uint8_t> blocks(total * SG_BLOCK_BYTES);
  std::vector<float> mul(total * SG_BLOCK, 0.0f), err(total * SG_BLOCK, 0.0f);
  std::vector<uint32_t> ids(total * SG_BLOCK, SG_PAD);
  uint64_t b = 0;
  for (uint32_t c = 0; c < kc; c++) {
    const auto& l = L->lists[c];
    for (uint32_t i = 0; i < nb[c]; i++, b++) {
      const uint32_t n0 = i * SG_BLOCK, cnt = std::min<uint32_t>(SG_BLOCK, cl[c] - n0);
      pack_block(l.data() + n0, cnt, blocks.data() + b * SG_BLOCK_BYTES);
      for (uint32_t k = 0; k < cnt; k++) {
        mul[b * SG_BLOCK + k] = l[n0 + k].mul;
        err[b * SG_BLOCK + k] = l[n0 + k].err;
        ids[b * SG_BLOCK + k] = l[n0 + k].id;
      }
    }
  }
  return sg::index_set_delta(L->h, nb.data(), cl.data(), blocks.data(), mul.data(), err.data(), ids.data(), total);
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) return SG_OK;
    p = nullptr;
    cudaGetLastError();
    return fail(SG_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
};

#define LV_CK(call)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(SG_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" {

int sg_live_open(sg_index* h, uint64_t max_rows, float soar_lambda, sg_live** out) {
  if (!h || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    std::unique_ptr<sg_live> L(new sg_live());
    std::lock_guard<std::mutex> g(h->mu);
    L->h = h;
    L->n = h->ix.n;
    L->max_rows = max_rows;
    L->soar = soar_lambda >= 0.0f;
    L->lambda = soar_lambda;
    const uint32_t kc = h->ix.kc;
    // every delta row takes one or two slots; every list may end in a partial block
    L->block_cap = (max_rows * (L->soar ? 2 : 1) + SG_BLOCK - 1) / SG_BLOCK + kc;
    int rc;
    if ((rc = sg::index_make_live(h, max_rows, L->block_cap))) return rc;
    const sg::DevIndex& x = h->ix;
    LV_CK(cudaMalloc(&L->cents_rot, (size_t)kc * SG_PDIM * 4));
    sg::k_rotate_rows<<<kc, SG_PDIM>>>(x.cent, x.rot, x.rot_norm, L->cents_rot);
    LV_CK(cudaGetLastError());
    L->words = (L->n + max_rows + 63) / 64;
    LV_CK(cudaMalloc(&L->alive, L->words * 8));
    L->deleted.assign(L->words, 0);
    L->lists.resize(kc);
    if ((rc = L->upload_alive())) return rc;
    LV_CK(cudaDeviceSynchronize());
    *out = L.release();
    return SG_OK;
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_live_close(sg_live* L) {
  if (!L) return SG_OK;
  cudaSetDevice(L->h->ix.device);
  cudaFree(L->cents_rot);
  cudaFree(L->alive);
  delete L;
  return SG_OK;
}

int sg_live_insert(sg_live* L, uint32_t m, const uint32_t* ext_ids, const float* vecs) {
  if (!L || (m && (!ext_ids || !vecs))) return fail(SG_ERR_INVALID, "null argument");
  if (m == 0) return SG_OK;
  std::lock_guard<std::mutex> lk(L->mu);
  if (L->rows + m > L->max_rows) return fail(SG_ERR_OOM, "the live index has no room for these rows");
  try {
    sg_index* h = L->h;
    std::lock_guard<std::mutex> g(h->mu);
    sg::DevIndex& x = h->ix;
    LV_CK(cudaSetDevice(x.device));
    const uint64_t id0 = L->n + L->rows;
    DevBuf<float> d_vecs, d_scores, d_fac;
    DevBuf<uint32_t> d_pair;
    DevBuf<uint8_t> d_codes;
    int rc;
    if ((rc = d_vecs.alloc((size_t)m * SG_DIM)) || (rc = d_scores.alloc((size_t)m * x.kc)) ||
        (rc = d_fac.alloc((size_t)m * 4)) || (rc = d_pair.alloc((size_t)m * 2)) ||
        (rc = d_codes.alloc((size_t)m * 2 * SG_CODE_BYTES)))
      return rc;
    LV_CK(cudaMemcpy(d_vecs.p, vecs, (size_t)m * SG_DIM * 4, cudaMemcpyHostToDevice));
    sg::EncodeArgs a{};
    a.vecs = d_vecs.p;
    a.qscale = x.qscale;
    a.cent = x.cent;
    a.cents_rot = L->cents_rot;
    a.kc = x.kc;
    a.signs = x.rot;
    a.rot_norm = x.rot_norm;
    a.t2_sigma = x.has_t2 ? x.t2_sigma : nullptr;
    a.soar = L->soar ? 1 : 0;
    a.lambda = L->lambda;
    a.scores = d_scores.p;
    a.rows = x.rerank + id0 * SG_DIM;
    a.norm256 = x.norm256 ? x.norm256 + id0 : nullptr;
    a.t2 = x.has_t2 ? x.t2_codes + id0 * SG_TIER2_BYTES : nullptr;
    a.t2_norm = x.has_t2 ? x.t2_norm + id0 : nullptr;
    a.pair = d_pair.p;
    a.codes = d_codes.p;
    a.factors = d_fac.p;
    sg::k_live_encode<<<m, 256>>>(a);
    LV_CK(cudaGetLastError());
    std::vector<uint32_t> pair((size_t)m * 2);
    std::vector<uint8_t> codes((size_t)m * 2 * SG_CODE_BYTES);
    std::vector<float> fac((size_t)m * 4);
    LV_CK(cudaMemcpy(pair.data(), d_pair.p, pair.size() * 4, cudaMemcpyDeviceToHost));
    LV_CK(cudaMemcpy(codes.data(), d_codes.p, codes.size(), cudaMemcpyDeviceToHost));
    LV_CK(cudaMemcpy(fac.data(), d_fac.p, fac.size() * 4, cudaMemcpyDeviceToHost));
    // Live::apply_insert's bookkeeping, row by row in order (src/live.rs:351-363)
    for (uint32_t j = 0; j < m; j++) {
      const uint32_t e = ext_ids[j];
      const int64_t old = L->current(e);
      if (old >= 0) L->set_deleted((uint64_t)old);
      const uint32_t id = (uint32_t)(id0 + j);
      L->ext.push_back(e);
      L->by_ext[e] = id;
      for (int t = 0; t < 2; t++) {
        const uint32_t c = pair[(size_t)j * 2 + t];
        if (c == SG_PAD) continue;
        sg_live::Slot s;
        memcpy(s.code, codes.data() + ((size_t)j * 2 + t) * SG_CODE_BYTES, SG_CODE_BYTES);
        s.mul = fac[((size_t)j * 2 + t) * 2];
        s.err = fac[((size_t)j * 2 + t) * 2 + 1];
        s.id = id;
        L->lists[c].push_back(s);
      }
    }
    L->rows += m;
    if ((rc = repack(L))) return rc;
    return L->upload_alive();
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_live_delete(sg_live* L, uint32_t m, const uint32_t* ext_ids) {
  if (!L || (m && !ext_ids)) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(L->mu);
  // Live::apply_delete (src/live.rs:297-304): unknown ids are ignored
  for (uint32_t j = 0; j < m; j++) {
    const int64_t id = L->current(ext_ids[j]);
    if (id >= 0) {
      L->set_deleted((uint64_t)id);
      L->by_ext.erase(ext_ids[j]);
    }
  }
  cudaSetDevice(L->h->ix.device);
  return L->upload_alive();
}

int sg_live_search(sg_live* L, uint32_t nq, const float* q768, const float* q256, const sg_params* params,
                   float* out_scores, uint32_t* out_ids, uint32_t* out_counts) {
  if (!L || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(L->mu);
  int rc = sg::index_search_allow(L->h, nq, q768, q256, *params, L->alive, L->words, out_scores, out_ids,
                                  out_counts);
  if (rc) return rc;
  // Live::search (src/live.rs:381-385): rows to external ids
  const uint32_t k = params->k;
  for (uint32_t q = 0; q < nq; q++)
    for (uint32_t i = 0; i < out_counts[q]; i++) {
      uint32_t& id = out_ids[(size_t)q * k + i];
      if (id >= L->n) id = L->ext[id - L->n];
    }
  return SG_OK;
}

int sg_live_info(sg_live* L, uint64_t* delta_rows, uint64_t* delta_slots, uint64_t* deleted) {
  if (!L) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(L->mu);
  if (delta_rows) *delta_rows = L->rows;
  if (delta_slots) {
    uint64_t s = 0;
    for (const auto& l : L->lists) s += l.size();
    *delta_slots = s;
  }
  if (deleted) {
    uint64_t d = 0;
    for (uint64_t w : L->deleted) d += (uint64_t)__builtin_popcountll(w);
    *deleted = d;
  }
  return SG_OK;
}

}  // extern "C"
