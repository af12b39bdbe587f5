// sieve_gpu.cu — the C ABI (include/sieve_gpu.h): index upload, workspace and the query pipeline.
//
// Pipeline of one batched call (every stage one kernel on the index's stream):
//   prefix (if q256 not given) -> prep -> route scores (BF16 tensor cores or exact FP32)
//   -> route select (+FP32 rescoring window, margin, budget, work items) -> scan (persistent,
//   drains the (query, probe, chunk) queue) -> cut + dedup -> prune / tier-2 / int8 rerank -> top-k.
#include <cuda_bf16.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "internal.hpp"

namespace sg {

std::string& last_error() {
  static thread_local std::string e;
  return e;
}

int fail(int code, const std::string& msg) {
  last_error() = msg;
  return code;
}

}  // namespace sg

using sg::fail;

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(SG_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

template <typename T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SG_ERR_OOM, std::string("cudaMalloc ") + std::to_string(n * sizeof(T)) +
                                " bytes: " + cudaGetErrorString(e));
  }
  return SG_OK;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

template <typename T>
int upload(T** d, const T* h, size_t n) {
  int rc = dalloc(d, n);
  if (rc) return rc;
  if (n) CK(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return SG_OK;
}

void free_index(sg::DevIndex& x) {
  dfree(x.cent);
  dfree(x.cent_t);
  dfree(x.cent_bf16);
  dfree(x.block_off);
  dfree(x.clen);
  dfree(x.blocks);
  dfree(x.blocks_tc);
  dfree(x.mul);
  dfree(x.err);
  dfree(x.ids);
  dfree(x.rot);
  dfree(x.t2_sigma);
  dfree(x.t2_codes);
  dfree(x.t2_norm);
  dfree(x.rerank);
  dfree(x.norm256);
  dfree(x.qscale);
  dfree(x.codes);
}

void free_ws(sg::Workspace& w) {
  dfree(w.allow_q);
  dfree(w.allow_wq);
  w.allow_q_cap = 0;
  dfree(w.brute);
  w.brute_cap = 0;
  dfree(w.q768);
  dfree(w.q256);
  dfree(w.q16);
  dfree(w.w8);
  dfree(w.fq);
  dfree(w.tc_start);
  dfree(w.tables);
  dfree(w.qp);
  dfree(w.qnorm);
  dfree(w.wq);
  dfree(w.winv);
  dfree(w.wq256);
  dfree(w.winv256);
  dfree(w.scores);
  dfree(w.probe_sc);
  dfree(w.probe_cl);
  dfree(w.probe_off);
  dfree(w.probe_n);
  dfree(w.scanned);
  dfree(w.items);
  dfree(w.seed_items);
  dfree(w.counters);
  dfree(w.inv_cnt);
  dfree(w.inv_fill);
  dfree(w.inv_off);
  dfree(w.inv_list);
  dfree(w.gitems);
  dfree(w.thr);
  dfree(w.ccount);
  dfree(w.cbuf_est);
  dfree(w.cbuf_info);
  dfree(w.overflow);
  dfree(w.cest);
  dfree(w.cid);
  dfree(w.cerr);
  dfree(w.cn);
  dfree(w.lid);
  dfree(w.lsc);
  dfree(w.ln);
  dfree(w.out_sc);
  dfree(w.out_id);
  dfree(w.out_n);
  dfree(w.allow);
  if (w.events)
    for (auto& e : w.ev) cudaEventDestroy(e);
  w = sg::Workspace();
}

}  // namespace

namespace sg {
// Per-cluster chunk and slot counts, largest first, as prefix sums over x.k clusters (from
// x.h_block_off): the work-queue and candidate-buffer bounds of a call probing P clusters.
void set_cluster_bounds(DevIndex& x, uint32_t chunk) {
  const uint32_t K = x.k;
  std::vector<uint32_t> ch(K);
  std::vector<uint64_t> sl(K);
  for (uint32_t c = 0; c < K; c++) {
    const uint64_t nb = x.h_block_off[c + 1] - x.h_block_off[c];
    ch[c] = (uint32_t)((nb + chunk - 1) / chunk);
    sl[c] = nb * SG_BLOCK;
  }
  std::sort(ch.begin(), ch.end(), std::greater<uint32_t>());
  std::sort(sl.begin(), sl.end(), std::greater<uint64_t>());
  x.h_chunks_desc_prefix.assign(K + 1, 0);
  x.h_slots_desc_prefix.assign(K + 1, 0);
  for (uint32_t c = 0; c < K; c++) {
    x.h_chunks_desc_prefix[c + 1] = x.h_chunks_desc_prefix[c] + ch[c];
    x.h_slots_desc_prefix[c + 1] = x.h_slots_desc_prefix[c] + sl[c];
  }
}
}  // namespace sg

namespace {
using sg::set_cluster_bounds;

int build_index(const sg_ivf_arrays* a, int device, sg_index** out) {
  if (!a || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  if (a->k == 0 || !a->centroids || !a->block_off)
    return fail(SG_ERR_INVALID, "index needs centroids and block_off");
  if (!a->ids || !a->blocks) return fail(SG_ERR_INVALID, "index needs ids.u32 and blocks.bin");
  // without rotation.f32 + factors.f32 the slots hold global sign codes (src/ivf.rs:700-717)
  const bool global = !a->factors || !a->rotation;
  if (!a->rerank || !a->quant_scale)
    return fail(SG_ERR_INVALID, "corpus needs rerank.i8 and quant.f32");
  const uint32_t K = a->k;
  if (a->block_off[0] != 0) return fail(SG_ERR_INVALID, "block_off[0] != 0");
  for (uint32_t c = 0; c < K; c++)
    if (a->block_off[c + 1] < a->block_off[c]) return fail(SG_ERR_INVALID, "block_off not monotonic");
  const uint64_t nblocks = a->block_off[K];
  if (nblocks * SG_BLOCK >= 0xFFFFFFFFull) return fail(SG_ERR_INVALID, "more than 2^32 slots");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(SG_ERR_DEVICE, "no such CUDA device");
  CK(cudaSetDevice(device));
  std::unique_ptr<sg_index> h(new sg_index());
  sg::DevIndex& x = h->ix;
  x.device = device;
  x.k = K;
  x.kc = K;
  x.n = a->n;
  x.nblocks = nblocks;
  x.nslots = nblocks * SG_BLOCK;
  x.global = global;
  // cluster lengths: PAD may only fill the tail of a cluster's last block (src/ivf.rs:378-380)
  x.h_block_off.assign(a->block_off, a->block_off + K + 1);
  x.h_clen.resize(K);
  for (uint32_t c = 0; c < K; c++) {
    uint64_t s0 = a->block_off[c] * SG_BLOCK, s1 = a->block_off[c + 1] * SG_BLOCK;
    uint64_t len = s0;
    while (len < s1 && a->ids[len] != SG_PAD) {
      if (a->ids[len] >= a->n) return fail(SG_ERR_INVALID, "ids.u32 holds a row beyond the corpus");
      len++;
    }
    for (uint64_t s = len; s < s1; s++)
      if (a->ids[s] != SG_PAD)
        return fail(SG_ERR_INVALID, "PAD slot inside a cluster (ids.u32 is not in build layout)");
    if (s1 - len >= SG_BLOCK) return fail(SG_ERR_INVALID, "a cluster holds a whole block of PAD");
    x.h_clen[c] = (uint32_t)(len - s0);
  }
  std::vector<uint32_t> boff32(K + 1);
  for (uint32_t c = 0; c <= K; c++) boff32[c] = (uint32_t)a->block_off[c];
  set_cluster_bounds(x, h->cfg.small_chunk_blocks);
  // centroids: row-major, transposed, BF16; largest norm for the routing error window
  std::vector<float> ct((size_t)K * SG_PDIM);
  std::vector<__nv_bfloat16> cb((size_t)K * SG_PDIM);
  float nmax = 0.0f;
  for (uint32_t c = 0; c < K; c++) {
    double s = 0;
    for (int t = 0; t < SG_PDIM; t++) {
      float v = a->centroids[(size_t)c * SG_PDIM + t];
      ct[(size_t)t * K + c] = v;
      cb[(size_t)c * SG_PDIM + t] = __float2bfloat16_rn(v);
      s += (double)v * v;
    }
    nmax = std::max(nmax, (float)sqrt(s));
  }
  x.cent_norm_max = nmax * 1.0001f;
  // factors.f32 [mul, err] per slot -> two planes; global sign codes: the score itself is the
  // ranking estimate (mul 1) and carries no bound (err +inf)
  std::vector<float> mul(x.nslots), err(x.nslots);
  for (uint64_t s = 0; s < x.nslots; s++) {
    mul[s] = global ? 1.0f : a->factors[2 * s];
    err[s] = global ? INFINITY : a->factors[2 * s + 1];
  }
  x.rot_norm = powf(256.0f, -1.5f);
  int rc;
  if ((rc = upload(&x.cent, a->centroids, (size_t)K * SG_PDIM)) ||
      (rc = upload(&x.cent_t, ct.data(), ct.size())) ||
      (rc = upload(&x.cent_bf16, cb.data(), cb.size())) ||
      (rc = upload(&x.block_off, boff32.data(), boff32.size())) ||
      (rc = upload(&x.clen, x.h_clen.data(), x.h_clen.size())) ||
      (rc = upload(&x.blocks, a->blocks, (size_t)nblocks * SG_BLOCK_BYTES)) ||
      (rc = upload(&x.mul, mul.data(), mul.size())) || (rc = upload(&x.err, err.data(), err.size())) ||
      (rc = upload(&x.ids, a->ids, x.nslots)) ||
      (!global && (rc = upload(&x.rot, a->rotation, 3 * SG_PDIM))) ||
      (rc = upload(&x.rerank, a->rerank, (size_t)a->n * SG_DIM)) ||
      (rc = upload(&x.qscale, a->quant_scale, SG_DIM))) {
    free_index(x);
    return rc;
  }
  if (!sg::route_gemm_ready()) {
    free_index(x);
    return fail(SG_ERR_DEVICE, "cuTensorMapEncodeTiled (the routing GEMM's TMA maps) is unavailable");
  }
  // the batched tensor-core scan reads its own copy of the codes, slot-major
  if (const char* tc = getenv("SIEVE_GPU_TC")) h->cfg.tc = atoi(tc) == 2 ? 2 : 1;
  if (const char* sp = getenv("SIEVE_GPU_TC_SPLIT")) h->cfg.tc_split = (uint32_t)strtoul(sp, nullptr, 10);
  if (const char* tm = getenv("SIEVE_GPU_TC_MIN")) h->cfg.tc_min_queries = (uint32_t)strtoul(tm, nullptr, 10);
  if ((rc = dalloc(&x.blocks_tc, (size_t)nblocks * 256))) {
    free_index(x);
    return rc;
  }
  sg::transcode_tc(x.blocks, nblocks, x.blocks_tc, 0);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
    free_index(x);
    return fail(SG_ERR_DEVICE, "transcode of the code blocks failed");
  }
  if ((a->norm256 && (rc = upload(&x.norm256, a->norm256, a->n))) ||
      (a->codes && (rc = upload(&x.codes, a->codes, (size_t)a->n * SG_CODE_BYTES)))) {
    free_index(x);
    return rc;
  }
  if (a->tier2_sigma && a->tier2_codes && a->tier2_norm) {
    if ((rc = upload(&x.t2_sigma, a->tier2_sigma, SG_PDIM)) ||
        (rc = upload(&x.t2_codes, a->tier2_codes, (size_t)a->n * SG_TIER2_BYTES)) ||
        (rc = upload(&x.t2_norm, a->tier2_norm, a->n))) {
      free_index(x);
      return rc;
    }
    x.has_t2 = true;
  }
  if (const char* sc = getenv("SIEVE_GPU_SOFT_CAP")) h->cfg.soft_cap = (uint32_t)strtoul(sc, nullptr, 10);
  {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
      h->cfg.cbuf_budget = std::min<uint64_t>(std::max<uint64_t>(free_b / 4, 8ull << 30), 32ull << 30);
  }
  if (const char* m = getenv("SIEVE_GPU_MMA")) h->cfg.mma = atoi(m);
  if (const char* gr = getenv("SIEVE_GPU_GRAPHS")) h->cfg.graphs = atoi(gr);
  if (const char* ss = getenv("SIEVE_GPU_SMALL_SEED"))
    h->cfg.small_seed_blocks =
        std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)strtoul(ss, nullptr, 10), sg::kMaxChunkBlocks));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  h->sms = prop.multiProcessorCount;
  CK(cudaStreamCreateWithFlags(&h->def.stream, cudaStreamNonBlocking));
  *out = h.release();
  return SG_OK;
}

// Sizes the workspace for nq queries under params p (grows, never shrinks).
// How a call routes: the index's own probing (plain search, the Post plan), or the Expand plan
// over a filter's per-cluster allowed slots.
struct RoutePlan {
  const uint32_t* per_cluster = nullptr;  // device [k]; set for Expand
  uint64_t target = 0;
  bool given = false;  // the probe lists are staged in ws.probe_sc / probe_cl / probe_n
  bool expand() const { return per_cluster != nullptr; }
};

// The device addresses a captured pipeline bakes in; when any moves, captured graphs are stale.
uint64_t ws_signature(const sg::Workspace& w) {
  const void* ptrs[] = {w.q768, w.q256, w.tables, w.qp, w.qnorm, w.wq, w.winv, w.wq256, w.winv256,
                        w.w8, w.fq, w.tc_start,
                        w.scores, w.probe_sc, w.probe_cl, w.probe_off, w.probe_n, w.scanned,
                        w.items, w.seed_items, w.counters, w.inv_cnt, w.inv_fill, w.inv_off,
                        w.inv_list, w.gitems, w.thr, w.ccount, w.cbuf_est, w.cbuf_info,
                        w.overflow, w.cest, w.cid, w.cerr, w.cn, w.lid, w.lsc, w.ln, w.out_sc,
                        w.out_id, w.out_n};
  uint64_t hsh = 1469598103934665603ull;
  for (const void* q : ptrs) hsh = (hsh ^ (uint64_t)(uintptr_t)q) * 1099511628211ull;
  hsh = (hsh ^ w.item_cap) * 1099511628211ull;
  hsh = (hsh ^ w.cbuf_per_q) * 1099511628211ull;
  return (hsh ^ w.gitems_cap) * 1099511628211ull;
}

void drop_graphs(sg::Ctx& c) {
  for (auto& g : c.graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  c.graphs.clear();
}

int ensure_ws_impl(sg_index* h, sg::Ctx& c, uint32_t nq, const sg_params& p, uint32_t cbuf_per_q);

int ensure_ws(sg_index* h, sg::Ctx& c, uint32_t nq, const sg_params& p, uint32_t cbuf_per_q) {
  const uint64_t before = ws_signature(c.ws);
  const int rc = ensure_ws_impl(h, c, nq, p, cbuf_per_q);
  if (ws_signature(c.ws) != before) {
    drop_graphs(c);
    c.gen++;
  }
  return rc;
}

int ensure_ws_impl(sg_index* h, sg::Ctx& c, uint32_t nq, const sg_params& p, uint32_t cbuf_per_q) {
  sg::Workspace& w = c.ws;
  cbuf_per_q = (cbuf_per_q + 3) & ~3u;
  const sg::DevIndex& x = h->ix;
  const uint32_t P = sg::probe_stride(x, p.nprobe);
  const uint32_t cand = std::max<uint32_t>(p.cand, 1);
  const uint32_t k = std::max<uint32_t>(p.k, 1);
  int rc;
  if (!w.events) {
    for (auto& e : w.ev) CK(cudaEventCreate(&e));
    w.events = true;
  }
  if (nq > w.nq_cap) {
    uint32_t n = std::max(nq, w.nq_cap * 2);
    dfree(w.q768); dfree(w.q256); dfree(w.q16); dfree(w.tables); dfree(w.qp); dfree(w.qnorm); dfree(w.wq);
    dfree(w.w8); dfree(w.fq); dfree(w.tc_start);
    dfree(w.winv); dfree(w.wq256); dfree(w.winv256); dfree(w.probe_n); dfree(w.scanned); dfree(w.seed_items);
    dfree(w.thr); dfree(w.ccount); dfree(w.overflow); dfree(w.cn); dfree(w.ln); dfree(w.out_n);
    if ((rc = dalloc(&w.q768, (size_t)n * SG_DIM)) || (rc = dalloc(&w.q256, (size_t)n * SG_PDIM)) ||
        (rc = dalloc(&w.q16, (size_t)n * SG_PDIM)) || (rc = dalloc(&w.w8, (size_t)n * SG_GROUPS)) ||
        (rc = dalloc(&w.fq, n)) || (rc = dalloc(&w.tc_start, n)) ||
        (rc = dalloc(&w.tables, (size_t)n * SG_GROUPS * 16)) || (rc = dalloc(&w.qp, n)) ||
        (rc = dalloc(&w.qnorm, n)) || (rc = dalloc(&w.wq, (size_t)n * SG_DIM)) ||
        (rc = dalloc(&w.winv, n)) || (rc = dalloc(&w.wq256, (size_t)n * SG_PDIM)) ||
        (rc = dalloc(&w.winv256, n)) || (rc = dalloc(&w.probe_n, n)) ||
        (rc = dalloc(&w.scanned, n)) || (rc = dalloc(&w.seed_items, n)) || (rc = dalloc(&w.thr, n)) || (rc = dalloc(&w.ccount, n)) ||
        (rc = dalloc(&w.overflow, n)) || (rc = dalloc(&w.cn, n)) || (rc = dalloc(&w.ln, n)) ||
        (rc = dalloc(&w.out_n, n)))
      return rc;
    w.nq_cap = n;
    w.P_cap = w.cand_cap = w.k_cap = 0;
    w.scores_cap = 0;
    w.item_cap = 0;
    w.cbuf_cap = 0;
  }
  const uint32_t n = w.nq_cap;
  if ((uint64_t)n * x.kc > w.scores_cap) {
    dfree(w.scores);
    if ((rc = dalloc(&w.scores, (size_t)n * x.kc))) return rc;
    w.scores_cap = (uint64_t)n * x.kc;
  }
  if (P > w.P_cap) {
    dfree(w.probe_sc); dfree(w.probe_cl); dfree(w.probe_off);
    if ((rc = dalloc(&w.probe_sc, (size_t)n * P)) || (rc = dalloc(&w.probe_cl, (size_t)n * P)) ||
        (rc = dalloc(&w.probe_off, (size_t)n * P)))
      return rc;
    w.P_cap = P;
  }
  if (cand > w.cand_cap) {
    dfree(w.cest); dfree(w.cid); dfree(w.cerr); dfree(w.lid); dfree(w.lsc);
    if ((rc = dalloc(&w.cest, (size_t)n * cand)) || (rc = dalloc(&w.cid, (size_t)n * cand)) ||
        (rc = dalloc(&w.cerr, (size_t)n * cand)) || (rc = dalloc(&w.lid, (size_t)n * cand)) ||
        (rc = dalloc(&w.lsc, (size_t)n * cand)))
      return rc;
    w.cand_cap = cand;
  }
  if (k > w.k_cap) {
    dfree(w.out_sc); dfree(w.out_id);
    if ((rc = dalloc(&w.out_sc, (size_t)n * k)) || (rc = dalloc(&w.out_id, (size_t)n * k))) return rc;
    w.k_cap = k;
  }
  const uint64_t items = (uint64_t)nq * x.h_chunks_desc_prefix[P];
  if (items > w.item_cap) {
    dfree(w.items);
    uint64_t want = std::max<uint64_t>(items, w.item_cap * 2);
    if ((rc = dalloc(&w.items, want))) return rc;
    w.item_cap = want;
  }
  if (!w.counters && (rc = dalloc(&w.counters, 8))) return rc;
  if (!w.inv_cnt || w.inv_k != x.k) {  // a live index has twice the clusters it opened with
    dfree(w.inv_cnt);
    dfree(w.inv_fill);
    dfree(w.inv_off);
    dfree(w.inv_list);
    dfree(w.gitems);
    w.inv_cap = 0;
    if ((rc = dalloc(&w.inv_cnt, x.k)) || (rc = dalloc(&w.inv_fill, x.k)) ||
        (rc = dalloc(&w.inv_off, (size_t)x.k + 1)))
      return rc;
    w.inv_k = x.k;
  }
  const uint64_t pairs = (uint64_t)nq * P;
  if (pairs > w.inv_cap) {
    dfree(w.inv_list);
    dfree(w.gitems);
    uint64_t want = std::max<uint64_t>(pairs, w.inv_cap * 2);
    if ((rc = dalloc(&w.inv_list, want)) || (rc = dalloc(&w.gitems, want / 64 + x.k + 1))) return rc;
    w.inv_cap = want;
    w.gitems_cap = want / 64 + x.k + 1;
  }
  const uint64_t cb = (uint64_t)nq * cbuf_per_q;
  if (cb > w.cbuf_cap) {
    dfree(w.cbuf_est);
    dfree(w.cbuf_info);
    if ((rc = dalloc(&w.cbuf_est, cb)) || (rc = dalloc(&w.cbuf_info, cb))) return rc;
    w.cbuf_cap = cb;
  }
  w.cbuf_per_q = cbuf_per_q;
  return SG_OK;
}

int check_params(const sg_index* h, const sg_params* p) {
  if (!p) return fail(SG_ERR_INVALID, "params is null");
  if (p->cand > sg::kMaxCand || p->k > sg::kMaxCand || p->rerank_r > sg::kMaxCand)
    return fail(SG_ERR_INVALID, "cand, k and rerank_r must be <= 4096");
  if (sg::probe_stride(h->ix, p->nprobe) > 4096)
    return fail(SG_ERR_INVALID, h->ix.live ? "nprobe must be <= 2048 in a live index" : "nprobe must be <= 4096");
  if (p->rerank_kind > SG_RERANK_SSD) return fail(SG_ERR_INVALID, "unknown rerank kind");
  if ((p->rerank_kind == SG_RERANK_PREFIX ||
       (p->rerank_kind == SG_RERANK_TIERED && !h->ix.has_t2)) &&
      !h->ix.norm256)
    return fail(SG_ERR_UNSUPPORTED, "prefix rerank needs norm256.f32");
  if (p->has_prune && !(p->prune_w == p->prune_w)) return fail(SG_ERR_INVALID, "prune_w is NaN");
  return SG_OK;
}

// Does a call of nq queries run the tensor-core scan? (It pays off once enough queries share each
// probed cluster; SIEVE_GPU_MMA forces it off (0) or on (2).)
bool use_mma(const sg_index* h, const sg::Config& cfg, uint32_t nq, uint32_t P) {
  const sg::DevIndex& x = h->ix;
  if (!x.blocks_tc || P <= 1 || P > 4096) return false;  // inverted lists keep 12-bit ranks
  if (x.global && cfg.tc != 1) return false;             // only the bound pass ranks global codes
  if (cfg.mma == 2) return true;
  if (cfg.mma != 1 || nq < 64) return false;
  // the batch splits per cluster on the device (few queries: ALU, many: tensor cores), so the
  // inverted path pays off once some cluster can gather tc_min_queries queries
  return (uint64_t)nq * (P - 1) >= (uint64_t)cfg.tc_min_queries * 16;
}

// Exact per-query candidate-buffer bound. A slot is appended at most once, so the probed
// clusters' slots bound it; the ALU scan also cuts every chunk to `cand`, so chunks x cand does.
uint32_t full_cap(const sg_index* h, const sg::Config& cfg, const sg_params& p, uint32_t nq) {
  const uint32_t P = sg::probe_stride(h->ix, p.nprobe);
  uint64_t b = h->ix.h_slots_desc_prefix[P];
  // (a global-code chunk keeps every slot tied with its cand-th score, so only the slots bound it)
  if (!use_mma(h, cfg, nq, P) && !h->ix.global)
    b = std::min<uint64_t>(b, (uint64_t)h->ix.h_chunks_desc_prefix[P] * std::max<uint32_t>(p.cand, 1));
  return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(b, 1), 0x7FFFFFFFull);
}

// Soft per-query buffer for batches: at least 16 x cand entries, and up to the index's
// candidate-buffer budget (a quarter of the device memory free at open, 8 to 32 GiB) shared by
// the batch. A query that fills it is re-run (see search_impl) with the exact bound.
uint32_t batch_cap(const sg_index* h, const sg::Config& cfg, const sg_params& p, uint32_t nq,
                   bool soft_always = false) {
  uint32_t full = full_cap(h, cfg, p, nq);
  if (cfg.soft_cap) return std::min(full, cfg.soft_cap);
  if (nq <= 8 && !soft_always) return full;
  uint64_t budget = cfg.cbuf_budget / (sizeof(uint4) * (uint64_t)nq);
  uint64_t soft = std::max<uint64_t>(16ull * std::max<uint32_t>(p.cand, 1), budget);
  return (uint32_t)std::min<uint64_t>(full, soft);
}

enum Stage { kToCandidates = 1, kToSearch = 2 };

// Runs the pipeline on queries already in ws.q768 / ws.q256 (have_q256 = false: derive it).
// With `timed`, events ev[0..7] bracket the stages (see collect_stats).
int run_pipeline(sg_index* h, const sg::Config& cfg, sg::Ctx& c, uint32_t nq, const sg_params& p,
                 bool have_q256, const uint64_t* d_allow, uint64_t allow_words, Stage stage, bool timed,
                 const RoutePlan& rp = RoutePlan()) {
  sg::Workspace& w = c.ws;
  sg::DevIndex& x = h->ix;
  cudaStream_t st = c.stream;
  uint32_t launches = 0;
  CK(cudaMemsetAsync(w.counters, 0, 8 * sizeof(uint32_t), st));
  CK(cudaMemsetAsync(w.thr, 0, nq * sizeof(uint32_t), st));
  CK(cudaMemsetAsync(w.ccount, 0, nq * sizeof(uint32_t), st));
  CK(cudaMemsetAsync(w.overflow, 0, nq, st));
  if (timed) CK(cudaEventRecord(w.ev[0], st));
  if (!have_q256) {
    sg::launch_prefix(w, nq, st);
    launches++;
  }
  sg::launch_prep(x, w, nq, st);
  if (timed) CK(cudaEventRecord(w.ev[1], st));
  const int route_prec = rp.expand() ? SG_ROUTE_FP32 : cfg.route_precision;
  if (!rp.given) CK(sg::launch_route_scores(x, w, nq, route_prec, st));
  if (timed) CK(cudaEventRecord(w.ev[2], st));
  // Few queries leave most SMs to the chunked pass: a short seed (one CTA per query scans it
  // alone) and short chunks keep the GPU busy.
  const bool small = nq < cfg.small_batch;
  const uint32_t cb = small ? cfg.small_chunk_blocks : cfg.chunk_blocks;
  const uint32_t sb = small ? cfg.small_seed_blocks : cfg.seed_blocks;
  // The tensor-core scan pays off once enough queries share each probed cluster.
  const uint32_t P = sg::probe_stride(x, p.nprobe);
  const bool mma = !rp.expand() && use_mma(h, cfg, nq, P);
  if (rp.expand())
    sg::launch_route_expand(x, w, nq, p, cb, sb, rp.per_cluster, rp.target, st);
  else if (rp.given)
    sg::launch_route_given(x, w, nq, p, cb, sb, !mma, w.probe_sc, w.probe_cl, w.probe_n, st);
  else
    sg::launch_route_select(x, w, nq, p, cfg.route_precision, cb, sb, !mma, st);
  if (timed) CK(cudaEventRecord(w.ev[3], st));
  launches += route_prec == SG_ROUTE_BF16 ? 4 : 3;  // prep, routing (BF16: + the bf16 queries), select
  if (p.cand > 0) {
    sg::launch_scan(x, w, nq, p, d_allow, allow_words, h->sms, 0, sb, cfg.scan_ctas_per_sm, st);
    if (timed) CK(cudaEventRecord(w.ev[9], st));
    if (mma)  // ALU chunks and tcgen05 tiles, split per cluster
      launches += sg::launch_scan_tc(x, w, nq, p, d_allow, allow_words, h->sms, cfg, cb, st);
    else
      sg::launch_scan(x, w, nq, p, d_allow, allow_words, h->sms, cb, 0, cfg.scan_ctas_per_sm, st);
    if (timed) CK(cudaEventRecord(w.ev[4], st));
    sg::launch_cut(x, w, nq, p, st);
    launches += 3;
  } else {
    if (timed) CK(cudaEventRecord(w.ev[9], st));
    if (timed) CK(cudaEventRecord(w.ev[4], st));
    CK(cudaMemsetAsync(w.cn, 0, nq * sizeof(uint32_t), st));
  }
  if (timed) CK(cudaEventRecord(w.ev[5], st));
  if (stage == kToSearch)
    launches += sg::launch_rerank(x, w, nq, p, st, timed ? w.ev[7] : nullptr,
                                  timed ? w.ev[8] : nullptr);
  if (timed) CK(cudaEventRecord(w.ev[6], st));
  CK(cudaGetLastError());
  w.last = sg_stats();
  w.last.launches = launches;
  return SG_OK;
}

// After the stream has synchronised: stage times of a timed run_pipeline.
void collect_stats(sg::Workspace& w, const sg_params& p) {
  float* ms[6] = {&w.last.ms_prep, &w.last.ms_route_gemm, &w.last.ms_route_select,
                  &w.last.ms_scan, &w.last.ms_cut, &w.last.ms_rerank};
  for (int i = 0; i < 6; i++) cudaEventElapsedTime(ms[i], w.ev[i], w.ev[i + 1]);
  cudaEventElapsedTime(&w.last.ms_total, w.ev[0], w.ev[6]);
  if (p.rerank_kind == SG_RERANK_TIERED) cudaEventElapsedTime(&w.last.ms_tier2, w.ev[7], w.ev[8]);
  if (p.cand > 0) cudaEventElapsedTime(&w.last.ms_seed, w.ev[3], w.ev[9]);
}

// Runs the search pipeline on c's stream: directly, or, for a call shape seen before and with
// graphs on, by replaying the CUDA graph captured for it (the second time a shape occurs; the
// first run of each kernel also sets its shared-memory attributes outside any capture).
int launch_pipeline(sg_index* h, const sg::Config& cfg, sg::Ctx& c, uint32_t nq, const sg_params& p,
                    bool have_q256, const uint64_t* d_allow, uint64_t allow_words, bool timed) {
  if (!cfg.graphs || timed)
    return run_pipeline(h, cfg, c, nq, p, have_q256, d_allow, allow_words, kToSearch, timed);
  sg::GraphKey key;
  memset(&key, 0, sizeof key);
  key.nq = nq;
  key.p = p;
  key.have_q256 = have_q256;
  key.allow = d_allow;
  key.allow_words = allow_words;
  key.gen = c.gen;
  key.cfg_gen = cfg.gen;
  for (auto& g : c.graphs)
    if (g.key.same(key)) {
      if (!g.exec) {  // seen once before: capture it now
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        int rc = run_pipeline(h, cfg, c, nq, p, have_q256, d_allow, allow_words, kToSearch, false);
        cudaError_t e = cudaStreamEndCapture(c.stream, &graph);
        if (rc) {
          if (graph) cudaGraphDestroy(graph);
          return rc;
        }
        if (e != cudaSuccess)
          return fail(SG_ERR_DEVICE, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
          return fail(SG_ERR_DEVICE, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        g.exec = exec;
        g.launches = c.ws.last.launches;
      }
      CK(cudaGraphLaunch(g.exec, c.stream));
      c.ws.last = sg_stats();
      c.ws.last.launches = g.launches;
      return SG_OK;
    }
  if (c.graphs.size() >= 32) {
    if (c.graphs.front().exec) cudaGraphExecDestroy(c.graphs.front().exec);
    c.graphs.erase(c.graphs.begin());
  }
  c.graphs.push_back({key, nullptr, 0});
  return run_pipeline(h, cfg, c, nq, p, have_q256, d_allow, allow_words, kToSearch, false);
}

int stage_inputs(sg::Ctx& c, uint32_t nq, const float* q768, const float* q256, bool device) {
  sg::Workspace& w = c.ws;
  cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault;
  if (q768) CK(cudaMemcpyAsync(w.q768, q768, (size_t)nq * SG_DIM * 4, kind, c.stream));
  else CK(cudaMemsetAsync(w.q768, 0, (size_t)nq * SG_DIM * 4, c.stream));
  if (q256) CK(cudaMemcpyAsync(w.q256, q256, (size_t)nq * SG_PDIM * 4, kind, c.stream));
  return SG_OK;
}

int stage_allow(sg::Ctx& c, const uint64_t* allow, uint64_t words, bool device,
                const uint64_t** d_allow) {
  *d_allow = nullptr;
  if (!allow) return SG_OK;
  if (device) {
    *d_allow = allow;
    return SG_OK;
  }
  sg::Workspace& w = c.ws;
  if (words > w.allow_cap) {
    dfree(w.allow);
    int rc = dalloc(&w.allow, words);
    if (rc) return rc;
    w.allow_cap = words;
  }
  CK(cudaMemcpyAsync(w.allow, allow, words * 8, cudaMemcpyDefault, c.stream));
  *d_allow = w.allow;
  return SG_OK;
}

// Full search of nq queries with inputs staged; copies results out (kind: D2H or D2D).
int search_impl(sg_index* h, const sg::Config& cfg, sg::Ctx& c, uint32_t nq, const float* q768,
                const float* q256, const sg_params& user_p, const uint64_t* allow, uint64_t allow_words,
                float* out_sc, uint32_t* out_id, uint32_t* out_n, sg_timing* t, bool device,
                bool allow_dev = false, const RoutePlan& rp = RoutePlan()) {
  int rc;
  if ((rc = check_params(h, &user_p))) return rc;
  if (nq == 0) return SG_OK;
  if (!q768) return fail(SG_ERR_INVALID, "q768 is null");
  CK(cudaSetDevice(h->ix.device));
  allow_dev = allow_dev || device;
  sg_params p = user_p;
  if (rp.expand()) {  // Index::route over every cluster, no margin or budget (src/filter.rs:81)
    p.nprobe = h->ix.k;
    p.has_margin = 0;
    p.has_budget = 0;
  }
  uint32_t cap = batch_cap(h, cfg, p, nq, rp.expand());
  if ((rc = ensure_ws(h, c, nq, p, cap))) return rc;
  if ((rc = stage_inputs(c, nq, q768, q256, device))) return rc;
  const uint64_t* d_allow;
  if ((rc = stage_allow(c, allow, allow_words, allow_dev, &d_allow))) return rc;
  const bool timed_run = t != nullptr || cfg.timing;
  if (rp.expand())
    rc = run_pipeline(h, cfg, c, nq, p, q256 != nullptr, d_allow, allow_words, kToSearch, timed_run, rp);
  else
    rc = launch_pipeline(h, cfg, c, nq, p, q256 != nullptr, d_allow, allow_words, timed_run);
  if (rc) return rc;
  sg::Workspace& w = c.ws;
  std::vector<uint8_t> ovf(nq);
  CK(cudaMemcpyAsync(ovf.data(), w.overflow, nq, cudaMemcpyDeviceToHost, c.stream));
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, w.counters + 2, 4, cudaMemcpyDeviceToHost, c.stream));
  const uint32_t k = p.k;
  cudaMemcpyKind okind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (k) {
    CK(cudaMemcpyAsync(out_sc, w.out_sc, (size_t)nq * k * 4, okind, c.stream));
    CK(cudaMemcpyAsync(out_id, w.out_id, (size_t)nq * k * 4, okind, c.stream));
  }
  CK(cudaMemcpyAsync(out_n, w.out_n, (size_t)nq * 4, okind, c.stream));
  std::vector<uint64_t> scanned;
  std::vector<uint32_t> probed, reranked, buffered;
  if (timed_run) {
    scanned.resize(nq);
    probed.resize(nq);
    reranked.resize(nq);
    buffered.resize(nq);
    CK(cudaMemcpyAsync(buffered.data(), w.ccount, nq * 4, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(scanned.data(), w.scanned, nq * 8, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(probed.data(), w.probe_n, nq * 4, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(reranked.data(), w.ln, nq * 4, cudaMemcpyDeviceToHost, c.stream));
  }
  CK(cudaStreamSynchronize(c.stream));
  if (status & sg::kStatusOverflow) return fail(SG_ERR_INVALID, "work queue overflow");
  if (status & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "a tensor-core wait ran out (routing GEMM or scan)");
  const bool timed = timed_run;
  if (timed) {
    collect_stats(w, p);
    uint64_t sc = 0, pr = 0, rr = 0, bu = 0;
    for (uint32_t i = 0; i < nq; i++) {
      sc += scanned[i];
      pr += probed[i];
      rr += reranked[i];
      bu += buffered[i];
    }
    w.last.scanned = sc;
    w.last.probed = pr;
    w.last.reranked = rr;
    w.last.buffered = bu;
  }
  if (t) {
    t->route += (uint64_t)((w.last.ms_prep + w.last.ms_route_gemm + w.last.ms_route_select) * 1e6);
    t->scan += (uint64_t)((w.last.ms_scan + w.last.ms_cut) * 1e6);
    t->rerank += (uint64_t)(w.last.ms_rerank * 1e6);
    t->tier2 += (uint64_t)(w.last.ms_tier2 * 1e6);
    t->scanned += w.last.scanned;
    t->probed += w.last.probed;
    t->reranked += w.last.reranked;
  }
  // queries whose candidate buffer filled up run again, in batches, with the exact bound
  const sg_stats saved = w.last;
  uint32_t retry_launches = 0;
  std::vector<uint32_t> redo;
  for (uint32_t i = 0; i < nq; i++)
    if (ovf[i]) redo.push_back(i);
  if (!redo.empty()) {
    uint32_t per = (uint32_t)redo.size();
    uint32_t fcap = full_cap(h, cfg, p, per);
    while (per > 1 && (uint64_t)per * fcap * sizeof(uint4) > cfg.cbuf_budget) {
      per = (per + 1) / 2;
      fcap = full_cap(h, cfg, p, per);
    }
    std::vector<float> hq768, hq256;
    std::vector<float> osc((size_t)per * std::max<uint32_t>(k, 1));
    std::vector<uint32_t> oid((size_t)per * std::max<uint32_t>(k, 1)), on(per);
    for (size_t s0 = 0; s0 < redo.size(); s0 += per) {
      const uint32_t m = (uint32_t)std::min<size_t>(per, redo.size() - s0);
      if ((rc = ensure_ws(h, c, m, p, fcap))) return rc;
      cudaMemcpyKind ik = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault;
      for (uint32_t j = 0; j < m; j++) {
        const uint32_t i = redo[s0 + j];
        CK(cudaMemcpyAsync(w.q768 + (size_t)j * SG_DIM, q768 + (size_t)i * SG_DIM, SG_DIM * 4, ik, c.stream));
        if (q256)
          CK(cudaMemcpyAsync(w.q256 + (size_t)j * SG_PDIM, q256 + (size_t)i * SG_PDIM, SG_PDIM * 4, ik, c.stream));
      }
      if ((rc = stage_allow(c, allow, allow_words, allow_dev, &d_allow))) return rc;
      if ((rc = run_pipeline(h, cfg, c, m, p, q256 != nullptr, d_allow, allow_words, kToSearch, false,
                             rp)))
        return rc;
      std::vector<uint8_t> o1(m);
      CK(cudaMemcpyAsync(o1.data(), w.overflow, m, cudaMemcpyDeviceToHost, c.stream));
      for (uint32_t j = 0; j < m; j++) {
        const uint32_t i = redo[s0 + j];
        if (k) {
          CK(cudaMemcpyAsync(out_sc + (size_t)i * k, w.out_sc + (size_t)j * k, k * 4, okind, c.stream));
          CK(cudaMemcpyAsync(out_id + (size_t)i * k, w.out_id + (size_t)j * k, k * 4, okind, c.stream));
        }
        CK(cudaMemcpyAsync(out_n + i, w.out_n + j, 4, okind, c.stream));
      }
      CK(cudaStreamSynchronize(c.stream));
      for (uint32_t j = 0; j < m; j++)
        if (o1[j]) return fail(SG_ERR_INVALID, "candidate buffer overflow at the exact bound");
      retry_launches += w.last.launches;
    }
    if ((rc = ensure_ws(h, c, nq, p, cap))) return rc;
  }
  w.last = saved;
  w.last.launches += retry_launches;
  w.last.retried = (uint32_t)redo.size();
  return SG_OK;
}

// filter::search Plan::Brute (src/filter.rs:95-105): exact int8 scores of every allowed row, in
// query batches whose score matrix stays under 1 GiB.
int brute_impl(sg_index* h, const sg::Config& cfg, sg::Ctx& c, const sg_filter* f, uint32_t nq,
               const float* q768, const float* q256, const sg_params& p, float* out_sc,
               uint32_t* out_id, uint32_t* out_n, sg_timing* t) {
  int rc;
  if ((rc = check_params(h, &p))) return rc;
  if (nq == 0) return SG_OK;
  if (!q768) return fail(SG_ERR_INVALID, "q768 is null");
  CK(cudaSetDevice(h->ix.device));
  const uint32_t R = (uint32_t)f->nrows;
  const uint32_t per = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(nq, (256ull << 20) / std::max<uint64_t>(R, 1)));
  if ((rc = ensure_ws(h, c, per, p, 1))) return rc;
  sg::Workspace& w = c.ws;
  if ((uint64_t)per * R > w.brute_cap) {
    dfree(w.brute);
    w.brute_cap = 0;
    if ((rc = dalloc(&w.brute, (size_t)per * R))) return rc;
    w.brute_cap = (uint64_t)per * R;
  }
  const bool timed = t != nullptr || cfg.timing;
  if (timed && !w.events) {
    for (auto& e : w.ev) CK(cudaEventCreate(&e));
    w.events = true;
  }
  uint32_t launches = 0;
  float ms = 0.0f;
  for (uint32_t q0 = 0; q0 < nq; q0 += per) {
    const uint32_t m = std::min(per, nq - q0);
    if ((rc = stage_inputs(c, m, q768 + (size_t)q0 * SG_DIM, q256 ? q256 + (size_t)q0 * SG_PDIM : nullptr,
                           false)))
      return rc;
    if (timed) CK(cudaEventRecord(w.ev[0], c.stream));
    if (!q256) {
      sg::launch_prefix(w, m, c.stream);
      launches++;
    }
    sg::launch_prep(h->ix, w, m, c.stream);
    launches += 1 + sg::launch_brute(h->ix, w, m, f->rows, R, p.k, w.brute, c.stream);
    if (timed) CK(cudaEventRecord(w.ev[6], c.stream));
    CK(cudaGetLastError());
    if (p.k) {
      CK(cudaMemcpyAsync(out_sc + (size_t)q0 * p.k, w.out_sc, (size_t)m * p.k * 4, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(out_id + (size_t)q0 * p.k, w.out_id, (size_t)m * p.k * 4, cudaMemcpyDeviceToHost, c.stream));
    }
    CK(cudaMemcpyAsync(out_n + q0, w.out_n, (size_t)m * 4, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (timed) {
      float e = 0.0f;
      CK(cudaEventElapsedTime(&e, w.ev[0], w.ev[6]));
      ms += e;
    }
  }
  w.last = sg_stats();
  w.last.launches = launches;
  w.last.reranked = (uint64_t)nq * R;
  if (timed) {
    w.last.ms_rerank = ms;
    w.last.ms_total = ms;
  }
  if (t) {
    t->rerank += (uint64_t)(ms * 1e6);
    t->reranked += (uint64_t)nq * R;
  }
  return SG_OK;
}

bool read_file(const std::string& path, std::vector<char>& out, bool optional, int* rc) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    if (!optional) *rc = fail(SG_ERR_IO, "cannot open " + path);
    return false;
  }
  std::streamsize n = f.tellg();
  f.seekg(0);
  out.resize((size_t)n);
  if (n && !f.read(out.data(), n)) {
    *rc = fail(SG_ERR_IO, "cannot read " + path);
    return false;
  }
  return true;
}

}  // namespace

namespace sg {
// Read-only views of an open index for entry points that live in other translation units.
const DevIndex* index_arrays(const sg_index* h) { return &h->ix; }
Config index_config(const sg_index* h) {
  std::lock_guard<std::mutex> g(h->cfg_mu);
  Config c = h->cfg;
  c.timing = h->timing_on.load(std::memory_order_relaxed);
  return c;
}
int index_sms(const sg_index* h) { return h->sms; }
int index_check_params(const sg_index* h, const sg_params* p) { return check_params(h, p); }

// ---- execution-context entry points for the serving loop (serve.cu) -------------------------
int ctx_prepare(sg_index* h, const Config& cfg, Ctx& c, uint32_t nq, const sg_params& p) {
  int rc;
  if ((rc = check_params(h, &p))) return rc;
  CK(cudaSetDevice(h->ix.device));
  return ensure_ws(h, c, nq, p, batch_cap(h, cfg, p, nq));
}

int ctx_launch(sg_index* h, const Config& cfg, Ctx& c, uint32_t nq, const sg_params& p, bool have_q256) {
  return run_pipeline(h, cfg, c, nq, p, have_q256, nullptr, 0, kToSearch, false);
}

int ctx_search_one(sg_index* h, const Config& cfg, Ctx& c, const float* q768, const float* q256,
                   const sg_params& p, const uint64_t* d_allow, uint64_t allow_words, float* out_sc,
                   uint32_t* out_id, uint32_t* out_n) {
  Config one = cfg;
  one.timing = false;
  return search_impl(h, one, c, 1, q768, q256, p, d_allow, allow_words, out_sc, out_id, out_n, nullptr,
                     false, true);
}

void free_ctx(Ctx& c) {
  if (c.stream) cudaStreamSynchronize(c.stream);
  drop_graphs(c);
  free_ws(c.ws);
  if (c.order_ev) cudaEventDestroy(c.order_ev);
  c.order_ev = nullptr;
  if (c.stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
}

// ---- live indexes (live.cu) ---------------------------------------------------------------
// Grows a device array from `have` to `want` elements, keeping its first `have` (device copy).
template <typename T>
static int grow(T*& p, size_t have, size_t want) {
  if (!p) return SG_OK;
  T* q = nullptr;
  int rc = dalloc(&q, want);
  if (rc) return rc;
  if (have) CK(cudaMemcpy(q, p, have * sizeof(T), cudaMemcpyDeviceToDevice));
  if (want > have) CK(cudaMemset(q + have, 0, (want - have) * sizeof(T)));
  dfree(p);
  p = q;
  return SG_OK;
}

int index_make_live(sg_index* h, uint64_t max_rows, uint64_t block_cap) {
  DevIndex& x = h->ix;
  if (x.live) return fail(SG_ERR_INVALID, "the index is live already");
  if (x.global) return fail(SG_ERR_UNSUPPORTED, "live updates need a RaBitQ index (src/live.rs:168)");
  if (2ull * x.kc > 4096ull * 1024) return fail(SG_ERR_INVALID, "too many clusters for a live index");
  if ((x.nblocks + block_cap) * SG_BLOCK >= 0xFFFFFFFFull) return fail(SG_ERR_INVALID, "more than 2^32 slots");
  CK(cudaSetDevice(x.device));
  CK(cudaDeviceSynchronize());
  const size_t nb = x.nblocks, nb2 = nb + block_cap, n = x.n, n2 = n + max_rows;
  int rc;
  if ((rc = grow(x.blocks, nb * SG_BLOCK_BYTES, nb2 * SG_BLOCK_BYTES)) ||
      (rc = grow(x.blocks_tc, nb * 256, nb2 * 256)) || (rc = grow(x.mul, nb * SG_BLOCK, nb2 * SG_BLOCK)) ||
      (rc = grow(x.err, nb * SG_BLOCK, nb2 * SG_BLOCK)) || (rc = grow(x.ids, nb * SG_BLOCK, nb2 * SG_BLOCK)) ||
      (rc = grow(x.rerank, n * SG_DIM, n2 * SG_DIM)) || (rc = grow(x.norm256, n, n2)) ||
      (rc = grow(x.t2_codes, n * SG_TIER2_BYTES, n2 * SG_TIER2_BYTES)) || (rc = grow(x.t2_norm, n, n2)) ||
      (rc = grow(x.codes, n * SG_CODE_BYTES, n2 * SG_CODE_BYTES)))
    return rc;
  // clusters kc..2kc-1: the delta lists, empty, after the base blocks
  const uint32_t kc = x.kc;
  x.h_block_off.resize(2 * (size_t)kc + 1, x.h_block_off[kc]);
  x.h_clen.resize(2 * (size_t)kc, 0);
  std::vector<uint32_t> boff32(2 * (size_t)kc + 1);
  for (size_t c = 0; c < boff32.size(); c++) boff32[c] = (uint32_t)x.h_block_off[c];
  dfree(x.block_off);
  dfree(x.clen);
  if ((rc = upload(&x.block_off, boff32.data(), boff32.size())) ||
      (rc = upload(&x.clen, x.h_clen.data(), x.h_clen.size())))
    return rc;
  x.k = 2 * kc;
  x.live = true;
  x.nslots = nb2 * SG_BLOCK;
  {
    std::lock_guard<std::mutex> g(h->cfg_mu);
    set_cluster_bounds(x, h->cfg.small_chunk_blocks);
    h->cfg.gen++;
  }
  // the default context's workspace is sized for the old cluster count
  free_ws(h->def.ws);
  drop_graphs(h->def);
  h->def.gen++;
  return SG_OK;
}

int index_set_delta(sg_index* h, const uint32_t* nb_of, const uint32_t* clen_of, const uint8_t* blocks,
                    const float* mul, const float* err, const uint32_t* ids, uint64_t nblocks) {
  DevIndex& x = h->ix;
  const uint32_t kc = x.kc;
  const uint64_t b0 = x.nblocks;
  if (b0 + nblocks > x.nslots / SG_BLOCK) return fail(SG_ERR_OOM, "the live index's delta lists are full");
  CK(cudaSetDevice(x.device));
  cudaStream_t st = h->def.stream;
  CK(cudaStreamSynchronize(st));
  if (nblocks) {
    CK(cudaMemcpy(x.blocks + b0 * SG_BLOCK_BYTES, blocks, nblocks * SG_BLOCK_BYTES, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x.mul + b0 * SG_BLOCK, mul, nblocks * SG_BLOCK * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x.err + b0 * SG_BLOCK, err, nblocks * SG_BLOCK * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x.ids + b0 * SG_BLOCK, ids, nblocks * SG_BLOCK * 4, cudaMemcpyHostToDevice));
    sg::transcode_tc(x.blocks + b0 * SG_BLOCK_BYTES, nblocks, x.blocks_tc + b0 * 256, st);
    CK(cudaGetLastError());
  }
  uint64_t off = b0;
  for (uint32_t c = 0; c < kc; c++) {
    x.h_block_off[kc + c] = off;
    x.h_clen[kc + c] = clen_of[c];
    off += nb_of[c];
  }
  x.h_block_off[2 * (size_t)kc] = off;
  std::vector<uint32_t> boff32(kc + 1);
  for (uint32_t c = 0; c <= kc; c++) boff32[c] = (uint32_t)x.h_block_off[kc + c];
  CK(cudaMemcpyAsync(x.block_off + kc, boff32.data(), (kc + 1) * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(x.clen + kc, x.h_clen.data() + kc, (size_t)kc * 4, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  std::lock_guard<std::mutex> g(h->cfg_mu);
  set_cluster_bounds(x, h->cfg.small_chunk_blocks);
  h->cfg.gen++;  // captured pipelines baked in the old bounds: their keys go stale
  return SG_OK;
}

int index_search_allow(sg_index* h, uint32_t nq, const float* q768, const float* q256, const sg_params& p,
                       const uint64_t* d_allow, uint64_t allow_words, float* out_sc, uint32_t* out_id,
                       uint32_t* out_n) {
  std::lock_guard<std::mutex> g(h->mu);
  return search_impl(h, index_config(h), h->def, nq, q768, q256, p, d_allow, allow_words, out_sc, out_id, out_n,
                     nullptr, false, true);
}

// Device scratch of a batch of nq queries with params p (the workspace ensure_ws grows to).
uint64_t ctx_bytes(const sg_index* h, const Config& cfg, const sg_params& p, uint32_t nq) {
  const uint64_t P = sg::probe_stride(h->ix, p.nprobe);
  const uint64_t cap = batch_cap(h, cfg, p, nq);
  const uint64_t per_q = SG_DIM * 4 * 2 + SG_PDIM * 5 + 1024 + 64 + (uint64_t)h->ix.k * 4 + P * 16 +
                         cap * 12 + (uint64_t)std::max<uint32_t>(p.cand, 1) * 20 +
                         (uint64_t)std::max<uint32_t>(p.k, 1) * 8 + 64;
  const uint64_t items = (uint64_t)h->ix.h_chunks_desc_prefix[P] * 16;
  return (uint64_t)nq * (per_q + items) + (uint64_t)h->ix.k * 16 + 4096;
}
}  // namespace sg

extern "C" {

const char* sg_last_error(void) { return sg::last_error().c_str(); }

const char* sg_version(void) { return "sieve_gpu 0.1 (sm_100a)"; }

int sg_open_ivf_arrays(const sg_ivf_arrays* a, int device, sg_index** out) {
  try {
    return build_index(a, device, out);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_open_ivf(const char* ingest_dir, const char* index_dir, int device, sg_index** out) {
  if (!ingest_dir || !index_dir || !out) return fail(SG_ERR_INVALID, "null argument");
  try {
    std::string I(ingest_dir), X(index_dir);
    std::vector<char> cent, boff, ids, blocks, fac, rot, sig, t2c, t2n, rer, n256, qs, codes;
    int rc = SG_OK;
    if (!read_file(X + "/centroids.f32", cent, false, &rc) ||
        !read_file(X + "/block_off.u64", boff, false, &rc) ||
        !read_file(X + "/ids.u32", ids, false, &rc) ||
        !read_file(X + "/blocks.bin", blocks, false, &rc) ||
        !read_file(I + "/rerank.i8", rer, false, &rc) ||
        !read_file(I + "/norm256.f32", n256, false, &rc) ||
        !read_file(I + "/quant.f32", qs, false, &rc))
      return rc;
    bool has_codes = read_file(I + "/codes.bin", codes, true, &rc);
    bool has_rot = read_file(X + "/rotation.f32", rot, true, &rc);
    bool has_fac = read_file(X + "/factors.f32", fac, true, &rc);
    bool has_t2 = read_file(X + "/tier2.bin", t2c, true, &rc) &&
                  read_file(X + "/tier2.sigma", sig, false, &rc) &&
                  read_file(X + "/tier2.norm", t2n, false, &rc);
    if (rc) return rc;
    sg_ivf_arrays a;
    memset(&a, 0, sizeof a);
    a.n = n256.size() / 4;
    a.k = (uint32_t)(cent.size() / (4 * SG_PDIM));
    if (boff.size() != 8 * ((size_t)a.k + 1))
      return fail(SG_ERR_INVALID, "block_off.u64 does not match centroids");
    if (rer.size() != a.n * SG_DIM) return fail(SG_ERR_INVALID, "rerank.i8 size");
    if (qs.size() != 4 * SG_DIM) return fail(SG_ERR_INVALID, "quant.f32 size");
    a.centroids = (const float*)cent.data();
    a.block_off = (const uint64_t*)boff.data();
    uint64_t nb = a.block_off[a.k];
    if (ids.size() != nb * SG_BLOCK * 4 || blocks.size() != nb * SG_BLOCK_BYTES)
      return fail(SG_ERR_INVALID, "ids.u32 / blocks.bin do not match block_off.u64");
    a.ids = (const uint32_t*)ids.data();
    a.blocks = (const uint8_t*)blocks.data();
    if (has_fac) {
      if (fac.size() != nb * SG_BLOCK * 8) return fail(SG_ERR_INVALID, "factors.f32 size");
      a.factors = (const float*)fac.data();
    }
    if (has_rot) {
      if (rot.size() != 3 * SG_PDIM * 4) return fail(SG_ERR_INVALID, "rotation.f32 is not 3 x 256");
      a.rotation = (const float*)rot.data();
    }
    if (has_t2) {
      if (t2c.size() != a.n * SG_TIER2_BYTES || t2n.size() != a.n * 4 || sig.size() != SG_PDIM * 4)
        return fail(SG_ERR_INVALID, "tier2 file sizes");
      a.tier2_codes = (const uint8_t*)t2c.data();
      a.tier2_norm = (const float*)t2n.data();
      a.tier2_sigma = (const float*)sig.data();
    }
    a.rerank = (const int8_t*)rer.data();
    a.norm256 = (const float*)n256.data();
    if (has_codes) {
      if (codes.size() != a.n * SG_CODE_BYTES) return fail(SG_ERR_INVALID, "codes.bin size");
      a.codes = (const uint8_t*)codes.data();
    }
    a.quant_scale = (const float*)qs.data();
    return build_index(&a, device, out);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_close(sg_index* h) {
  if (!h) return SG_OK;
  cudaSetDevice(h->ix.device);
  if (h->def.stream) cudaStreamSynchronize(h->def.stream);
  drop_graphs(h->def);
  free_ws(h->def.ws);
  free_index(h->ix);
  if (h->def.stream) cudaStreamDestroy(h->def.stream);
  delete h;
  return SG_OK;
}

int sg_index_info(const sg_index* h, uint32_t* k, uint64_t* n, uint64_t* nblocks,
                  uint32_t* has_tier2) {
  if (!h) return fail(SG_ERR_INVALID, "null index");
  if (k) *k = h->ix.kc;
  if (n) *n = h->ix.n;
  if (nblocks) *nblocks = h->ix.nblocks;
  if (has_tier2) *has_tier2 = h->ix.has_t2;
  return SG_OK;
}

int sg_set_route_precision(sg_index* h, int precision) {
  if (!h) return fail(SG_ERR_INVALID, "null index");
  if (precision != SG_ROUTE_FP32 && precision != SG_ROUTE_BF16)
    return fail(SG_ERR_INVALID, "precision must be SG_ROUTE_FP32 or SG_ROUTE_BF16");
  std::lock_guard<std::mutex> lk(h->cfg_mu);
  if (h->cfg.route_precision != precision) {
    h->cfg.route_precision = precision;
    h->cfg.gen++;  // captured pipelines launch the other routing kernel: their keys go stale
  }
  return SG_OK;
}

int sg_set_timing(sg_index* h, int on) {
  if (!h) return fail(SG_ERR_INVALID, "null index");
  h->timing_on.store(on != 0, std::memory_order_relaxed);
  return SG_OK;
}

int sg_last_stats(const sg_index* h, sg_stats* out) {
  if (!h || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = h->def.ws.last;
  return SG_OK;
}

int sg_search(sg_index* h, uint32_t nq, const float* q768, const float* q256,
              const sg_params* params, const uint64_t* allow_bits, uint64_t allow_words,
              float* out_scores, uint32_t* out_ids, uint32_t* out_counts, sg_timing* timing) {
  if (!h || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  return search_impl(h, sg::index_config(h), h->def, nq, q768, q256, *params, allow_bits, allow_words,
                     out_scores, out_ids, out_counts, timing, false);
}

}  // extern "C"

namespace {
// sg_search_device on context c: c's stream waits for the caller's stream (one reusable event),
// and the call returns after the results are in the caller's device buffers.
int search_device_on(sg_index* h, sg::Ctx& c, uint32_t nq, const float* d_q768, const float* d_q256,
                     const sg_params* params, const uint64_t* d_allow_bits, uint64_t allow_words,
                     float* d_out_scores, uint32_t* d_out_ids, uint32_t* d_out_counts, void* stream) {
  CK(cudaSetDevice(h->ix.device));
  if (!c.order_ev) CK(cudaEventCreateWithFlags(&c.order_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(c.order_ev, (cudaStream_t)stream));
  CK(cudaStreamWaitEvent(c.stream, c.order_ev, 0));
  return search_impl(h, sg::index_config(h), c, nq, d_q768, d_q256, *params, d_allow_bits, allow_words,
                     d_out_scores, d_out_ids, d_out_counts, nullptr, true);
}
}  // namespace

extern "C" {

int sg_search_device(sg_index* h, uint32_t nq, const float* d_q768, const float* d_q256,
                     const sg_params* params, const uint64_t* d_allow_bits, uint64_t allow_words,
                     float* d_out_scores, uint32_t* d_out_ids, uint32_t* d_out_counts,
                     void* stream) {
  if (!h || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  return search_device_on(h, h->def, nq, d_q768, d_q256, params, d_allow_bits, allow_words, d_out_scores,
                          d_out_ids, d_out_counts, stream);
}

int sg_context_open(sg_index* h, sg_context** out) {
  if (!h || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    std::unique_ptr<sg_context> c(new sg_context());
    c->h = h;
    CK(cudaSetDevice(h->ix.device));
    CK(cudaStreamCreateWithFlags(&c->ctx.stream, cudaStreamNonBlocking));
    *out = c.release();
    return SG_OK;
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_context_close(sg_context* c) {
  if (!c) return SG_OK;
  {
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->h->ix.device);
    sg::free_ctx(c->ctx);
  }
  delete c;
  return SG_OK;
}

int sg_search_ctx(sg_context* c, uint32_t nq, const float* q768, const float* q256,
                  const sg_params* params, const uint64_t* allow_bits, uint64_t allow_words,
                  float* out_scores, uint32_t* out_ids, uint32_t* out_counts, sg_timing* timing) {
  if (!c || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(c->mu);
  try {
    return search_impl(c->h, sg::index_config(c->h), c->ctx, nq, q768, q256, *params, allow_bits,
                       allow_words, out_scores, out_ids, out_counts, timing, false);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_search_device_ctx(sg_context* c, uint32_t nq, const float* d_q768, const float* d_q256,
                         const sg_params* params, const uint64_t* d_allow_bits, uint64_t allow_words,
                         float* d_out_scores, uint32_t* d_out_ids, uint32_t* d_out_counts,
                         void* stream) {
  if (!c || !params) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(c->mu);
  try {
    return search_device_on(c->h, c->ctx, nq, d_q768, d_q256, params, d_allow_bits, allow_words,
                            d_out_scores, d_out_ids, d_out_counts, stream);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_context_last_stats(sg_context* c, sg_stats* out) {
  if (!c || !out) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(c->mu);
  *out = c->ctx.ws.last;
  return SG_OK;
}

int sg_route(sg_index* h, uint32_t nq, const float* q256, const sg_params* params,
             float* out_scores, uint32_t* out_clusters, uint32_t* out_counts) {
  if (!h || !params || !q256) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  int rc;
  if ((rc = check_params(h, params))) return rc;
  if (nq == 0) return SG_OK;
  CK(cudaSetDevice(h->ix.device));
  if ((rc = ensure_ws(h, h->def, nq, *params, 1))) return rc;
  if ((rc = stage_inputs(h->def, nq, nullptr, q256, false))) return rc;
  sg::Workspace& w = h->def.ws;
  cudaStream_t st = h->def.stream;
  CK(cudaMemsetAsync(w.counters, 0, 32, st));
  sg::launch_prep(h->ix, w, nq, st);
  const sg::Config cfg = sg::index_config(h);
  CK(sg::launch_route_scores(h->ix, w, nq, cfg.route_precision, st));
  sg::launch_route_select(h->ix, w, nq, *params, cfg.route_precision, cfg.chunk_blocks, cfg.seed_blocks,
                          true, st);
  CK(cudaGetLastError());
  const uint32_t P = std::min<uint32_t>(params->nprobe, h->ix.k);
  if (P) {
    CK(cudaMemcpyAsync(out_scores, w.probe_sc, (size_t)nq * P * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out_clusters, w.probe_cl, (size_t)nq * P * 4, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaMemcpyAsync(out_counts, w.probe_n, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, w.counters + 2, 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (status & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "routing GEMM: a tensor-core wait ran out");
  return SG_OK;
}

int sg_route_scores(sg_index* h, uint32_t nq, const float* q256, float* out_scores) {
  if (!h || !q256 || !out_scores) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  int rc;
  if (nq == 0) return SG_OK;
  CK(cudaSetDevice(h->ix.device));
  sg_params p;
  memset(&p, 0, sizeof p);
  p.nprobe = 1;
  p.cand = 1;
  p.k = 1;
  if ((rc = ensure_ws(h, h->def, nq, p, 1))) return rc;
  if ((rc = stage_inputs(h->def, nq, nullptr, q256, false))) return rc;
  sg::Workspace& w = h->def.ws;
  cudaStream_t st = h->def.stream;
  CK(cudaMemsetAsync(w.counters, 0, 32, st));
  CK(sg::launch_route_scores(h->ix, w, nq, sg::index_config(h).route_precision, st));
  CK(cudaGetLastError());
  uint32_t status = 0;
  CK(cudaMemcpyAsync(out_scores, w.scores, (size_t)nq * h->ix.kc * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&status, w.counters + 2, 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (status & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "routing GEMM: a tensor-core wait ran out");
  return SG_OK;
}

int sg_candidates(sg_index* h, uint32_t nq, const float* q256, const sg_params* params,
                  const uint64_t* allow_bits, uint64_t allow_words, float* out_est,
                  uint32_t* out_ids, float* out_err, uint32_t* out_counts) {
  if (!h || !params || !q256) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  int rc;
  if ((rc = check_params(h, params))) return rc;
  if (nq == 0) return SG_OK;
  CK(cudaSetDevice(h->ix.device));
  const sg_params& p = *params;
  const sg::Config cfg = sg::index_config(h);
  uint32_t cap = full_cap(h, cfg, p, 1);
  for (uint32_t q0 = 0; q0 < nq; q0++) {
    // one query at a time with the exact buffer bound: this entry point is for parity checks
    if ((rc = ensure_ws(h, h->def, 1, p, cap))) return rc;
    if ((rc = stage_inputs(h->def, 1, nullptr, q256 + (size_t)q0 * SG_PDIM, false))) return rc;
    const uint64_t* d_allow;
    if ((rc = stage_allow(h->def, allow_bits, allow_words, false, &d_allow))) return rc;
    if ((rc = run_pipeline(h, cfg, h->def, 1, p, true, d_allow, allow_words, kToCandidates, false))) return rc;
    sg::Workspace& w = h->def.ws;
    const uint32_t c = std::max<uint32_t>(p.cand, 1);
    if (p.cand) {
      CK(cudaMemcpyAsync(out_est + (size_t)q0 * c, w.cest, (size_t)c * 4, cudaMemcpyDeviceToHost, h->def.stream));
      CK(cudaMemcpyAsync(out_ids + (size_t)q0 * c, w.cid, (size_t)c * 4, cudaMemcpyDeviceToHost, h->def.stream));
      CK(cudaMemcpyAsync(out_err + (size_t)q0 * c, w.cerr, (size_t)c * 4, cudaMemcpyDeviceToHost, h->def.stream));
    }
    CK(cudaMemcpyAsync(out_counts + q0, w.cn, 4, cudaMemcpyDeviceToHost, h->def.stream));
    uint8_t o = 0;
    CK(cudaMemcpyAsync(&o, w.overflow, 1, cudaMemcpyDeviceToHost, h->def.stream));
    CK(cudaStreamSynchronize(h->def.stream));
    if (o) return fail(SG_ERR_INVALID, "candidate buffer overflow at the exact bound");
    // the device list is unordered; Index::candidates returns it in row order
    if (p.cand) {
      const uint32_t n = out_counts[q0];
      float* e = out_est + (size_t)q0 * c;
      uint32_t* id = out_ids + (size_t)q0 * c;
      float* er = out_err + (size_t)q0 * c;
      std::vector<uint32_t> ord(n);
      for (uint32_t i = 0; i < n; i++) ord[i] = i;
      std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return id[x] < id[y]; });
      std::vector<float> e2(n), er2(n);
      std::vector<uint32_t> id2(n);
      for (uint32_t i = 0; i < n; i++) {
        e2[i] = e[ord[i]];
        id2[i] = id[ord[i]];
        er2[i] = er[ord[i]];
      }
      std::copy(e2.begin(), e2.end(), e);
      std::copy(id2.begin(), id2.end(), id);
      std::copy(er2.begin(), er2.end(), er);
    }
  }
  return SG_OK;
}

int sg_candidates_probes(sg_index* h, uint32_t nq, const float* q256, const float* probe_scores,
                         const uint32_t* probe_clusters, const uint32_t* probe_counts, const sg_params* params,
                         const uint64_t* allow_bits, uint64_t allow_words, float* out_est, uint32_t* out_ids,
                         float* out_err, uint32_t* out_counts) {
  if (!h || !params || (nq && (!q256 || !probe_counts || !out_counts)))
    return fail(SG_ERR_INVALID, "null argument");
  int rc;
  if ((rc = check_params(h, params))) return rc;
  if (nq == 0) return SG_OK;
  const sg_params& p = *params;
  if (h->ix.live) return fail(SG_ERR_UNSUPPORTED, "probe lists of a live index come from its own routing");
  const uint32_t P = sg::probe_stride(h->ix, p.nprobe);
  for (uint32_t q = 0; q < nq; q++) {
    if (probe_counts[q] > P) return fail(SG_ERR_INVALID, "a probe list is longer than min(nprobe, k)");
    for (uint32_t r = 0; r < probe_counts[q]; r++)
      if (probe_clusters[(size_t)q * P + r] >= h->ix.k) return fail(SG_ERR_INVALID, "probe cluster >= k");
  }
  if (P && (!probe_scores || !probe_clusters)) return fail(SG_ERR_INVALID, "null probe list");
  if (p.cand && (!out_est || !out_ids || !out_err)) return fail(SG_ERR_INVALID, "null output");
  std::lock_guard<std::mutex> g(h->mu);
  try {
    CK(cudaSetDevice(h->ix.device));
    const sg::Config cfg = sg::index_config(h);
    sg::Ctx& c = h->def;
    sg::Workspace& w = c.ws;
    const uint32_t cw = std::max<uint32_t>(p.cand, 1);
    RoutePlan rp;
    rp.given = true;
    // queries [q0, q0 + m) with per-query buffers of `cap` entries; their overflow flags in ovf
    auto run = [&](uint32_t q0, uint32_t m, uint32_t cap, uint8_t* ovf) -> int {
      int rc2;
      if ((rc2 = ensure_ws(h, c, m, p, cap))) return rc2;
      if ((rc2 = stage_inputs(c, m, nullptr, q256 + (size_t)q0 * SG_PDIM, false))) return rc2;
      if (P) {
        CK(cudaMemcpyAsync(w.probe_sc, probe_scores + (size_t)q0 * P, (size_t)m * P * 4, cudaMemcpyHostToDevice, c.stream));
        CK(cudaMemcpyAsync(w.probe_cl, probe_clusters + (size_t)q0 * P, (size_t)m * P * 4, cudaMemcpyHostToDevice,
                           c.stream));
      }
      CK(cudaMemcpyAsync(w.probe_n, probe_counts + q0, (size_t)m * 4, cudaMemcpyHostToDevice, c.stream));
      const uint64_t* d_allow;
      if ((rc2 = stage_allow(c, allow_bits, allow_words, false, &d_allow))) return rc2;
      if ((rc2 = run_pipeline(h, cfg, c, m, p, true, d_allow, allow_words, kToCandidates, false, rp))) return rc2;
      if (p.cand) {
        CK(cudaMemcpyAsync(out_est + (size_t)q0 * cw, w.cest, (size_t)m * cw * 4, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaMemcpyAsync(out_ids + (size_t)q0 * cw, w.cid, (size_t)m * cw * 4, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaMemcpyAsync(out_err + (size_t)q0 * cw, w.cerr, (size_t)m * cw * 4, cudaMemcpyDeviceToHost, c.stream));
      }
      CK(cudaMemcpyAsync(out_counts + q0, w.cn, (size_t)m * 4, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(ovf, w.overflow, m, cudaMemcpyDeviceToHost, c.stream));
      uint32_t status = 0;
      CK(cudaMemcpyAsync(&status, w.counters + 2, 4, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaStreamSynchronize(c.stream));
      if (status & sg::kStatusOverflow) return fail(SG_ERR_INVALID, "work queue overflow");
      if (status & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "a tensor-core wait ran out (scan)");
      return SG_OK;
    };
    std::vector<uint8_t> ovf(nq);
    if ((rc = run(0, nq, batch_cap(h, cfg, p, nq), ovf.data()))) return rc;
    // a query whose buffer filled up runs again alone with its exact bound
    for (uint32_t q = 0; q < nq; q++) {
      if (!ovf[q]) continue;
      uint8_t o1 = 0;
      if ((rc = run(q, 1, full_cap(h, cfg, p, 1), &o1))) return rc;
      if (o1) return fail(SG_ERR_INVALID, "candidate buffer overflow at the exact bound");
    }
    // the device lists are unordered; Index::candidates returns them in row order
    for (uint32_t q = 0; q < nq && p.cand; q++) {
      const uint32_t n = out_counts[q];
      float* e = out_est + (size_t)q * cw;
      uint32_t* id = out_ids + (size_t)q * cw;
      float* er = out_err + (size_t)q * cw;
      std::vector<uint32_t> ord(n);
      for (uint32_t i = 0; i < n; i++) ord[i] = i;
      std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return id[x] < id[y]; });
      std::vector<float> e2(n), er2(n);
      std::vector<uint32_t> id2(n);
      for (uint32_t i = 0; i < n; i++) {
        e2[i] = e[ord[i]];
        id2[i] = id[ord[i]];
        er2[i] = er[ord[i]];
      }
      std::copy(e2.begin(), e2.end(), e);
      std::copy(id2.begin(), id2.end(), id);
      std::copy(er2.begin(), er2.end(), er);
    }
    return SG_OK;
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_rerank(sg_index* h, uint32_t nq, const float* q768, const float* q256, const float* cand_est,
              const uint32_t* cand_ids, const float* cand_err, const uint32_t* cand_counts, uint32_t cand_stride,
              const sg_params* params, float* out_scores, uint32_t* out_ids, uint32_t* out_counts) {
  if (!h || !params || (nq && (!q768 || !cand_counts || !out_counts))) return fail(SG_ERR_INVALID, "null argument");
  sg_params p = *params;
  p.cand = cand_stride;
  int rc;
  if ((rc = check_params(h, &p))) return rc;
  if (nq == 0) return SG_OK;
  if (cand_stride && (!cand_est || !cand_ids)) return fail(SG_ERR_INVALID, "null candidate list");
  if (p.k && (!out_scores || !out_ids)) return fail(SG_ERR_INVALID, "null output");
  for (uint32_t q = 0; q < nq; q++) {
    if (cand_counts[q] > cand_stride) return fail(SG_ERR_INVALID, "a candidate list is longer than its stride");
    for (uint32_t i = 0; i < cand_counts[q]; i++)
      if (cand_ids[(size_t)q * cand_stride + i] >= h->ix.n) return fail(SG_ERR_INVALID, "candidate row >= n");
  }
  std::lock_guard<std::mutex> g(h->mu);
  try {
    CK(cudaSetDevice(h->ix.device));
    sg::Ctx& c = h->def;
    sg::Workspace& w = c.ws;
    if ((rc = ensure_ws(h, c, nq, p, 1))) return rc;
    if ((rc = stage_inputs(c, nq, q768, q256, false))) return rc;
    cudaStream_t st = c.stream;
    if (!q256) sg::launch_prefix(w, nq, st);
    sg::launch_prep(h->ix, w, nq, st);
    const size_t nc = (size_t)nq * cand_stride;
    if (nc) {
      CK(cudaMemcpyAsync(w.cest, cand_est, nc * 4, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(w.cid, cand_ids, nc * 4, cudaMemcpyHostToDevice, st));
      if (cand_err) CK(cudaMemcpyAsync(w.cerr, cand_err, nc * 4, cudaMemcpyHostToDevice, st));
      else CK(cudaMemsetAsync(w.cerr, 0, nc * 4, st));
    }
    CK(cudaMemcpyAsync(w.cn, cand_counts, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
    sg::launch_rerank(h->ix, w, nq, p, st, nullptr, nullptr);
    CK(cudaGetLastError());
    if (p.k) {
      CK(cudaMemcpyAsync(out_scores, w.out_sc, (size_t)nq * p.k * 4, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(out_ids, w.out_id, (size_t)nq * p.k * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaMemcpyAsync(out_counts, w.out_n, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SG_OK;
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_filter_new(sg_index* h, const uint64_t* allow_bits, uint64_t allow_words, sg_filter** out) {
  if (!h || !out || (!allow_bits && allow_words)) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  std::lock_guard<std::mutex> g(h->mu);
  CK(cudaSetDevice(h->ix.device));
  std::unique_ptr<sg_filter> f(new sg_filter());
  f->h = h;
  f->words = allow_words;
  int rc;
  auto cleanup = [&]() {
    dfree(f->allow);
    dfree(f->rows);
    dfree(f->per_cluster);
  };
  if ((rc = dalloc(&f->allow, std::max<uint64_t>(allow_words, 1))) ||
      (rc = dalloc(&f->per_cluster, std::max<uint32_t>(h->ix.k, 1)))) {
    cleanup();
    return rc;
  }
  cudaError_t e = cudaSuccess;
  if (allow_words)
    e = cudaMemcpyAsync(f->allow, allow_bits, allow_words * 8, cudaMemcpyHostToDevice, h->def.stream);
  if (e != cudaSuccess) {
    cleanup();
    return fail(SG_ERR_DEVICE, std::string("filter upload: ") + cudaGetErrorString(e));
  }
  if ((rc = sg::filter_build(h->ix, f->allow, allow_words, &f->rows, &f->nrows, f->per_cluster,
                             h->def.stream)) ||
      (rc = cudaStreamSynchronize(h->def.stream) == cudaSuccess ? SG_OK
                                                               : fail(SG_ERR_DEVICE, "filter build"))) {
    cleanup();
    return rc;
  }
  *out = f.release();
  return SG_OK;
}

int sg_filter_info(const sg_filter* f, uint64_t* nrows, uint32_t* out_per_cluster, uint32_t* out_rows) {
  if (!f) return fail(SG_ERR_INVALID, "null filter");
  if (nrows) *nrows = f->nrows;
  CK(cudaSetDevice(f->h->ix.device));
  if (out_per_cluster)
    CK(cudaMemcpy(out_per_cluster, f->per_cluster, (size_t)f->h->ix.k * 4, cudaMemcpyDeviceToHost));
  if (out_rows && f->nrows)
    CK(cudaMemcpy(out_rows, f->rows, (size_t)f->nrows * 4, cudaMemcpyDeviceToHost));
  return SG_OK;
}

int sg_filter_free(sg_filter* f) {
  if (!f) return SG_OK;
  {
    std::lock_guard<std::mutex> g(f->h->mu);
    cudaSetDevice(f->h->ix.device);
    cudaStreamSynchronize(f->h->def.stream);
    dfree(f->allow);
    dfree(f->rows);
    dfree(f->per_cluster);
  }
  delete f;
  return SG_OK;
}

int sg_plan_resolve(int plan, uint64_t allowed_rows, uint64_t n) {
  if (plan != SG_PLAN_AUTO) return plan;
  if (allowed_rows <= SG_BRUTE_MAX) return SG_PLAN_BRUTE;
  if ((double)allowed_rows >= SG_POST_MIN * (double)n) return SG_PLAN_POST;
  return SG_PLAN_EXPAND;
}

int sg_filter_search(sg_index* h, const sg_filter* f, int plan, uint64_t expand_target, uint32_t nq,
                     const float* q768, const float* q256, const sg_params* params,
                     float* out_scores, uint32_t* out_ids, uint32_t* out_counts, sg_timing* timing) {
  if (!h || !f || !params) return fail(SG_ERR_INVALID, "null argument");
  if (f->h != h) return fail(SG_ERR_INVALID, "the filter belongs to another index");
  if (plan < SG_PLAN_POST || plan > SG_PLAN_AUTO) return fail(SG_ERR_INVALID, "unknown plan");
  const int resolved = sg_plan_resolve(plan, f->nrows, h->ix.n);
  if (plan == SG_PLAN_AUTO && resolved == SG_PLAN_EXPAND) expand_target = SG_EXPAND_TARGET;
  std::lock_guard<std::mutex> g(h->mu);
  const sg::Config cfg = sg::index_config(h);
  try {
    if (resolved == SG_PLAN_BRUTE)
      return brute_impl(h, cfg, h->def, f, nq, q768, q256, *params, out_scores, out_ids, out_counts, timing);
    if (resolved == SG_PLAN_POST)
      return search_impl(h, cfg, h->def, nq, q768, q256, *params, f->allow, f->words, out_scores, out_ids,
                         out_counts, timing, false, true);
    if (h->ix.k > sg::kExpandMaxK)
      return fail(SG_ERR_UNSUPPORTED, "plan Expand needs k <= 16384 clusters");
    RoutePlan rp;
    rp.per_cluster = f->per_cluster;
    rp.target = expand_target;
    return search_impl(h, cfg, h->def, nq, q768, q256, *params, f->allow, f->words, out_scores, out_ids,
                       out_counts, timing, false, true, rp);
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, e.what());
  }
}

int sg_flat_hamming(sg_index* h, uint32_t nq, const float* q768, const float* q256, uint32_t cand,
                    uint32_t k, float* out_scores, uint32_t* out_ids, uint32_t* out_counts) {
  if (!h || (nq && (!q768 || !out_counts || (k && (!out_scores || !out_ids)))))
    return fail(SG_ERR_INVALID, "null argument");
  if (!h->ix.codes) return fail(SG_ERR_UNSUPPORTED, "the flat Hamming baseline needs codes.bin");
  if (cand > sg::kMaxCand || k > sg::kMaxCand) return fail(SG_ERR_INVALID, "cand and k must be <= 4096");
  if (nq == 0) return SG_OK;
  if (k == 0 || cand == 0) {
    memset(out_counts, 0, (size_t)nq * 4);
    return SG_OK;
  }
  std::lock_guard<std::mutex> g(h->mu);
  try {
    CK(cudaSetDevice(h->ix.device));
    sg_params p;
    memset(&p, 0, sizeof p);
    p.nprobe = 1;
    p.cand = cand;
    p.k = k;
    int rc;
    if ((rc = ensure_ws(h, h->def, nq, p, 1))) return rc;
    if ((rc = stage_inputs(h->def, nq, q768, q256, false))) return rc;
    sg::Workspace& w = h->def.ws;
    cudaStream_t st = h->def.stream;
    if (!q256) sg::launch_prefix(w, nq, st);
    sg::launch_flat_hamming(h->ix, w, nq, cand, k, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out_scores, w.out_sc, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out_ids, w.out_id, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out_counts, w.out_n, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SG_OK;
  } catch (const std::exception& e) {
    return fail(SG_ERR_OOM, std::string("host allocation: ") + e.what());
  }
}

int sg_query_prep(sg_index* h, uint32_t nq, const float* q256, uint8_t* out_tables,
                  float* out_scale, float* out_bias, float* out_a, float* out_b) {
  if (!h || !q256) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (nq == 0) return SG_OK;
  CK(cudaSetDevice(h->ix.device));
  sg_params p;
  memset(&p, 0, sizeof p);
  p.nprobe = 1;
  p.cand = 1;
  p.k = 1;
  int rc;
  if ((rc = ensure_ws(h, h->def, nq, p, 1))) return rc;
  if ((rc = stage_inputs(h->def, nq, nullptr, q256, false))) return rc;
  sg::launch_prep(h->ix, h->def.ws, nq, h->def.stream);
  CK(cudaGetLastError());
  std::vector<float4> qp(nq);
  CK(cudaMemcpyAsync(out_tables, h->def.ws.tables, (size_t)nq * 1024, cudaMemcpyDeviceToHost, h->def.stream));
  CK(cudaMemcpyAsync(qp.data(), h->def.ws.qp, nq * sizeof(float4), cudaMemcpyDeviceToHost, h->def.stream));
  CK(cudaStreamSynchronize(h->def.stream));
  for (uint32_t i = 0; i < nq; i++) {
    if (out_scale) out_scale[i] = qp[i].x;
    if (out_bias) out_bias[i] = qp[i].y;
    if (out_a) out_a[i] = qp[i].z;
    if (out_b) out_b[i] = qp[i].w;
  }
  return SG_OK;
}

int sg_lut_scan(uint32_t groups, const uint8_t* tables, const uint8_t* blocks, uint64_t nblocks,
                uint16_t* out_scores) {
  if (groups != 64 && groups != 32) return fail(SG_ERR_INVALID, "groups must be 64 or 32");
  if (!tables || (!blocks && nblocks) || (!out_scores && nblocks))
    return fail(SG_ERR_INVALID, "null argument");
  if (nblocks == 0) return SG_OK;
  uint8_t *dt = nullptr, *db = nullptr;
  uint16_t* dout = nullptr;
  int rc;
  if ((rc = dalloc(&dt, groups * 16)) || (rc = dalloc(&db, nblocks * groups * 16)) ||
      (rc = dalloc(&dout, nblocks * SG_BLOCK))) {
    dfree(dt); dfree(db); dfree(dout);
    return rc;
  }
  cudaError_t e = cudaMemcpy(dt, tables, groups * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, blocks, nblocks * groups * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sg::launch_lut_scan(groups, dt, db, nblocks, dout, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(out_scores, dout, nblocks * SG_BLOCK * 2, cudaMemcpyDeviceToHost);
  dfree(dt); dfree(db); dfree(dout);
  if (e != cudaSuccess) return fail(SG_ERR_DEVICE, std::string("sg_lut_scan: ") + cudaGetErrorString(e));
  return SG_OK;
}

int sg_get_tuning(const sg_index* h, sg_tuning* out) {
  if (!h || !out) return fail(SG_ERR_INVALID, "null argument");
  const sg::Config cfg = sg::index_config(h);
  out->tc_min_queries = cfg.tc_min_queries;
  out->chunk_blocks = cfg.chunk_blocks;
  out->scan_ctas_per_sm = cfg.scan_ctas_per_sm;
  out->seed_blocks = cfg.seed_blocks;
  out->tc_split = cfg.tc_split;
  return SG_OK;
}

int sg_set_tuning(sg_index* h, const sg_tuning* t) {
  if (!h || !t) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(h->cfg_mu);
  // chunks of at least the small-batch chunk keep the work-queue capacity bound valid
  if (t->chunk_blocks < h->cfg.small_chunk_blocks || t->chunk_blocks > sg::kMaxChunkBlocks)
    return fail(SG_ERR_INVALID, "chunk_blocks must lie in [small chunk, 512]");
  if (t->seed_blocks == 0 || t->seed_blocks > sg::kMaxChunkBlocks)
    return fail(SG_ERR_INVALID, "seed_blocks must lie in [1, 512]");
  if (t->scan_ctas_per_sm < 1 || t->scan_ctas_per_sm > 2) return fail(SG_ERR_INVALID, "scan_ctas_per_sm: 1 or 2");
  if (t->tc_min_queries == 0) return fail(SG_ERR_INVALID, "tc_min_queries must be >= 1");
  if (t->tc_split > 4096) return fail(SG_ERR_INVALID, "tc_split must be <= 4096");
  h->cfg.tc_min_queries = t->tc_min_queries;
  h->cfg.chunk_blocks = t->chunk_blocks;
  h->cfg.scan_ctas_per_sm = t->scan_ctas_per_sm;
  h->cfg.seed_blocks = t->seed_blocks;
  h->cfg.tc_split = t->tc_split;
  h->cfg.gen++;
  return SG_OK;
}

// The autotuner: coordinate descent over the batched path's shapes, timing the caller's own
// batch (device time of the whole pipeline, best of `reps` runs per candidate). Every shape
// gives identical results, so only speed is compared.
int sg_autotune(sg_index* h, uint32_t nq, const float* d_q768, const float* d_q256, const sg_params* params,
                uint32_t reps, sg_tuning* out, float* out_ms) {
  if (!h || !params || !d_q768 || nq == 0) return fail(SG_ERR_INVALID, "null argument or empty batch");
  if (nq < sg::index_config(h).small_batch)
    return fail(SG_ERR_INVALID, "the autotuner tunes batches of >= 64 queries");
  int rc;
  if ((rc = check_params(h, params))) return rc;
  CK(cudaSetDevice(h->ix.device));
  const uint32_t k = std::max<uint32_t>(params->k, 1);
  float* osc = nullptr;
  uint32_t *oid = nullptr, *on = nullptr;
  if ((rc = dalloc(&osc, (size_t)nq * k)) || (rc = dalloc(&oid, (size_t)nq * k)) || (rc = dalloc(&on, nq))) {
    dfree(osc); dfree(oid); dfree(on);
    return rc;
  }
  reps = std::max<uint32_t>(reps, 1);
  auto time_batch = [&](float* ms) -> int {
    float best = INFINITY;
    for (uint32_t r = 0; r < reps + 1; r++) {  // the first run warms the workspace
      std::lock_guard<std::mutex> g(h->mu);
      sg::Config cfg = sg::index_config(h);
      cfg.timing = true;
      int rc2 = search_impl(h, cfg, h->def, nq, d_q768, d_q256, *params, nullptr, 0, osc, oid, on, nullptr,
                            true);
      if (rc2) return rc2;
      if (r > 0) best = std::min(best, h->def.ws.last.ms_total);
    }
    *ms = best;
    return SG_OK;
  };
  sg_tuning t;
  sg_get_tuning(h, &t);
  float base_ms = 0.0f, cur = 0.0f;
  if ((rc = time_batch(&base_ms))) goto done;
  cur = base_ms;
  {
    const uint32_t tmins[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 0xFFFFFFFFu};
    const uint32_t chunks[] = {64, 128, 256, 512};
    const uint32_t seeds[] = {128, 256, 512};
    const uint32_t ctas[] = {1, 2};
    const uint32_t splits[] = {0, 2, 3, 6};
    auto sweep = [&](uint32_t* field, const uint32_t* vals, size_t nv) -> int {
      const uint32_t keep = *field;
      uint32_t best_v = keep;
      for (size_t i = 0; i < nv; i++) {
        if (vals[i] == keep) continue;
        if (field == &t.chunk_blocks && vals[i] < sg::index_config(h).small_chunk_blocks) continue;
        *field = vals[i];
        int rc2 = sg_set_tuning(h, &t);
        if (rc2) return rc2;
        float ms;
        if ((rc2 = time_batch(&ms))) return rc2;
        if (ms < cur * 0.995f) {
          cur = ms;
          best_v = vals[i];
        }
      }
      *field = best_v;
      return sg_set_tuning(h, &t);
    };
    if ((rc = sweep(&t.tc_min_queries, tmins, sizeof tmins / 4)) ||
        (rc = sweep(&t.chunk_blocks, chunks, sizeof chunks / 4)) ||
        (rc = sweep(&t.seed_blocks, seeds, sizeof seeds / 4)) ||
        (rc = sweep(&t.scan_ctas_per_sm, ctas, sizeof ctas / 4)) ||
        (rc = sweep(&t.tc_split, splits, sizeof splits / 4)))
      goto done;
  }
  if (out) *out = t;
  if (out_ms) {
    out_ms[0] = base_ms;
    out_ms[1] = cur;
  }
done:
  cudaDeviceSynchronize();
  dfree(osc); dfree(oid); dfree(on);
  return rc;
}

int sg_lut_scan_batch(uint32_t nq, const uint8_t* tables, const uint8_t* blocks, uint64_t nblocks,
                      uint16_t* out_scores) {
  if ((nq && !tables) || (nblocks && !blocks) || (nq && nblocks && !out_scores))
    return fail(SG_ERR_INVALID, "null argument");
  if (nq == 0 || nblocks == 0) return SG_OK;
  if ((uint64_t)nq * nblocks * SG_BLOCK > (1ull << 34)) return fail(SG_ERR_INVALID, "output above 2^34 scores");
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  uint8_t *dt = nullptr, *db = nullptr;
  uint32_t *dc = nullptr, *dcnt = nullptr;
  uint16_t* dout = nullptr;
  const uint64_t nslots = nblocks * SG_BLOCK;
  int rc;
  if ((rc = dalloc(&dt, (size_t)nq * SG_GROUPS * 16)) || (rc = dalloc(&db, nblocks * SG_BLOCK_BYTES)) ||
      (rc = dalloc(&dc, nblocks * 256)) || (rc = dalloc(&dcnt, 2)) || (rc = dalloc(&dout, nq * nslots))) {
    dfree(dt); dfree(db); dfree(dc); dfree(dcnt); dfree(dout);
    return rc;
  }
  cudaError_t e = cudaMemcpy(dt, tables, (size_t)nq * SG_GROUPS * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, blocks, nblocks * SG_BLOCK_BYTES, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dcnt, 0, 8);
  if (e == cudaSuccess) {
    sg::transcode_tc(db, nblocks, dc, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    sg::launch_lut_scan_tc(nq, dt, dc, nblocks, dout, dcnt, sms, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  uint32_t status = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&status, dcnt, 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(out_scores, dout, nq * nslots * 2, cudaMemcpyDeviceToHost);
  dfree(dt); dfree(db); dfree(dc); dfree(dcnt); dfree(dout);
  if (e != cudaSuccess) return fail(SG_ERR_DEVICE, std::string("sg_lut_scan_batch: ") + cudaGetErrorString(e));
  if (status & sg::kStatusTimeout) return fail(SG_ERR_DEVICE, "sg_lut_scan_batch: a pipeline wait ran out");
  return SG_OK;
}

int sg_dot_i8i8(const int8_t* query, const int8_t* rows, uint64_t nrows, uint32_t dim,
                int32_t* out_dots) {
  if (dim == 0 || dim % 4) return fail(SG_ERR_INVALID, "dim must be a positive multiple of 4");
  if (!query || (!rows && nrows) || (!out_dots && nrows)) return fail(SG_ERR_INVALID, "null argument");
  if (nrows == 0) return SG_OK;
  int8_t *dq = nullptr, *dr = nullptr;
  int32_t* dout = nullptr;
  int rc;
  if ((rc = dalloc(&dq, dim)) || (rc = dalloc(&dr, nrows * dim)) || (rc = dalloc(&dout, nrows))) {
    dfree(dq); dfree(dr); dfree(dout);
    return rc;
  }
  cudaError_t e = cudaMemcpy(dq, query, dim, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dr, rows, nrows * dim, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sg::launch_dot_i8i8(dq, dr, nrows, dim, dout, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out_dots, dout, nrows * 4, cudaMemcpyDeviceToHost);
  dfree(dq); dfree(dr); dfree(dout);
  if (e != cudaSuccess) return fail(SG_ERR_DEVICE, std::string("sg_dot_i8i8: ") + cudaGetErrorString(e));
  return SG_OK;
}

}  // extern "C"
