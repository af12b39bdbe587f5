// internal.hpp — device-resident index, per-call workspace and kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sieve_gpu.h"

namespace sg {

// Runs a kernel-attribute setter (such as raising the dynamic shared-memory limit) once per
// device: an attribute set on one device does not carry over to a kernel launched on another.
// Racing first calls may both run the setter, which is idempotent. A device index past 63 runs
// it every time.
struct PerDeviceOnce {
  std::atomic<uint64_t> done{0};
  template <typename F>
  cudaError_t operator()(F&& set) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev >= 0 && dev < 64 ? 1ull << dev : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = set();
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
  }
};

// Blocks (32 slots) a scan work item covers at most; the scan CTA holds one chunk's estimates
// in shared memory (4 B per slot plus one padding word per block), so kMaxChunkBlocks = 512
// is 66 KB.
constexpr uint32_t kMaxChunkBlocks = 512;
constexpr uint32_t kChunkBlocks = 256;   // default chunk of the batched scan
constexpr uint32_t kSeedBlocks = 512;    // block budget of each query's seed (its first probes)
constexpr uint32_t kMaxSegs = 64;        // probes one seed can cover
// Largest cand / k / r the select kernels sort in shared memory.
constexpr uint32_t kMaxCand = 4096;
// Most clusters the filter plan Expand sorts per query in shared memory (128 KB of keys).
constexpr uint32_t kExpandMaxK = 16384;
// Status bits a kernel raises in Workspace::status.
constexpr uint32_t kStatusOverflow = 1u;   // a candidate buffer filled up (query is retried)
constexpr uint32_t kStatusWindow = 2u;     // a BF16 routing window exceeded its buffer
constexpr uint32_t kStatusTimeout = 4u;    // a tensor-core wait ran out (the CTA stopped)

// HBM layout of one IVF index (all arrays on the index's device).
struct DevIndex {
  int device = 0;
  uint32_t k = 0;   // clusters: the centroids', plus in a live index one delta list per centroid
  uint32_t kc = 0;  // centroids (routing scores these)
  // A live index (sg_live_open): cluster kc + c is cluster c's delta list (rows inserted since the
  // build, src/live.rs:39-66), scanned right after c's base list; routing expands every probe c
  // whose delta list holds slots into (c, kc + c) with the same centroid score.
  bool live = false;
  uint64_t n = 0, nblocks = 0, nslots = 0;
  float* cent = nullptr;             // [k*256] centroids.f32
  float* cent_t = nullptr;           // [256*k] transposed, for the exact routing kernel
  __nv_bfloat16* cent_bf16 = nullptr;  // [k*256] BF16 copy for the tensor-core routing GEMM
  float cent_norm_max = 0.0f;
  uint32_t* block_off = nullptr;     // [k+1] first block of each cluster
  uint32_t* clen = nullptr;          // [k] real (non-PAD) slots of each cluster
  uint8_t* blocks = nullptr;         // [nblocks*1024] nibble-transposed codes (blocks.bin)
  uint32_t* blocks_tc = nullptr;     // [nslots*8] the same codes slot-major (tcgen05 scan)
  float* mul = nullptr;              // [nslots] factors.f32 [.., 0]
  float* err = nullptr;              // [nslots] factors.f32 [.., 1]
  uint32_t* ids = nullptr;           // [nslots] ids.u32
  float* rot = nullptr;              // [768] rotation.f32 (null for global sign codes)
  float rot_norm = 0.0f;             // (256 as f32).powf(-1.5)
  // Global sign codes (an index without rotation.f32 / factors.f32, src/ivf.rs:700-717): slots
  // hold their rows' sign codes, the LUT is built on the unrotated prefix, candidates are ranked
  // by the u16 LUT score with ties by row, and mul = 1, err = +inf fill the factor planes.
  bool global = false;
  bool has_t2 = false;
  float* t2_sigma = nullptr;         // [256]
  uint8_t* t2_codes = nullptr;       // [n*64]
  float* t2_norm = nullptr;          // [n]
  int8_t* rerank = nullptr;          // [n*768]
  float* norm256 = nullptr;          // [n]
  float* qscale = nullptr;           // [768]
  uint8_t* codes = nullptr;          // [n*32] codes.bin, when given (the flat Hamming baseline)
  std::vector<uint64_t> h_block_off;
  std::vector<uint32_t> h_clen;
  std::vector<uint32_t> h_chunks_desc_prefix;  // prefix sums of per-cluster chunk counts, largest first
  std::vector<uint64_t> h_slots_desc_prefix;   // prefix sums of per-cluster slot counts, largest first
};

// Stride of a call's probe arrays: min(nprobe, centroids), doubled in a live index (each probe may
// be followed by its delta list).
inline uint32_t probe_stride(const DevIndex& x, uint32_t nprobe) {
  const uint32_t p = nprobe < x.kc ? nprobe : x.kc;
  return x.live ? 2 * p : p;
}

// Device buffers of one batched call, grown on demand and reused.
struct Workspace {
  uint32_t nq_cap = 0, P_cap = 0, cand_cap = 0, k_cap = 0, r_cap = 0;
  uint64_t item_cap = 0, cbuf_cap = 0;
  float* q768 = nullptr;       // [nq*768]
  float* q256 = nullptr;       // [nq*256]
  uint8_t* tables = nullptr;   // [nq*1024]
  float4* qp = nullptr;        // [nq] (scale, bias, a, b)
  float* qnorm = nullptr;      // [nq]
  int8_t* wq = nullptr;        // [nq*768]
  float* winv = nullptr;       // [nq]
  int8_t* wq256 = nullptr;     // [nq*256]
  float* winv256 = nullptr;    // [nq]
  __nv_bfloat16* q16 = nullptr;  // [nq*256] q256 rounded to bf16: the routing GEMM's B operand
  uint32_t* w8 = nullptr;      // [nq*64] s8 weights of the tensor-core bound, 4 per word
  float4* fq = nullptr;        // [nq] (gamma, R_hi, R_lo, -) of the bound
  uint32_t* tc_start = nullptr;  // [nq] candidate-buffer entries before the bound pass
  float* scores = nullptr;     // [nq*k] routing scores
  uint64_t scores_cap = 0;
  float* probe_sc = nullptr;   // [nq*P]
  uint32_t* probe_cl = nullptr;  // [nq*P]
  uint32_t* probe_off = nullptr;  // [nq*P] admission offset of each probe's first slot
  uint32_t* probe_n = nullptr;   // [nq]
  uint64_t* scanned = nullptr;   // [nq]
  uint4* items = nullptr;        // [item_cap] (query, probe rank, first block, end block)
  uint4* seed_items = nullptr;   // [nq] each query's first rank-0 chunk (the seed)
  uint32_t* counters = nullptr;  // [8]: nitems, next item, status, -, mma groups, next group
  uint32_t inv_k = 0;            // clusters the per-cluster arrays below are sized for
  uint32_t* inv_cnt = nullptr;   // [k] (query, probe >= 1) pairs per cluster
  uint32_t* inv_fill = nullptr;  // [k]
  uint32_t* inv_off = nullptr;   // [k+1]
  uint32_t* inv_list = nullptr;  // [nq*P] (query << 12 | probe rank), grouped by cluster
  uint2* gitems = nullptr;       // [gitems_cap] (cluster, group of 64 queries)
  uint64_t gitems_cap = 0, inv_cap = 0;
  uint32_t* thr = nullptr;       // [nq] running lower bound of the cand-th estimate (ordered)
  uint32_t* ccount = nullptr;    // [nq] entries appended to a query's candidate buffer
  uint32_t* cbuf_est = nullptr;  // [nq*cbuf_per_q] candidate buffer: estimate (f32 bits)
  uint2* cbuf_info = nullptr;    // [nq*cbuf_per_q] (admission key, slot) of the same entry
  uint32_t cbuf_per_q = 0;       // a multiple of 4 (the cut reads estimates four at a time)
  uint8_t* overflow = nullptr;   // [nq]
  float* cest = nullptr;         // [nq*cand] candidates after cut + dedup, in row order
  uint32_t* cid = nullptr;
  float* cerr = nullptr;
  uint32_t* cn = nullptr;        // [nq]
  uint32_t* lid = nullptr;       // [nq*cand] rerank list (after pruning / tier-2)
  float* lsc = nullptr;          // [nq*cand] scores of the rerank list
  uint32_t* ln = nullptr;        // [nq]
  float* out_sc = nullptr;       // [nq*k]
  uint32_t* out_id = nullptr;
  uint32_t* out_n = nullptr;
  uint64_t* allow = nullptr;     // [allow_words]
  uint64_t allow_cap = 0;
  // Per-query allow bitsets (the serving loop batches queries with different filters): when
  // per_query_allow is set the scans read allow_q[q] / allow_wq[q] instead of the call's bitset.
  const uint64_t** allow_q = nullptr;  // [allow_q_cap] device pointers
  uint64_t* allow_wq = nullptr;        // [allow_q_cap] words of each
  uint64_t allow_q_cap = 0;
  bool per_query_allow = false;
  float* brute = nullptr;        // [brute_cap] exact scores of the filter plan Brute
  uint64_t brute_cap = 0;
  void* host_pinned = nullptr;   // pinned staging for host<->device copies
  size_t host_pinned_cap = 0;
  cudaEvent_t ev[12] = {};
  bool events = false;
  sg_stats last = {};
};

// One execution context of an index: a workspace, the stream its work runs on, and the CUDA
// graphs captured for the call shapes it has seen. sg_search uses the index's default context;
// the serving loop runs several so that batches overlap on the device.
struct GraphKey {
  uint32_t nq;
  sg_params p;
  bool have_q256;
  const uint64_t* allow;
  uint64_t allow_words;
  uint64_t gen;
  uint64_t cfg_gen;  // the index's Config generation the graph was captured under
  bool same(const GraphKey& o) const {
    return nq == o.nq && have_q256 == o.have_q256 && allow == o.allow &&
           allow_words == o.allow_words && gen == o.gen && cfg_gen == o.cfg_gen &&
           memcmp(&p, &o.p, sizeof(sg_params)) == 0;
  }
};

// A pipeline captured as a CUDA graph for one call shape (exec is null until the shape has been
// seen twice) and the launches it replays.
struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec;
  uint32_t launches;
};

struct Ctx {
  Workspace ws;
  cudaStream_t stream = nullptr;
  cudaEvent_t order_ev = nullptr;  // orders this stream after a caller's stream (created on first use)
  uint64_t gen = 1;  // bumped whenever a workspace buffer moves (captured graphs go stale)
  std::vector<GraphEntry> graphs;
};

struct Config {
  uint32_t chunk_blocks = kChunkBlocks;  // batched scan chunk (autotuned)
  uint32_t small_chunk_blocks = 64;      // chunk when few queries share the GPU
  uint32_t small_batch = 64;             // below this many queries use the small chunk
  uint32_t seed_blocks = kSeedBlocks;
  uint32_t small_seed_blocks = 256;      // seed budget below small_batch queries
  uint32_t scan_ctas_per_sm = 2;
  uint32_t soft_cap = 0;  // per-query buffer override (0: automatic); SIEVE_GPU_SOFT_CAP
  int graphs = 1;         // capture and replay CUDA graphs per call shape (SIEVE_GPU_GRAPHS)
  int mma = 1;            // SIEVE_GPU_MMA: 0 ALU scan only, 1 automatic, 2 tensor cores whenever nprobe > 1
  int tc = 1;             // SIEVE_GPU_TC: 1 the tcgen05 bound scan, 2 the tcgen05 one-hot scan (kept
                          // for comparison)
  uint32_t tc_split = 0;  // SIEVE_GPU_TC_SPLIT (> 1): a first tcgen05 round over the ranks below it
  // Clusters probed by fewer queries than this in a batch are scanned by the ALU kernel: a
  // tcgen05 tile costs the same ~32 x 101 cycles per 128 slots for any query count up to 128,
  // an ALU (slot, query) pair ~6 (SIEVE_GPU_TC_MIN overrides; the autotuner measures it)
  uint32_t tc_min_queries = 6;
  int route_precision = SG_ROUTE_BF16;  // sg_set_route_precision
  bool timing = false;                  // per-stage device timing (sg_set_timing) of this call
  uint64_t gen = 1;  // bumped whenever a field changes (captured graphs of an older one are stale)
  // device memory a batch's candidate buffers may take (a quarter of what the index leaves
  // free at open, between 8 and 32 GiB); a query that fills its share is re-run alone
  uint64_t cbuf_budget = 8ull << 30;
};

std::string& last_error();
void set_cluster_bounds(DevIndex& x, uint32_t chunk);
int fail(int code, const std::string& msg);

// Views of an open index for entry points in other translation units (sieve_gpu.cu defines them).
const DevIndex* index_arrays(const sg_index* h);
// A copy of the index's tuning and routing precision, taken under the index's config lock: a call
// works from one snapshot, so a concurrent sg_set_tuning / sg_autotune cannot change it midway.
Config index_config(const sg_index* h);
int index_sms(const sg_index* h);
int index_check_params(const sg_index* h, const sg_params* p);

// kernel launchers (one per .cu file section)
void launch_prefix(Workspace& w, uint32_t nq, cudaStream_t st);
void launch_prep(const DevIndex& ix, Workspace& w, uint32_t nq, cudaStream_t st);
// Looks up the driver's tensor-map encoder the BF16 routing GEMM needs (once per process);
// false if the driver does not provide it.
bool route_gemm_ready();
// A 2-D TMA map over a bf16 matrix of `rows` rows of `cols` elements, `row_bytes` apart (a multiple
// of 16), whose box is one k-chunk of box_rows rows: 16 bytes (8 elements) without swizzle, or
// 128 bytes (64 elements) in the 128-byte swizzle (sw128); rows and columns past the matrix read
// as zeros. False if the encoder is missing or rejects the shape.
bool encode_bf16_rows(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint64_t row_bytes,
                      uint32_t box_rows, bool sw128);

// ---- bigann routing on the tcgen05 tensor cores (bg_route.cu) --------------------------------
constexpr uint32_t kBgSubStep = 16;  // the threshold subset: every 16th leaf
struct BgRoutePlan {
  uint32_t ksub;  // leaves in the subset
  uint32_t cap;   // emitted entries one query's list holds
  bool subset;    // false: every leaf is emitted (cap = K)
};
BgRoutePlan bg_route_plan(uint32_t K, uint32_t P);
// Elements of the [rows x 208] bf16 hi/lo matrix, and its fill from the f32 leaves [K x 100].
size_t bg_route_tc_hl_elems(uint32_t rows);
int bg_route_tc_prepare(const float* d_leaves, uint32_t K, __nv_bfloat16* d_hl, cudaStream_t st);
struct BgRouteTc {
  uint32_t K, P, nq;
  int sms;
  float margin, cmax, cmax2;  // cmax: the largest leaf norm, cmax2 its square (rounded up)
  const int8_t* q;
  __nv_bfloat16* qhl;  // [nq x 208] scratch
  const __nv_bfloat16* hl;
  const float* leaves;
  const float* ln;
  const float* qq;     // |q|^2 per query
  float* sub_scores;   // [nq x ksub]
  float* lim;          // [nq]
  uint2* ent;          // [nq x cap]
  uint32_t* cnt;       // [nq]
  uint32_t* probe;     // [nq x P]
  float* probe_cent;   // [nq x P]
  uint32_t* probe_n;   // [nq]
  uint32_t* status;    // kStatus* bits
};
// Five launches: queries to bf16, the subset GEMM (when the plan has a subset), the thresholds,
// the filtered GEMM, the per-query select.
cudaError_t launch_bg_route_tc(const BgRouteTc& r, cudaStream_t st);
// BF16: two launches (the queries to bf16, then the tcgen05 GEMM); FP32: one. Returns the
// launch error, or cudaErrorInvalidValue if the GEMM's TMA tensor maps cannot be encoded.
cudaError_t launch_route_scores(const DevIndex& ix, Workspace& w, uint32_t nq, int precision,
                                cudaStream_t st);
// alu_ranks = false leaves probe ranks >= 1 to the MMA scan (only rank-0 chunks past the seed
// become ALU work items).
inline uint32_t next_pow2_host(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}
// filter::search Plan::Expand routing: needs exact f32 scores (launch_route_scores FP32) and a
// probe-array stride of k.
void launch_route_expand(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                         uint32_t chunk_blocks, uint32_t seed_blocks,
                         const uint32_t* per_cluster, uint64_t target, cudaStream_t st);
void launch_route_select(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                         int precision, uint32_t chunk_blocks, uint32_t seed_blocks,
                         bool alu_ranks, cudaStream_t st);
// The caller's probe lists (device arrays [nq * P], counts [nq], P = min(nprobe, k)) in place of
// routing: Index::candidates over given probes. Cluster numbers must be < k.
// The lists may be w.probe_sc / w.probe_cl / w.probe_n themselves: each CTA reads its query's
// list before it writes the probe list.
void launch_route_given(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p, uint32_t chunk_blocks,
                        uint32_t seed_blocks, bool alu_ranks, const float* given_sc, const uint32_t* given_cl,
                        const uint32_t* given_n, cudaStream_t st);
void launch_invert(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t P, uint32_t qg, uint32_t rlo,
                   uint32_t rhi, cudaStream_t st, uint32_t tmin = 1, uint32_t alu_chunk = 0);
// The batched pass after the seed (scan_tc.cu): the (query, probe) pairs of clusters probed by
// fewer than cfg.tc_min_queries queries go to the ALU chunk scan (with the routing kernel's
// rank-0 chunks), the others to the tcgen05 scan, which has the same admission as
// the ALU scan. With cfg.tc_split > 1 it scans probe ranks [1, split) first, raises every
// query's threshold to the cand-th best estimate its buffer then holds, and scans the rest.
struct Config;
int launch_scan_tc(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                   const uint64_t* allow, uint64_t allow_words, int sms, const Config& cfg,
                   uint32_t chunk_blocks, cudaStream_t st);
// scan_tcf.cu: per-query weights and residual bounds of the tensor-core bound (after
// launch_prep), and one bound pass over launch_invert's items with the exact recheck of what it
// admitted (returns the kernels launched).
void launch_filter_prep(Workspace& w, uint32_t nq, cudaStream_t st);
int launch_scan_tcf(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t P, const uint64_t* allow,
                    uint64_t allow_words, int sms, cudaStream_t st);
// Launch errors of these two are left for the caller's cudaGetLastError.
void transcode_tc(const uint8_t* blocks, uint64_t nblocks, uint32_t* out, cudaStream_t st);
void launch_lut_scan_tc(uint32_t nq, const uint8_t* tables, const uint32_t* codes, uint64_t nblocks,
                        uint16_t* out, uint32_t* counters, int sms, cudaStream_t st);
// The seed pass (one CTA per query, rank-0 seed item; skipped when seed_blocks is 0) then the
// persistent pass over the queue (skipped when chunk_blocks is 0).
void launch_scan(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                 const uint64_t* allow, uint64_t allow_words, int sms, uint32_t chunk_blocks,
                 uint32_t seed_blocks, int ctas_per_sm, cudaStream_t st);
void launch_cut(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                cudaStream_t st);
int launch_rerank(const DevIndex& ix, Workspace& w, uint32_t nq, const sg_params& p,
                  cudaStream_t st, cudaEvent_t ev_t2_begin, cudaEvent_t ev_t2_end);
void launch_lut_scan(uint32_t groups, const uint8_t* tables, const uint8_t* blocks,
                     uint64_t nblocks, uint16_t* out, cudaStream_t st);
// Filter::new on the device: allowed rows ascending (nrows of them) and allowed slots per cluster.
int filter_build(const DevIndex& ix, const uint64_t* allow, uint64_t words, uint32_t** rows,
                 uint64_t* nrows, uint32_t* per_cluster, cudaStream_t st);
// filter::search Plan::Brute for queries [q0, q0+nq) prepared in w: exact int8 scores of the
// `nrows` allowed rows, then the top k by (score desc, row asc) into w.out_*. `scores` holds
// nq x nrows floats.
int launch_brute(const DevIndex& ix, Workspace& w, uint32_t nq, const uint32_t* rows,
                 uint32_t nrows, uint32_t k, float* scores, cudaStream_t st);
// Top n of per-query scored lists by (score desc, id asc), sorted.
void launch_top_list(const float* sc, const uint32_t* id, const uint32_t* n_in, uint64_t sc_stride,
                     uint64_t id_stride, uint32_t nsel, float* out_sc, uint32_t* out_id,
                     uint32_t* n_out, uint32_t stride_out, uint32_t nq, cudaStream_t st);
void launch_dot_i8i8(const int8_t* q, const int8_t* rows, uint64_t nrows, uint32_t dim,
                     int32_t* out, cudaStream_t st);
// hamming.cu: the flat Hamming baseline for the queries staged in w (q768 and q256): rows in
// w.lid / w.ln (stride cand), scores in w.lsc, the top k in w.out_* (stride k).
int launch_flat_hamming(const DevIndex& ix, Workspace& w, uint32_t nq, uint32_t cand, uint32_t k,
                        cudaStream_t st);

}  // namespace sg

// An open IVF index: its arrays in HBM, the default execution context of sg_search, and the
// tuning of its kernels. The arrays are read-only after open, so any number of contexts search
// them at once; `mu` serialises only the users of the default context.
struct sg_index {
  sg::DevIndex ix;
  sg::Ctx def;  // the context of sg_search / sg_search_device
  std::mutex mu;
  sg::Config cfg;  // guarded by cfg_mu; calls read it through sg::index_config
  mutable std::mutex cfg_mu;
  int sms = 148;
  std::atomic<bool> timing_on{false};
};

// A search context (ivf::Scratch, src/ivf.rs:497-513): one thread's scratch, stream and captured
// graphs over a shared index, so that threads searching one index overlap on the GPU.
struct sg_context {
  sg_index* h = nullptr;
  sg::Ctx ctx;
  std::mutex mu;  // a context serves one call at a time
};

// filter::Filter (src/filter.rs:18-25) resident on its index's device.
struct sg_filter {
  sg_index* h = nullptr;
  uint64_t words = 0;
  uint64_t* allow = nullptr;        // [words] the allow bitset
  uint32_t* rows = nullptr;         // [nrows] allowed rows, ascending
  uint64_t nrows = 0;
  uint32_t* per_cluster = nullptr;  // [k] allowed slots per cluster
};

namespace sg {
// Execution-context entry points (sieve_gpu.cu) for the serving loop: grow c's scratch for a
// batch, launch the whole pipeline on the queries already staged in c.ws (no host sync), run one
// query synchronously (host queries, device allow bitset), and the scratch bytes of a batch. A
// batch passes the same config snapshot to each.
int ctx_prepare(sg_index* h, const Config& cfg, Ctx& c, uint32_t nq, const sg_params& p);
int ctx_launch(sg_index* h, const Config& cfg, Ctx& c, uint32_t nq, const sg_params& p, bool have_q256);
int ctx_search_one(sg_index* h, const Config& cfg, Ctx& c, const float* q768, const float* q256,
                   const sg_params& p, const uint64_t* d_allow, uint64_t allow_words, float* out_sc,
                   uint32_t* out_id, uint32_t* out_n);
uint64_t ctx_bytes(const sg_index* h, const Config& cfg, const sg_params& p, uint32_t nq);
void free_ctx(Ctx& c);
// Live indexes (live.cu): make `h` live with room for max_rows inserted rows and block_cap delta
// blocks (its slot and row arrays are reallocated; the caller holds no other call on h); replace
// the delta lists (nb_of / clen_of [kc] per cluster, then nblocks blocks of codes, factors and ids
// in cluster order); search with a device allow bitset.
int index_make_live(sg_index* h, uint64_t max_rows, uint64_t block_cap);
int index_set_delta(sg_index* h, const uint32_t* nb_of, const uint32_t* clen_of, const uint8_t* blocks,
                    const float* mul, const float* err, const uint32_t* ids, uint64_t nblocks);
int index_search_allow(sg_index* h, uint32_t nq, const float* q768, const float* q256, const sg_params& p,
                       const uint64_t* d_allow, uint64_t allow_words, float* out_sc, uint32_t* out_id,
                       uint32_t* out_n);
}  // namespace sg
