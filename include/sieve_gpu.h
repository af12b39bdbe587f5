/*
 * sieve_gpu.h — C ABI of the B200 (sm_100a) query path of the sieve IVF engine.
 *
 * The reference (a Rust crate) has no FFI; its query API is the in-process Rust API of
 * `ivf::Index` / `ivf::Corpus` / `ivf::Params` / `filter::search` / `bigann::Index`. Each entry
 * point below replaces one of those calls and names the reference item it stands for.
 *
 * Conventions
 *   - Every function returns an int status: SG_OK (0) or a negative SG_ERR_* code. Nothing
 *     aborts across the boundary; sg_last_error() gives a message for the calling thread.
 *   - The library owns all device memory it allocates; callers own their host buffers.
 *   - Functions named *_device take device pointers (inputs already resident in HBM) and a
 *     cudaStream_t passed as void*; everything else takes host pointers and copies.
 *   - Vectors are row-major float32 (queries) or int8 (rerank rows); ids are uint32 corpus rows.
 *   - Results are (score, id) best first, ties broken by ascending id, exactly as the
 *     reference's TopK::into_sorted orders them (src/topk.rs:57-61).
 */
#ifndef SIEVE_GPU_H
#define SIEVE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define SG_OK 0
#define SG_ERR_INVALID -1    /* bad argument or inconsistent index files                     */
#define SG_ERR_IO -2         /* a file could not be read                                       */
#define SG_ERR_OOM -3        /* device or host allocation failed                               */
#define SG_ERR_DEVICE -4     /* a CUDA call failed                                             */
#define SG_ERR_TIMEOUT -5    /* a bounded device-side wait gave up                             */
#define SG_ERR_ADMISSION -6  /* serving: no scratch free for this request right now            */
#define SG_ERR_UNSUPPORTED -7 /* the index lacks the files this request needs                  */

/* ---- constants of the reference (src/lib.rs:21-26, src/lut.rs:42-44, src/ivf.rs:18) -------- */
#define SG_DIM 768          /* full embedding width                                           */
#define SG_PDIM 256         /* Matryoshka prefix the codes are built from                     */
#define SG_CODE_BYTES 32    /* 1-bit code of the prefix                                       */
#define SG_GROUPS 64        /* 4-dim LUT groups of the prefix                                 */
#define SG_BLOCK 32         /* slots per nibble-transposed block                              */
#define SG_BLOCK_BYTES 1024 /* GROUPS * 16                                                    */
#define SG_TIER2_BYTES 64   /* 2-bit middle tier code (src/tier2.rs:7)                        */
#define SG_PAD 0xFFFFFFFFu  /* id of a padding slot                                           */
#define SG_COUNT_FAILED 0xFFFFFFFFu /* a device-written result count: the call failed on the GPU
                                       (see sg_search_noalloc)                                  */

/* ---- ivf::Rerank (src/ivf.rs:425-439) --------------------------------------------------- */
typedef enum {
  SG_RERANK_NONE = 0,   /* Rerank::None: order by the code estimate                           */
  SG_RERANK_PREFIX = 1, /* Rerank::Prefix: int8 256-d prefix cosine                           */
  SG_RERANK_FULL = 2,   /* Rerank::Full: int8 768-d dot of every candidate                     */
  SG_RERANK_TIERED = 3, /* Rerank::Tiered(r): 2-bit tier (or prefix) to r, then full           */
  SG_RERANK_SSD = 4     /* Rerank::Ssd(r): best r by estimate, then full (rows are in HBM)     */
} sg_rerank_kind;

/* ---- ivf::Params (src/ivf.rs:441-460) --------------------------------------------------- */
typedef struct {
  uint32_t nprobe;      /* clusters probed (cap)                                                */
  uint32_t cand;        /* candidates kept by the code scan                                     */
  uint32_t rerank_kind; /* sg_rerank_kind                                                       */
  uint32_t rerank_r;    /* r of Tiered(r) / Ssd(r)                                              */
  uint32_t k;           /* results returned                                                     */
  uint32_t has_prune;   /* prune: Some((prune_m, prune_w))                                      */
  uint32_t prune_m;
  float prune_w;
  uint32_t has_margin;  /* margin: Some(margin)                                                 */
  float margin;
  uint32_t has_budget;  /* budget: Some(budget) in stored slots                                 */
  uint32_t reserved;
  uint64_t budget;
} sg_params;

/* ---- ivf::Timing (src/ivf.rs:521-538): device times of one call, in nanoseconds ----------- */
typedef struct {
  uint64_t route;    /* routing GEMM + probe selection                                         */
  uint64_t scan;     /* query prep + LUT scan + candidate cut + dedup                          */
  uint64_t rerank;   /* pruning + tier-2 + int8 rerank                                         */
  uint64_t tier2;    /* part of rerank spent in the 2-bit tier                                 */
  uint64_t scanned;  /* slots scanned (padding included), summed over queries                  */
  uint64_t reranked; /* candidates reaching the rerank stage after dedup and pruning           */
  uint64_t probed;   /* clusters scanned                                                       */
  uint64_t fetch;    /* always 0: no SSD tier                                                  */
  uint64_t wait;     /* always 0: no shard fan-out                                             */
} sg_timing;

/* Routing precision. FP32 scores every centroid with the reference's sequential f32 dot
 * (src/blas.rs:43-54). BF16 runs the tensor-core GEMM, then rescores in FP32 every centroid
 * whose BF16 score lies inside the rigorous error window of the nprobe-th best, so the probe
 * set and the centroid scores equal the FP32 path's exactly. */
typedef enum { SG_ROUTE_FP32 = 0, SG_ROUTE_BF16 = 1 } sg_route_precision;

/* Device-side stage times (ms) and work counters of the last search call, recorded when timing is
 * on (sg_set_timing). No counterpart in the reference beyond ivf::Timing; used for rooflines. */
typedef struct {
  float ms_prep;          /* prefix + rotation + LUT + int8 query weights                       */
  float ms_route_gemm;    /* routing scores (BF16 tensor-core GEMM or exact FP32)               */
  float ms_route_select;  /* probe selection, FP32 rescoring window, work items                 */
  float ms_scan;          /* LUT scan + estimate + admission (the persistent scan kernel)        */
  float ms_cut;           /* candidate cut + SOAR dedup                                           */
  float ms_rerank;        /* prune + tier-2 + int8 rerank + top-k                                 */
  float ms_tier2;         /* part of ms_rerank in the 2-bit tier                                  */
  float ms_total;
  uint32_t launches;      /* kernels of this library launched by the call                          */
  uint32_t reserved;
  uint64_t scanned;       /* slots scanned, padding included, summed over queries                 */
  uint64_t probed;        /* clusters probed, summed over queries                                 */
  uint64_t reranked;      /* candidates reaching the rerank stage, summed over queries            */
  uint64_t buffered;      /* scan entries appended to the candidate buffers, summed over queries  */
  float ms_seed;          /* part of ms_scan in the seed pass (each query's best cluster)         */
  uint32_t retried;       /* queries re-run with their exact buffer bound after a batch's buffer
                             filled up                                                      */
} sg_stats;

typedef struct sg_index sg_index;

/* Host arrays of an IVF index plus its corpus, laid out exactly as the reference's files
 * (src/ivf.rs:75-90 Corpus::open, src/ivf.rs:553-578 Index::open). Optional members may be
 * NULL: tier2_* (no 2-bit tier), rotation/factors (both NULL: a global sign-code index, whose
 * slots hold their rows' sign codes, ranked by the u16 LUT score of the unrotated prefix with
 * ties by row and no error bound, src/ivf.rs:700-717), norm256 (no prefix rerank), codes (no
 * flat Hamming baseline). */
typedef struct {
  uint64_t n;                 /* corpus rows                                                   */
  uint32_t k;                 /* clusters                                                      */
  const float* centroids;     /* centroids.f32   [k * 256]                                     */
  const uint64_t* block_off;  /* block_off.u64   [k + 1]                                       */
  const uint32_t* ids;        /* ids.u32         [nblocks * 32]                                */
  const uint8_t* blocks;      /* blocks.bin      [nblocks * 1024]                              */
  const float* factors;       /* factors.f32     [nblocks * 32 * 2] = [mul, err] per slot      */
  const float* rotation;      /* rotation.f32    [3 * 256] signs                               */
  const float* tier2_sigma;   /* tier2.sigma     [256]                                         */
  const uint8_t* tier2_codes; /* tier2.bin       [n * 64]                                      */
  const float* tier2_norm;    /* tier2.norm      [n]                                           */
  const int8_t* rerank;       /* rerank.i8       [n * 768]                                     */
  const float* norm256;       /* norm256.f32     [n]                                           */
  const float* quant_scale;   /* quant.f32       [768]                                         */
  const uint8_t* codes;       /* codes.bin       [n * 32] global sign codes of the rows
                                 (nullable: only sg_flat_hamming reads them)                 */
} sg_ivf_arrays;

/* ---- bigann: L2 search over int8 rows (src/bigann.rs) ---------------------------------- */
#define SG_BG_DIM 100          /* bigann::D: SPACEV row width                                   */
#define SG_BG_PDIM 128         /* bigann::PD: padded width of the rotation and the codes        */
#define SG_BG_GROUPS 32        /* LUT groups of a 128-bit code                                  */
#define SG_BG_CODE 16          /* bigann::CODE: bytes of a 1-bit code                           */
#define SG_BG_BLOCK_BYTES 512  /* bigann::BLOCK_BYTES                                           */
#define SG_BG_MAX_BITS 3       /* bigann::MAX_BITS                                              */

/* bigann::Params (src/bigann.rs:610-623). */
typedef struct {
  uint32_t nprobe;  /* leaves probed (cap)                                                      */
  uint32_t cand;    /* candidates reranked exactly from the base rows                           */
  uint32_t k;       /* results returned                                                         */
  uint32_t refine;  /* multi-bit index: 1-bit shortlist re-estimated from all planes; 0 = off   */
  float margin;     /* keep leaves with |q-c|^2 <= (1 + margin) |q-c1|^2; 0 = off               */
  uint32_t route_fp32; /* 0: route on the tensor cores (bf16 hi/lo GEMM, exact FP32 rescoring of a
                          window: the same probe lists); 1: the exact FP32 dot of every leaf     */
} sg_bigann_params;

/* bigann::Timing (src/bigann.rs:624-632): device times in nanoseconds. */
typedef struct {
  uint64_t route;
  uint64_t scan;
  uint64_t io_wait;  /* always 0: every record is resident in HBM                               */
  uint64_t rerank;
  uint64_t scanned;  /* slots scanned, padding included                                         */
  uint64_t probes;   /* leaves probed                                                           */
} sg_bigann_timing;

/* Host arrays of a bigann index and its base, de-interleaved from the reference's postings.bin
 * records (src/postings.rs:9-14, :31-34; src/bigann.rs:405-432): per slot, a 16-byte 1-bit
 * code in 512-byte nibble-transposed blocks, [mul, |x|^2] factors, the row id and, with
 * bits > 1, (bits - 1) * 16 bytes of refinement planes followed by the f32 scale f. */
typedef struct {
  uint64_t n;                 /* base rows                                                     */
  uint32_t k;                 /* leaves                                                        */
  uint32_t bits;              /* bits.u64: refinement width 1..3                               */
  const float* leaves;        /* centroids.f32   [k * 100]                                     */
  const uint64_t* block_off;  /* block_off.u64   [k + 1]                                       */
  const uint32_t* ids;        /* record ids      [nblocks * 32]                                */
  const uint8_t* blocks;      /* record blocks   [nblocks * 512]                               */
  const float* factors;       /* record factors  [nblocks * 32 * 2] = [mul, |x|^2] per slot    */
  const uint8_t* ext;         /* record extra    [nblocks * 32 * extra], extra = (bits-1)*16+4 */
  const float* rotation;      /* rotation.f32    [3 * 128] signs                               */
  const int8_t* base;         /* base.NN         [n * 100]                                     */
} sg_bigann_arrays;

/* ---- errors ----------------------------------------------------------------------------- */
const char* sg_last_error(void);
/* Library version string and the device it was built for. */
const char* sg_version(void);

/* ---- open / close ----------------------------------------------------------------------- */
/* ivf::Corpus::open(ingest_dir) + ivf::Index::open(index_dir) (src/ivf.rs:75-90, :553-578):
 * reads the reference's files and uploads them to HBM on `device`. */
int sg_open_ivf(const char* ingest_dir, const char* index_dir, int device, sg_index** out);
/* The same from host arrays already in memory (the files' contents). */
int sg_open_ivf_arrays(const sg_ivf_arrays* a, int device, sg_index** out);
int sg_close(sg_index* index);
/* Index facts: clusters, corpus rows, blocks, whether a 2-bit tier is resident. */
int sg_index_info(const sg_index* index, uint32_t* k, uint64_t* n, uint64_t* nblocks,
                  uint32_t* has_tier2);
int sg_set_route_precision(sg_index* index, int precision);
/* Turns per-stage device timing of every search on (1) or off (0). */
int sg_set_timing(sg_index* index, int on);
/* Stage times and counters of the last sg_search / sg_search_device on this index. */
int sg_last_stats(const sg_index* index, sg_stats* out);

/* ---- search ----------------------------------------------------------------------------- */
/* ivf::Index::search / search_view (src/ivf.rs:621-633) for nq queries at once.
 * q768 [nq*768] and q256 [nq*256] are unit length (q256 may be NULL: it is then the
 * renormalised prefix of q768, as quant::prefix, src/quant.rs:17-20). params is one sg_params
 * shared by all queries. allow_bits (nullable, allow_words u64 words) is View::allow
 * (src/ivf.rs:465-483): only rows with a set bit are returned. Outputs: out_scores/out_ids
 * [nq * params.k], out_counts [nq] (results per query, <= k). timing is nullable. */
int sg_search(sg_index* index, uint32_t nq, const float* q768, const float* q256,
              const sg_params* params, const uint64_t* allow_bits, uint64_t allow_words,
              float* out_scores, uint32_t* out_ids, uint32_t* out_counts, sg_timing* timing);
/* The same with every pointer on the device and the work issued on `stream` (cudaStream_t). */
int sg_search_device(sg_index* index, uint32_t nq, const float* d_q768, const float* d_q256,
                     const sg_params* params, const uint64_t* d_allow_bits,
                     uint64_t allow_words, float* d_out_scores, uint32_t* d_out_ids,
                     uint32_t* d_out_counts, void* stream);

/* ---- search contexts: ivf::Scratch (src/ivf.rs:497-513) --------------------------------- */
/* The reference shares one Index across rayon workers, each with its own Scratch
 * (src/bin/search.rs:312-323). A context is that per-thread state on the GPU: its own stream,
 * device scratch and captured CUDA graphs over a shared index. sg_search / sg_search_device use
 * the index's default context and serialise their callers; threads that search through contexts
 * of their own run concurrently and overlap on the device. A context serves one call at a time
 * and must be closed before its index. */
typedef struct sg_context sg_context;
int sg_context_open(sg_index* index, sg_context** out);
int sg_context_close(sg_context* ctx);
/* ivf::Index::search(&self, &Corpus, q768, q256, &Params, &mut Scratch, &mut Timing)
 * (src/ivf.rs:621-623) for nq queries on the context's scratch; arguments as sg_search. */
int sg_search_ctx(sg_context* ctx, uint32_t nq, const float* q768, const float* q256,
                  const sg_params* params, const uint64_t* allow_bits, uint64_t allow_words,
                  float* out_scores, uint32_t* out_ids, uint32_t* out_counts, sg_timing* timing);
/* The same with device pointers, ordered after `stream` (cudaStream_t); returns once the results
 * are in the output buffers. */
int sg_search_device_ctx(sg_context* ctx, uint32_t nq, const float* d_q768, const float* d_q256,
                         const sg_params* params, const uint64_t* d_allow_bits, uint64_t allow_words,
                         float* d_out_scores, uint32_t* d_out_ids, uint32_t* d_out_counts,
                         void* stream);
/* Stage times and counters of the context's last search (timing on: sg_set_timing). */
int sg_context_last_stats(sg_context* ctx, sg_stats* out);

/* No counterpart in the reference. One query through the same path as sg_search, for callers
 * that must not allocate device memory while serving: a latency-critical serving thread (cudaFree
 * synchronises the device, cudaMalloc can wait behind running kernels) or a host whose device
 * memory budget is fixed up front. All scratch comes from one fixed 32 MiB device array that
 * every GPU loading the library holds until exit; the call allocates nothing (no cudaMalloc,
 * cudaFree or allocating library routine). Params whose buffers exceed 32 MiB are rejected with
 * SG_ERR_INVALID. Pointers are device pointers (d_q256 nullable); results (k scores, k ids, one
 * count) are written on `stream` asynchronously, as sg_search orders them. A failure on the
 * device (a bounded tensor-core wait that ran out, an overflowed buffer) cannot be returned by
 * the asynchronous call: *d_out_count then reads SG_COUNT_FAILED and the results are void. The
 * first call on a device looks up the array's device address (once per device, that device
 * current), so make it before any stream capture. Calls share the array: calls that overlap on
 * the GPU race. */
int sg_search_noalloc(sg_index* index, const float* d_q768, const float* d_q256,
                      const sg_params* params, const uint64_t* d_allow_bits, uint64_t allow_words,
                      float* d_out_scores, uint32_t* d_out_ids, uint32_t* d_out_count,
                      void* stream);

/* The flat Hamming baseline of the reference's search binary (flat_hamming_rerank,
 * src/bin/search.rs:251-269): no index; each query's sign code (of q256, NULL: derived from q768)
 * against every row's code (codes.bin) by 256 - Hamming distance (lut::hamming,
 * src/lut.rs:156-165), the best `cand` rows by (score desc, row asc), reranked by the float-weight
 * int8 dot quant::dot_i8 (src/quant.rs:72-84) into the top k, best first. Needs the index opened
 * with codes (SG_ERR_UNSUPPORTED otherwise); cand, k <= 4096. out_* [nq * k], out_counts [nq]. */
int sg_flat_hamming(sg_index* index, uint32_t nq, const float* q768, const float* q256, uint32_t cand,
                    uint32_t k, float* out_scores, uint32_t* out_ids, uint32_t* out_counts);

/* ivf::Index::route (src/ivf.rs:589-613): the probe list of each query, best first, as
 * (centroid score, cluster). out_scores/out_clusters [nq * params.nprobe], out_counts [nq]. */
int sg_route(sg_index* index, uint32_t nq, const float* q256, const sg_params* params,
             float* out_scores, uint32_t* out_clusters, uint32_t* out_counts);

/* The centroid scores behind ivf::Index::route (src/ivf.rs:592: blas::gemm_abt of the queries
 * against the centroids, src/blas.rs:46-52) at the index's routing precision: out_scores
 * [nq * k], query-major. FP32 gives the reference's sequential sums bit for bit; BF16 gives the
 * tensor-core GEMM's scores, within 0.0085 |q| max|c| of them (the window that sg_route
 * rescores exactly). */
int sg_route_scores(sg_index* index, uint32_t nq, const float* q256, float* out_scores);

/* ivf::Index::candidates (src/ivf.rs:647-729) over the index's own routing: the best
 * params.cand slots by RaBitQ estimate, deduplicated by row, in row order, as
 * (estimate, row, error half-width). out_* [nq * params.cand], out_counts [nq]. */
int sg_candidates(sg_index* index, uint32_t nq, const float* q256, const sg_params* params,
                  const uint64_t* allow_bits, uint64_t allow_words, float* out_est,
                  uint32_t* out_ids, float* out_err, uint32_t* out_counts);

/* ivf::Index::candidates over the caller's probe lists (src/ivf.rs:647-729), as a shard server
 * runs it on the clusters it owns (src/shard.rs:189-191): query q's probes are probe_scores /
 * probe_clusters [q * P + r], r < probe_counts[q] <= P = min(params.nprobe, k), in scan order
 * (their order is the admission order). Outputs as sg_candidates (row order). */
int sg_candidates_probes(sg_index* index, uint32_t nq, const float* q256, const float* probe_scores,
                         const uint32_t* probe_clusters, const uint32_t* probe_counts, const sg_params* params,
                         const uint64_t* allow_bits, uint64_t allow_words, float* out_est, uint32_t* out_ids,
                         float* out_err, uint32_t* out_counts);

/* ivf::Index::rerank (src/ivf.rs:734-815) of the caller's candidates, as a shard server runs
 * phase 2 of the two-phase merge (src/shard.rs:192-195): query q's (estimate, row, error)
 * triples cand_* [q * cand_stride + i], i < cand_counts[q] (cand_err nullable: widths 0), are
 * pruned (params.has_prune) and reranked by params.rerank_kind into the top params.k; params.cand
 * is ignored (cand_stride <= 4096 takes its place). Outputs as sg_search. */
int sg_rerank(sg_index* index, uint32_t nq, const float* q768, const float* q256, const float* cand_est,
              const uint32_t* cand_ids, const float* cand_err, const uint32_t* cand_counts, uint32_t cand_stride,
              const sg_params* params, float* out_scores, uint32_t* out_ids, uint32_t* out_counts);

/* ---- live updates: ivf live layer (src/live.rs) ------------------------------------------ */
/* Inserts, deletes and upserts over an open index without a rebuild (Live, src/live.rs:1-17):
 * an inserted row is encoded on the device as Live::apply_insert encodes it (src/live.rs:318-350)
 * and its slots join per-centroid delta lists in the base block layout, scanned right after each
 * probed cluster's base list (src/ivf.rs:682-684); a delete tombstones the row (View::hidden,
 * src/ivf.rs:474-483). Results carry external ids: a corpus row's is its row, an inserted row's
 * the id it was inserted under; inserting a live id replaces it. The write-ahead log, its replay
 * and compaction are host file I/O and not part of this path. */
typedef struct sg_live sg_live;
/* Live::open (src/live.rs:167-209) over a RaBitQ index: its row and slot arrays grow on the
 * device to hold max_rows inserted rows (the old arrays are copied, so the device briefly holds
 * both). soar_lambda < 0: inserts take no SOAR secondary (the index was built without SOAR).
 * Search a live index through sg_live_search only; close the live handle before the index. */
int sg_live_open(sg_index* index, uint64_t max_rows, float soar_lambda, sg_live** out);
int sg_live_close(sg_live* live);
/* Live::insert (src/live.rs:274-292): m unit 768-d vectors vecs [m * 768] under ext_ids [m]. */
int sg_live_insert(sg_live* live, uint32_t m, const uint32_t* ext_ids, const float* vecs);
/* Live::delete (src/live.rs:295-305): external ids; unknown ones are ignored. */
int sg_live_delete(sg_live* live, uint32_t m, const uint32_t* ext_ids);
/* Live::search (src/live.rs:381-385) for nq queries; outputs as sg_search, with external ids. */
int sg_live_search(sg_live* live, uint32_t nq, const float* q768, const float* q256, const sg_params* params,
                   float* out_scores, uint32_t* out_ids, uint32_t* out_counts);
/* Rows inserted, slots in delta lists, rows tombstoned (each nullable). */
int sg_live_info(sg_live* live, uint64_t* delta_rows, uint64_t* delta_slots, uint64_t* deleted);

/* ---- filters: filter::Filter / Plan / search (src/filter.rs) ---------------------------- */
/* filter::Plan (src/filter.rs:42-53). */
typedef enum {
  SG_PLAN_POST = 0,   /* the unfiltered probes, disallowed rows skipped at admission            */
  SG_PLAN_EXPAND = 1, /* probe clusters in route order until expand_target allowed slots        */
  SG_PLAN_BRUTE = 2,  /* exact int8 scores of every allowed row; no index                        */
  SG_PLAN_AUTO = 3    /* one of the above from the filter's size (sg_plan_resolve)               */
} sg_plan;
#define SG_BRUTE_MAX 250000u     /* filter::BRUTE_MAX (src/filter.rs:55)                       */
#define SG_POST_MIN 0.3          /* filter::POST_MIN (src/filter.rs:57)                        */
#define SG_EXPAND_TARGET 200000u /* filter::EXPAND_TARGET (src/filter.rs:59)                   */

typedef struct sg_filter sg_filter;
/* filter::Filter::new (src/filter.rs:27-38) on the index's device: keeps the allow bitset, the
 * allowed rows ascending and the allowed slots per cluster in HBM. Bits at rows >= n are
 * ignored. The filter belongs to `index` and must be freed before it. */
int sg_filter_new(sg_index* index, const uint64_t* allow_bits, uint64_t allow_words,
                  sg_filter** out);
/* The filter's allowed-row count, and (each nullable) per_cluster [k] and rows [nrows]. */
int sg_filter_info(const sg_filter* filter, uint64_t* nrows, uint32_t* out_per_cluster,
                   uint32_t* out_rows);
int sg_filter_free(sg_filter* filter);
/* filter::Plan::resolve (src/filter.rs:62-71): the plan Auto stands for, given the allowed rows
 * and the corpus size (SG_PLAN_EXPAND then means Expand(SG_EXPAND_TARGET)); other plans are
 * returned as they are. */
int sg_plan_resolve(int plan, uint64_t allowed_rows, uint64_t n);
/* filter::search (src/filter.rs:74-110) for nq queries: the top params.k allowed rows of each
 * as (score, row), best first. expand_target is Expand's target (ignored by other plans; Auto
 * uses SG_EXPAND_TARGET). Expand needs k <= 16384 clusters. Outputs as sg_search. */
int sg_filter_search(sg_index* index, const sg_filter* filter, int plan, uint64_t expand_target,
                     uint32_t nq, const float* q768, const float* q256, const sg_params* params,
                     float* out_scores, uint32_t* out_ids, uint32_t* out_counts,
                     sg_timing* timing);

/* ---- serving: continuous batching ------------------------------------------------------- */
/* No counterpart in the reference beyond calling ivf::Index::search from many threads
 * (src/bin/search.rs:272-323). A server queues single-query requests and a dispatcher thread
 * batches whatever is pending each time one of `contexts` execution contexts (a stream with its
 * own device scratch) frees up: requests that arrive while others run join the next batch, and
 * batches on different contexts overlap on the GPU. A batch holds requests with the same params;
 * each may carry its own filter (the Post plan). Every result equals the query run alone. */
typedef struct sg_server sg_server;
typedef struct {
  uint32_t max_batch;      /* queries per batch (0: 1024)                                        */
  uint32_t contexts;       /* batches in flight at once (0: 2)                                   */
  uint64_t scratch_bytes;  /* HBM budget for all contexts' scratch (0: 8 GiB); batches are cut to
                              fit a context's share, and a request that cannot fit alone is
                              refused with SG_ERR_ADMISSION                                     */
  uint32_t max_pending;    /* queued requests before submit refuses (0: 2^20)                    */
  uint32_t reserved;
} sg_server_config;
typedef struct {
  float queue_ms;    /* submit to the launch of its batch                                       */
  float service_ms;  /* launch to results on the host                                           */
  uint32_t batch;    /* queries in its batch                                                     */
  uint32_t retried;  /* 1 when its candidate buffer filled up and it ran again alone            */
} sg_request_info;
typedef struct {
  uint64_t submitted, completed, rejected, batches, queries_batched, retried;
  uint32_t pending, in_flight;
} sg_server_stats;
int sg_server_start(sg_index* index, const sg_server_config* config, sg_server** out);
/* Queues one query (q768 [768], q256 [256] nullable); filter (nullable) restricts it to the
 * filter's rows. Returns a ticket for sg_server_poll. */
int sg_server_submit(sg_server* server, const float* q768, const float* q256,
                     const sg_params* params, const sg_filter* filter, uint64_t* ticket);
/* Waits up to wait_ms (< 0: forever; 0: no wait) for the ticket's results: out_scores/out_ids
 * [params.k], out_count. SG_ERR_TIMEOUT while it runs; after SG_OK the ticket is gone. */
int sg_server_poll(sg_server* server, uint64_t ticket, int wait_ms, float* out_scores,
                   uint32_t* out_ids, uint32_t* out_count, sg_request_info* info);
int sg_server_get_stats(sg_server* server, sg_server_stats* out);
/* An open-loop load from a library thread (no counterpart in the reference; its bench replays
 * queries from rayon workers, src/bin/search.rs:742-748): request i is submitted at arrival_ns[i]
 * after the call starts, whatever the state of earlier requests, with the query
 * q768 + which[i] * 768 and the filter filters[filter_of[i]] (none where filter_of is NULL or
 * filter_of[i] < 0); a second thread collects the results in order. out_latency_ms[i] is the
 * request's submit-to-results time on the library's clock (-1 if it failed), out_batch[i]
 * (nullable) the size of its batch, *out_wall_s (nullable) the time from the first arrival to the
 * last result. Returns the first failure of a submit or a poll. */
int sg_server_replay(sg_server* server, uint32_t nreq, const uint64_t* arrival_ns, const float* q768,
                     const uint32_t* which, const sg_params* params, const sg_filter* const* filters,
                     const int32_t* filter_of, float* out_latency_ms, uint32_t* out_batch,
                     double* out_wall_s);
/* Runs every queued request to completion, then stops the dispatcher and frees the contexts. */
int sg_server_stop(sg_server* server);

/* ---- bigann: billion-scale L2 search over int8 rows (src/bigann.rs) -------------------- */
typedef struct sg_bigann sg_bigann;
/* bigann::Index::open(dir, base_dir, cache) (src/bigann.rs:635-641) with every record resident:
 * reads centroids.f32, rotation.f32, bits.u64 (absent: 1), block_off.u64, postings.off and
 * postings.bin from index_dir and base.NN (while base.NN.done exists) from base_dir, and uploads
 * them to HBM on `device`. */
int sg_open_bigann(const char* index_dir, const char* base_dir, int device, sg_bigann** out);
/* The same from host arrays (the records already de-interleaved). */
int sg_open_bigann_arrays(const sg_bigann_arrays* a, int device, sg_bigann** out);
int sg_close_bigann(sg_bigann* index);
int sg_bigann_info(const sg_bigann* index, uint32_t* k, uint64_t* n, uint64_t* nblocks,
                   uint32_t* bits);
/* Routing passes (since open) in which some query's tensor-core routing fell back to the exact
 * FP32 dot of every leaf: its emitted list or its rescoring window overflowed. No reference
 * counterpart; the results are the same either way. */
int sg_bigann_route_fallbacks(const sg_bigann* index, uint64_t* passes);
/* bigann::Index::search (src/bigann.rs:653-657) for nq int8 queries q100 [nq * 100]: the top
 * params.k rows by 2<q,x> - |x|^2 as (score, row), best first. out_* [nq * k], out_counts [nq]. */
int sg_search_bigann(sg_bigann* index, uint32_t nq, const int8_t* q100,
                     const sg_bigann_params* params, float* out_scores, uint32_t* out_ids,
                     uint32_t* out_counts, sg_bigann_timing* timing);
/* The same with device pointers, ordered after `stream` (cudaStream_t). */
int sg_search_bigann_device(sg_bigann* index, uint32_t nq, const int8_t* d_q100,
                            const sg_bigann_params* params, float* d_out_scores,
                            uint32_t* d_out_ids, uint32_t* d_out_counts, void* stream);
/* bigann::Index::route (src/bigann.rs:660-678): the probed leaves, best first.
 * out_probe [nq * min(nprobe, k)], out_counts [nq]. */
int sg_bigann_route(sg_bigann* index, uint32_t nq, const int8_t* q100,
                    const sg_bigann_params* params, uint32_t* out_probe, uint32_t* out_counts);
/* bigann::Index::candidates (src/bigann.rs:683-732) after the index's own routing: the best
 * params.cand slots as (row, estimate, |x|^2), best first. out_* [nq * cand], out_counts [nq]. */
int sg_bigann_candidates(sg_bigann* index, uint32_t nq, const int8_t* q100,
                         const sg_bigann_params* params, uint32_t* out_ids, float* out_est,
                         float* out_nx, uint32_t* out_counts);

/* ---- autotuner (no counterpart in the reference: the shapes of the batched GPU path) ------ */
typedef struct {
  uint32_t tc_min_queries;    /* clusters probed by fewer queries of a batch go to the ALU scan,
                                 the others to the tcgen05 scan                                  */
  uint32_t chunk_blocks;      /* ALU scan work-item size, blocks (64..512)                      */
  uint32_t scan_ctas_per_sm;  /* ALU scan CTAs per SM (1 or 2)                                   */
  uint32_t seed_blocks;       /* block budget of each query's seed pass (1..512)                */
  uint32_t tc_split;          /* > 1: probe ranks below it are scanned first and each query's
                                 threshold raised to its buffer's cand-th estimate (0: off)      */
} sg_tuning;
int sg_get_tuning(const sg_index* index, sg_tuning* out);
/* Applies to batches of >= 64 queries; captured CUDA graphs of the previous tuning are retired. */
int sg_set_tuning(sg_index* index, const sg_tuning* tuning);
/* Times the caller's batch (nq device-resident queries, params) under candidate tunings, one
 * field at a time (coordinate descent, best of `reps` device-timed runs each), and keeps the
 * fastest. Results are identical under every tuning. out_ms[0], out_ms[1]: the batch's device
 * time before and after, ms (either output may be null). */
int sg_autotune(sg_index* index, uint32_t nq, const float* d_q768, const float* d_q256,
                const sg_params* params, uint32_t reps, sg_tuning* out, float* out_ms);

/* ---- kernel-level entry points (parity tests and micro-benchmarks) ----------------------- */
/* rabitq::Query::new (src/rabitq.rs:119-125) on the device: rotated LUT tables [nq*64*16] u8,
 * and per query scale, bias, a, b. */
int sg_query_prep(sg_index* index, uint32_t nq, const float* q256, uint8_t* out_tables,
                  float* out_scale, float* out_bias, float* out_a, float* out_b);
/* lut::scan (src/lut.rs:96-126) for G = groups (64 or 32): u16 scores of nblocks blocks,
 * 32 per block, against one u8 table set [groups * 16]. Stateless (no index needed). */
int sg_lut_scan(uint32_t groups, const uint8_t* tables, const uint8_t* blocks, uint64_t nblocks,
                uint16_t* out_scores);
/* lut::scan (src/lut.rs:96-126, G = 64) of nq query table sets [nq * 64 * 16] against nblocks
 * blocks, on the tcgen05 tensor cores (the contraction of the batched scan): u16 scores
 * out_scores[q * nblocks * 32 + slot]. Stateless. */
int sg_lut_scan_batch(uint32_t nq, const uint8_t* tables, const uint8_t* blocks, uint64_t nblocks,
                      uint16_t* out_scores);
/* quant::dot_i8i8 (src/quant.rs:113-125) of one int8 query against `rows` int8 rows of
 * length dim (a multiple of 4): exact int32 dots. Stateless. */
int sg_dot_i8i8(const int8_t* query, const int8_t* rows, uint64_t nrows, uint32_t dim,
                int32_t* out_dots);

#ifdef __cplusplus
}
#endif
#endif /* SIEVE_GPU_H */
