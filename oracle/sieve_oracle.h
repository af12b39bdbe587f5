/*
 * sieve_oracle.h — CPU oracle: a C restatement of the reference's portable query path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links or calls this library; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline / reference arm load it, as the checker.
 *
 * What it restates (file:line of the reference crate, 18Abhinav07/A-Game-Of-Vectors):
 *   splitmix64 Rng ........................ src/ivf.rs:119-135
 *   Rotation (signs, FWHT x3, d^-1.5) ..... src/rabitq.rs:34-84
 *   rabitq::encode / Query / estimate ..... src/rabitq.rs:88-131
 *   Lut::new / score_code / scan ........... src/lut.rs:33-126 (the scalar, non-aarch64 path)
 *   pack_block / unpack_slot ............... src/lut.rs:72-93
 *   TopK ................................... src/topk.rs:4-62 (canonical tie order, see below)
 *   gemm_abt (portable) .................... src/blas.rs:43-54
 *   normalize/prefix/sign_code/Int8Quantizer/query_i8/dot_i8i8/dot_f32/dot_i8 src/quant.rs:6-125
 *   Tier2 fit/encode/tables/score .......... src/tier2.rs:18-75
 *   Index::route/candidates/rerank/search .. src/ivf.rs:543-832
 *   filter::Filter/Plan/search ............. src/filter.rs:27-110
 *   recall_at .............................. src/eval.rs:7-10
 *   bigann refine_encode/Refiner/route/candidates/rerank src/bigann.rs:65-108, :568-602, :653-747
 *
 * Floating point follows the Rust code operation for operation: f32 throughout, no FMA
 * contraction (built with -ffp-contract=off), sums sequential from -0.0 as Rust's
 * `Iterator::sum` for f32, `round` = roundf (half away from zero), f32::min/max = fminf/fmaxf.
 *
 * Tie order. TopK (src/topk.rs) rejects a push whose score is <= the threshold and compacts
 * with select_nth_unstable, so which of several *equal* scores survives at the k-th place is
 * unspecified in the reference. The oracle has two rules (or_set_tie_rule): the canonical one
 * (the default) keeps the k best under the total order (score desc, id asc), which agrees with
 * the reference whenever the survivors are the earlier-pushed of the tied items (the reference's
 * `<=` rejection already prefers them); the reference rule restates TopK's own mechanics
 * (`<=` rejection, a selection by score alone, the k-th score as threshold). Every TopK records
 * whether its k-th place was tied (an item left out with the k-th kept score); or_search_batch
 * reports it per query, so parity runs can tell tied queries from mismatches.
 *
 * Parity pin: the reference is Rust and cannot be built here (no cargo/rustc, no network) and
 * ships no golden vectors. The oracle is pinned by ports of the reference's own unit and
 * property tests (tests/test_oracle_*.py) with their known answers.
 */
#ifndef SIEVE_ORACLE_H
#define SIEVE_ORACLE_H

#include <stdint.h>
#include "../include/sieve_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

uint64_t or_rng_next(uint64_t* state);
uint64_t or_rng_below(uint64_t* state, uint64_t n);

void or_rotation_signs(uint64_t seed, uint32_t d, float* signs);
void or_rotation_apply(const float* signs, uint32_t d, float* v);
float or_rotation_norm(uint32_t d);
void or_rabitq_encode(const float* xr, const float* cr, uint32_t d, uint8_t* code, float* mul_err);

void or_lut_new(const float* q, uint32_t groups, uint8_t* tables, float* scale, float* bias);
uint16_t or_score_code(const uint8_t* tables, uint32_t groups, const uint8_t* code);
float or_float_score(const float* q, uint32_t d, const uint8_t* code);
float or_lut_to_float(float scale, float bias, uint16_t s);
void or_pack_block(const uint8_t* codes, uint32_t ncodes, uint32_t groups, uint8_t* out);
void or_unpack_slot(const uint8_t* block, uint32_t groups, uint32_t k, uint8_t* code);
void or_scan(const uint8_t* tables, uint32_t groups, const uint8_t* blocks, uint64_t nblocks,
             uint16_t* out);
uint32_t or_hamming(const uint8_t* a, const uint8_t* b, uint32_t nbytes);

void or_query_new(const float* signs, uint32_t d, const float* q, uint8_t* tables, float* scale,
                  float* bias, float* a, float* b);
float or_estimate(float a, float b, float cent, float mul, uint16_t s);

float or_normalize(float* v, uint32_t n);
float or_prefix(const float* full, float* out);
void or_sign_code(const float* prefix, uint8_t* out);
void or_int8_fit(const float* rows, uint64_t n, float* scale);
void or_int8_encode(const float* scale, const float* v, int8_t* out);
void or_int8_query_weights(const float* scale, const float* q, uint32_t n, float* w);
float or_dot_i8(const float* w, const int8_t* x, uint32_t n);
float or_dot_f32(const float* a, const float* b, uint32_t n);
float or_query_i8(const float* w, uint32_t n, int8_t* out);
int32_t or_dot_i8i8(const int8_t* a, const int8_t* b, uint32_t n);

void or_tier2_fit(const float* rows, uint64_t n, float* sigma);
float or_tier2_encode(const float* sigma, const float* prefix, uint8_t* out);
void or_tier2_tables(const float* sigma, const float* q, float* tables);
float or_tier2_score(const float* tables, const uint8_t* code, float norm);

/* TopK: pushes (scores[i], ids[i]) in order into TopK::new(k) and returns into_sorted. */
uint32_t or_topk(const float* scores, const uint32_t* ids, uint64_t n, uint32_t k,
                 float* out_scores, uint32_t* out_ids);
void or_gemm_abt(const float* a, const float* b, uint64_t m, uint64_t n, uint64_t k, float* c);

uint32_t or_route(const sg_ivf_arrays* ix, const float* q256, const sg_params* p,
                  float* out_scores, uint32_t* out_clusters);
uint32_t or_candidates(const sg_ivf_arrays* ix, const float* q256, const float* probe_scores,
                       const uint32_t* probe_clusters, uint32_t nprobe, const sg_params* p,
                       const uint64_t* allow, uint64_t allow_words, float* out_est,
                       uint32_t* out_ids, float* out_err, uint64_t* scanned);
float or_prune_threshold(const float* est, const float* err, uint32_t n, uint32_t m, float w);
uint32_t or_rerank(const sg_ivf_arrays* ix, const float* q768, const float* q256,
                   const float* est, const uint32_t* ids, const float* err, uint32_t n,
                   const sg_params* p, float* out_scores, uint32_t* out_ids,
                   uint64_t* reranked);
uint32_t or_search(const sg_ivf_arrays* ix, const float* q768, const float* q256,
                   const sg_params* p, const uint64_t* allow, uint64_t allow_words,
                   float* out_scores, uint32_t* out_ids, sg_timing* t);
/* ivf::build (src/ivf.rs:268-395) over the corpus's int8 rows: centroids [k * 256], tier2 sigma
 * [256], codes [n * 64] and norms [n], block_off [k + 1]; with the returned block count <=
 * max_blocks also ids [nb * 32], blocks [nb * 1024] and factors [nb * 64]. Sample seed 42,
 * k-means seed 7, rotation seed 11, 16 SOAR candidates, as the reference. */
uint64_t or_build_ivf(uint64_t n, const int8_t* rerank, const float* quant_scale, uint32_t k, uint64_t sample_n,
                      uint32_t iters, int has_balance, float balance, int has_soar, float lambda, float* cents,
                      float* sigma, uint8_t* t2_codes, float* t2_norm, uint64_t* block_off, uint32_t* ids,
                      uint8_t* blocks, float* factors, uint64_t max_blocks);
/* Live::apply_insert's encoding of one unit 768-d row v (src/live.rs:274-350); cents_rot are the
 * index's centroids rotated (Live::open, src/live.rs:171-179). Outputs: row [768], *norm256,
 * pair [2] (PAD without SOAR), codes [2 * 32], factors [2 * 2], t2 [64] and *t2_norm (when the
 * index has a 2-bit tier). */
void or_live_encode(const sg_ivf_arrays* ix, const float* cents_rot, int soar, float lambda, const float* v,
                    int8_t* row, float* norm256, uint32_t* pair, uint8_t* codes, float* factors, uint8_t* t2,
                    float* t2_norm);
/* The flat Hamming baseline (src/bin/search.rs:251-269) over codes.bin [n * 32]: out_* [k]. */
uint32_t or_flat_hamming(const uint8_t* codes, uint64_t n, const int8_t* rerank, const float* quant_scale,
                         const float* q768, const float* q256, uint32_t cand, uint32_t k, float* out_scores,
                         uint32_t* out_ids);
/* Many queries over `threads` OpenMP threads (the rayon par_iter of src/bin/search.rs:312-323).
 * out_* are [nq * p->k]; returns the total slots scanned. */
uint64_t or_search_batch(const sg_ivf_arrays* ix, uint32_t nq, const float* q768,
                         const float* q256, const sg_params* p, const uint64_t* allow,
                         uint64_t allow_words, int threads, float* out_scores,
                         uint32_t* out_ids, uint32_t* out_counts, uint8_t* out_tied);
/* Tie rules of every TopK (process-wide; set it before a batch, not during one). */
#define OR_TIE_CANONICAL 0
#define OR_TIE_REFERENCE 1
void or_set_tie_rule(int rule);
int or_tie_rule(void);
/* Whether a TopK on this thread cut a tie since the last or_clear_tied (or batch query). */
int or_last_tied(void);
void or_clear_tied(void);

/* filter.rs: allowed slots per cluster, the Auto plan, and filter::search. */
void or_filter_per_cluster(const sg_ivf_arrays* ix, const uint64_t* allow, uint64_t words,
                           uint32_t* per_cluster);
/* plan: 0 Post, 1 Expand(expand_target), 2 Brute, 3 Auto. Returns the resolved plan. */
int or_plan_resolve(int plan, uint64_t allowed_rows, uint64_t n);
uint32_t or_filter_search(const sg_ivf_arrays* ix, const uint64_t* allow, uint64_t words,
                          const uint32_t* rows, uint64_t nrows, const uint32_t* per_cluster,
                          int plan, uint64_t expand_target, const float* q768,
                          const float* q256, const sg_params* p, float* out_scores,
                          uint32_t* out_ids);

/* bigann.rs: refinement codes, routing, candidates, rerank, search (src/bigann.rs:65-108,
 * :568-602, :653-747). The scan visits the probed leaves in probe order, as Postings::fetch_each
 * does when every record is resident (src/postings.rs:287-317). */
uint32_t or_bg_extra(uint32_t bits);
float or_bg_refine_encode(const float* r, uint32_t bits, uint8_t* planes);
void or_bg_refiner_new(const float* qr, uint32_t bits, float* tab, float* off);
float or_bg_refiner_estimate(const float* tab, float off, uint32_t bits, const uint8_t* sign,
                             const uint8_t* planes, float f);
uint32_t or_bg_route(const sg_bigann_arrays* ix, const int8_t* q, const sg_bigann_params* p,
                     uint32_t* out_probe, float* out_probe_scores, float* dots);
uint32_t or_bg_candidates(const sg_bigann_arrays* ix, const int8_t* q, const uint32_t* probe,
                          uint32_t nprobe, const float* dots, const sg_bigann_params* p,
                          uint32_t* out_ids, float* out_est, float* out_nx, uint64_t* scanned);
uint32_t or_bg_rerank(const sg_bigann_arrays* ix, const int8_t* q, const uint32_t* ids,
                      const float* nx, uint32_t n, const sg_bigann_params* p, float* out_scores,
                      uint32_t* out_ids);
uint32_t or_bg_search(const sg_bigann_arrays* ix, const int8_t* q, const sg_bigann_params* p,
                      float* out_scores, uint32_t* out_ids, sg_bigann_timing* t);
uint64_t or_bg_search_batch(const sg_bigann_arrays* ix, uint32_t nq, const int8_t* q,
                            const sg_bigann_params* p, int threads, float* out_scores,
                            uint32_t* out_ids, uint32_t* out_counts);

double or_recall_at(uint32_t k, const uint32_t* got, uint32_t ngot, const uint32_t* truth,
                    uint32_t ntruth);

#ifdef __cplusplus
}
#endif
#endif
