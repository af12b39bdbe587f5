/*
 * sieve_oracle.c — CPU oracle (test infrastructure only; see sieve_oracle.h for scope,
 * float rules and the tie convention). Every function cites the reference code it restates.
 * Build: oracle/Makefile (gcc -O3 -march=native -ffp-contract=off -fopenmp).
 */
#include "sieve_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NEG0 (-0.0f)

/* ---- splitmix64: src/ivf.rs:119-135 ------------------------------------------------------ */
uint64_t or_rng_next(uint64_t* s) {
  *s += 0x9E3779B97F4A7C15ull;
  uint64_t z = *s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t or_rng_below(uint64_t* s, uint64_t n) { return or_rng_next(s) % n; }

/* ---- Rotation: src/rabitq.rs:34-84 ------------------------------------------------------- */
void or_rotation_signs(uint64_t seed, uint32_t d, float* signs) {
  uint64_t s = seed;
  for (uint32_t i = 0; i < 3 * d; i++) signs[i] = (or_rng_next(&s) & 1) ? 1.0f : -1.0f;
}

static void fwht(float* v, uint32_t n) {
  for (uint32_t h = 1; h < n; h *= 2)
    for (uint32_t blk = 0; blk < n; blk += 2 * h)
      for (uint32_t i = 0; i < h; i++) {
        float x = v[blk + i], y = v[blk + h + i];
        v[blk + i] = x + y;
        v[blk + h + i] = x - y;
      }
}

float or_rotation_norm(uint32_t d) { return powf((float)d, -1.5f); }

void or_rotation_apply(const float* signs, uint32_t d, float* v) {
  for (uint32_t r = 0; r < 3; r++) {
    for (uint32_t i = 0; i < d; i++) v[i] *= signs[r * d + i];
    fwht(v, d);
  }
  float norm = or_rotation_norm(d);
  for (uint32_t i = 0; i < d; i++) v[i] *= norm;
}

/* rabitq::encode: src/rabitq.rs:88-108 */
void or_rabitq_encode(const float* xr, const float* cr, uint32_t d, uint8_t* code,
                      float* mul_err) {
  memset(code, 0, d / 8);
  float nr2 = 0.0f, l1 = 0.0f;
  for (uint32_t i = 0; i < d; i++) {
    float r = xr[i] - cr[i];
    nr2 += r * r;
    l1 += fabsf(r);
    if (r > 0.0f) code[i >> 3] |= (uint8_t)(1u << (i & 7));
  }
  if (l1 < 1e-12f) {
    mul_err[0] = 0.0f;
    mul_err[1] = 0.0f;
    return;
  }
  float df = (float)d;
  float nr = sqrtf(nr2);
  float od = l1 / (nr * sqrtf(df));
  float inner = (1.0f - od * od) / (od * od * (df - 1.0f));
  float err = nr * 1.9f * sqrtf(fmaxf(inner, 0.0f));
  mul_err[0] = nr2 / l1;
  mul_err[1] = err;
}

/* ---- Lut: src/lut.rs:33-126 -------------------------------------------------------------- */
void or_lut_new(const float* q, uint32_t groups, uint8_t* tables, float* scale_out,
                float* bias_out) {
  float* f = (float*)malloc(sizeof(float) * groups * 16);
  float* mins = (float*)malloc(sizeof(float) * groups);
  for (uint32_t g = 0; g < groups; g++)
    for (uint32_t c = 0; c < 16; c++) {
      float s = NEG0;
      for (uint32_t j = 0; j < 4; j++)
        if ((c >> j) & 1) s += q[4 * g + j];
      f[g * 16 + c] = s;
    }
  for (uint32_t g = 0; g < groups; g++) {
    float m = FLT_MAX;
    for (uint32_t c = 0; c < 16; c++) m = fminf(m, f[g * 16 + c]);
    mins[g] = m;
  }
  float max_range = 0.0f;
  for (uint32_t g = 0; g < groups; g++) {
    float mx = -FLT_MAX;
    for (uint32_t c = 0; c < 16; c++) mx = fmaxf(mx, f[g * 16 + c]);
    max_range = fmaxf(max_range, mx - mins[g]);
  }
  float scale = max_range > 0.0f ? 255.0f / max_range : 1.0f;
  for (uint32_t g = 0; g < groups; g++)
    for (uint32_t c = 0; c < 16; c++) {
      float v = roundf((f[g * 16 + c] - mins[g]) * scale);
      v = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
      tables[g * 16 + c] = (uint8_t)v;
    }
  float bias = NEG0;
  for (uint32_t g = 0; g < groups; g++) bias += mins[g];
  *scale_out = scale;
  *bias_out = bias;
  free(f);
  free(mins);
}

static inline uint8_t nibble(const uint8_t* code, uint32_t g) {
  return (uint8_t)((code[g >> 1] >> ((g & 1) * 4)) & 0x0F);
}

uint16_t or_score_code(const uint8_t* tables, uint32_t groups, const uint8_t* code) {
  uint16_t s = 0;
  for (uint32_t g = 0; g < groups; g++) s = (uint16_t)(s + tables[g * 16 + nibble(code, g)]);
  return s;
}

float or_float_score(const float* q, uint32_t d, const uint8_t* code) {
  float s = NEG0;
  for (uint32_t i = 0; i < d; i++)
    if ((code[i >> 3] >> (i & 7)) & 1) s += q[i];
  return s;
}

float or_lut_to_float(float scale, float bias, uint16_t s) { return (float)s / scale + bias; }

/* pack_block: src/lut.rs:72-82; `codes` holds ncodes raw codes of groups/2 bytes each. */
void or_pack_block(const uint8_t* codes, uint32_t ncodes, uint32_t groups, uint8_t* out) {
  uint32_t cb = groups / 2;
  for (uint32_t g = 0; g < groups; g++)
    for (uint32_t k = 0; k < 16; k++) {
      uint8_t lo = k < ncodes ? nibble(codes + (size_t)k * cb, g) : 0;
      uint8_t hi = k + 16 < ncodes ? nibble(codes + (size_t)(k + 16) * cb, g) : 0;
      out[g * 16 + k] = (uint8_t)(lo | (hi << 4));
    }
}

/* unpack_slot: src/lut.rs:84-93 */
void or_unpack_slot(const uint8_t* block, uint32_t groups, uint32_t k, uint8_t* code) {
  memset(code, 0, groups / 2);
  for (uint32_t g = 0; g < groups; g++) {
    uint8_t b = block[g * 16 + (k & 15)];
    uint8_t nib = k < 16 ? (b & 0x0F) : (b >> 4);
    code[g >> 1] |= (uint8_t)(nib << ((g & 1) * 4));
  }
}

/* scan + scan_block_scalar: src/lut.rs:96-102, :116-126 */
void or_scan(const uint8_t* tables, uint32_t groups, const uint8_t* blocks, uint64_t nblocks,
             uint16_t* out) {
  for (uint64_t b = 0; b < nblocks; b++) {
    const uint8_t* blk = blocks + b * (uint64_t)groups * 16;
    uint16_t* o = out + b * 32;
    for (int k = 0; k < 32; k++) o[k] = 0;
    for (uint32_t g = 0; g < groups; g++) {
      const uint8_t* t = tables + g * 16;
      for (uint32_t k = 0; k < 16; k++) {
        uint8_t by = blk[g * 16 + k];
        o[k] = (uint16_t)(o[k] + t[by & 0x0F]);
        o[k + 16] = (uint16_t)(o[k + 16] + t[by >> 4]);
      }
    }
  }
}

/* hamming: src/lut.rs:156-165 */
uint32_t or_hamming(const uint8_t* a, const uint8_t* b, uint32_t nbytes) {
  uint32_t s = 0;
  for (uint32_t i = 0; i + 8 <= nbytes; i += 8) {
    uint64_t x, y;
    memcpy(&x, a + i, 8);
    memcpy(&y, b + i, 8);
    s += (uint32_t)__builtin_popcountll(x ^ y);
  }
  return s;
}

/* rabitq::Query::new / estimate: src/rabitq.rs:118-130 */
void or_query_new(const float* signs, uint32_t d, const float* q, uint8_t* tables, float* scale,
                  float* bias, float* a, float* b) {
  float* qr = (float*)malloc(sizeof(float) * d);
  memcpy(qr, q, sizeof(float) * d);
  or_rotation_apply(signs, d, qr);
  or_lut_new(qr, d / 4, tables, scale, bias);
  float sum = NEG0;
  for (uint32_t i = 0; i < d; i++) sum += qr[i];
  *a = 2.0f / *scale;
  *b = 2.0f * *bias - sum;
  free(qr);
}

float or_estimate(float a, float b, float cent, float mul, uint16_t s) {
  return cent + mul * (a * (float)s + b);
}

/* ---- quant.rs: src/quant.rs:6-125 -------------------------------------------------------- */
float or_normalize(float* v, uint32_t n) {
  float s = NEG0;
  for (uint32_t i = 0; i < n; i++) s += v[i] * v[i];
  float nrm = sqrtf(s);
  if (nrm > 0.0f) {
    float inv = 1.0f / nrm;
    for (uint32_t i = 0; i < n; i++) v[i] *= inv;
  }
  return nrm;
}

float or_prefix(const float* full, float* out) {
  memcpy(out, full, sizeof(float) * SG_PDIM);
  return or_normalize(out, SG_PDIM);
}

void or_sign_code(const float* prefix, uint8_t* out) {
  memset(out, 0, SG_CODE_BYTES);
  for (uint32_t i = 0; i < SG_PDIM; i++)
    if (prefix[i] > 0.0f) out[i >> 3] |= (uint8_t)(1u << (i & 7));
}

void or_int8_fit(const float* rows, uint64_t n, float* scale) {
  float m[SG_DIM];
  for (int i = 0; i < SG_DIM; i++) m[i] = 1e-6f;
  for (uint64_t r = 0; r < n; r++)
    for (int i = 0; i < SG_DIM; i++) m[i] = fmaxf(m[i], fabsf(rows[r * SG_DIM + i]));
  for (int i = 0; i < SG_DIM; i++) scale[i] = 127.0f / m[i];
}

static inline int8_t clamp_i8(float v, float lo, float hi) {
  v = v < lo ? lo : (v > hi ? hi : v);
  return (int8_t)v;
}

void or_int8_encode(const float* scale, const float* v, int8_t* out) {
  for (int i = 0; i < SG_DIM; i++) out[i] = clamp_i8(roundf(v[i] * scale[i]), -127.0f, 127.0f);
}

void or_int8_query_weights(const float* scale, const float* q, uint32_t n, float* w) {
  for (uint32_t i = 0; i < n; i++) w[i] = q[i] / scale[i];
}

float or_dot_i8(const float* w, const int8_t* x, uint32_t n) {
  float acc[16];
  for (int i = 0; i < 16; i++) acc[i] = 0.0f;
  uint32_t full = n / 16 * 16;
  for (uint32_t c = 0; c < full; c += 16)
    for (int i = 0; i < 16; i++) acc[i] += w[c + i] * (float)x[c + i];
  float tail = NEG0;
  for (uint32_t i = full; i < n; i++) tail += w[i] * (float)x[i];
  float s = NEG0;
  for (int i = 0; i < 16; i++) s += acc[i];
  return s + tail;
}

float or_dot_f32(const float* a, const float* b, uint32_t n) {
  float acc[16];
  for (int i = 0; i < 16; i++) acc[i] = 0.0f;
  uint32_t full = n / 16 * 16;
  for (uint32_t c = 0; c < full; c += 16)
    for (int i = 0; i < 16; i++) acc[i] += a[c + i] * b[c + i];
  float tail = NEG0;
  for (uint32_t i = full; i < n; i++) tail += a[i] * b[i];
  float s = NEG0;
  for (int i = 0; i < 16; i++) s += acc[i];
  return s + tail;
}

/* query_i8: src/quant.rs:104-110. Rust's `as i8` saturates. */
float or_query_i8(const float* w, uint32_t n, int8_t* out) {
  float m = 1e-12f;
  for (uint32_t i = 0; i < n; i++) m = fmaxf(m, fabsf(w[i]));
  float s = 127.0f / m;
  for (uint32_t i = 0; i < n; i++) out[i] = clamp_i8(roundf(w[i] * s), -128.0f, 127.0f);
  return s;
}

int32_t or_dot_i8i8(const int8_t* a, const int8_t* b, uint32_t n) {
  int32_t s = 0;
  for (uint32_t i = 0; i < n; i++) s += (int32_t)a[i] * (int32_t)b[i];
  return s;
}

/* ---- tier2.rs: src/tier2.rs:18-75 --------------------------------------------------------- */
static const float T2_T = 0.9816f;
static const float T2_LEVELS[4] = {-1.510f, -0.4528f, 0.4528f, 1.510f};

void or_tier2_fit(const float* rows, uint64_t n, float* sigma) {
  double ss[SG_PDIM];
  for (int i = 0; i < SG_PDIM; i++) ss[i] = 0.0;
  float nf = (float)(n > 0 ? n : 1);
  for (uint64_t r = 0; r < n; r++)
    for (int i = 0; i < SG_PDIM; i++) {
      float x = rows[r * SG_PDIM + i];
      ss[i] += (double)(x * x);
    }
  for (int i = 0; i < SG_PDIM; i++) sigma[i] = fmaxf((float)sqrt(ss[i] / (double)nf), 1e-6f);
}

static inline uint8_t t2_level(float x, float s) {
  float t = T2_T * s;
  if (x < -t) return 0;
  if (x < 0.0f) return 1;
  if (x < t) return 2;
  return 3;
}

float or_tier2_encode(const float* sigma, const float* prefix, uint8_t* out) {
  memset(out, 0, SG_TIER2_BYTES);
  float nn = 0.0f;
  for (int i = 0; i < SG_PDIM; i++) {
    uint8_t l = t2_level(prefix[i], sigma[i]);
    out[i >> 2] |= (uint8_t)(l << ((i & 3) * 2));
    float v = T2_LEVELS[l] * sigma[i];
    nn += v * v;
  }
  return sqrtf(nn);
}

void or_tier2_tables(const float* sigma, const float* q, float* tables) {
  for (int g = 0; g < SG_TIER2_BYTES; g++) {
    float half[2][16];
    for (int h = 0; h < 2; h++)
      for (int b = 0; b < 16; b++) {
        float s = NEG0;
        for (int j = 0; j < 2; j++) {
          int i = 4 * g + 2 * h + j;
          s += q[i] * T2_LEVELS[(b >> (2 * j)) & 3] * sigma[i];
        }
        half[h][b] = s;
      }
    for (int b = 0; b < 256; b++) tables[g * 256 + b] = half[0][b & 15] + half[1][b >> 4];
  }
}

float or_tier2_score(const float* tables, const uint8_t* code, float norm) {
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int g = 0; g < SG_TIER2_BYTES; g++) acc[g & 3] += tables[g * 256 + code[g]];
  return (acc[0] + acc[1] + acc[2] + acc[3]) / norm;
}

/* ---- TopK: src/topk.rs:4-62 (two tie rules, see header) -------------------------------- */
typedef struct {
  float s;
  uint32_t id;
} item;

/* OR_TIE_CANONICAL keeps the k best by (score desc, id asc). OR_TIE_REFERENCE restates the
 * reference's own mechanics: a push is rejected when score <= threshold (src/topk.rs:28-31), a
 * full buffer is cut with a selection by score alone (select_nth_unstable_by, src/topk.rs:38-44)
 * and the threshold becomes the k-th score; only the final sort orders (score desc, id asc)
 * (src/topk.rs:57-61). Which of several equal scores the selection keeps is unspecified in
 * Rust; this selection is a median-of-three Hoare quickselect, so the two rules can differ only
 * on a query whose boundary is tied, which every TopK records (see `tied` below). */
static int g_tie_rule = OR_TIE_CANONICAL;
void or_set_tie_rule(int rule) { g_tie_rule = rule == OR_TIE_REFERENCE ? OR_TIE_REFERENCE : OR_TIE_CANONICAL; }
int or_tie_rule(void) { return g_tie_rule; }

/* Set when any TopK of the current query (on this thread) cut a tie at its k-th place. */
static _Thread_local int g_tied = 0;

static inline int better(item a, item b) {
  if (g_tie_rule == OR_TIE_REFERENCE) return a.s > b.s;
  return a.s > b.s || (a.s == b.s && a.id < b.id);
}

static void select_nth(item* v, int64_t n, int64_t kth) {
  int64_t lo = 0, hi = n - 1;
  while (hi > lo) {
    int64_t mid = lo + (hi - lo) / 2;
    /* median of three as pivot */
    item a = v[lo], b = v[mid], c = v[hi], p;
    if (better(a, b)) p = better(b, c) ? b : (better(a, c) ? c : a);
    else p = better(a, c) ? a : (better(b, c) ? c : b);
    int64_t i = lo, j = hi;
    while (i <= j) {
      while (better(v[i], p)) i++;
      while (better(p, v[j])) j--;
      if (i <= j) {
        item t = v[i];
        v[i] = v[j];
        v[j] = t;
        i++;
        j--;
      }
    }
    if (kth <= j) hi = j;
    else if (kth >= i) lo = i;
    else return;
  }
}

typedef struct {
  uint32_t k;
  item* items;
  uint32_t len;
  int has_thr;
  item thr;
  int has_out;  /* some item was rejected or cut off; out_s is the best such score */
  float out_s;
} topk;

static void topk_init(topk* t, uint32_t k) {
  t->k = k ? k : 1;
  t->items = (item*)malloc(sizeof(item) * 2 * t->k);
  t->len = 0;
  t->has_thr = 0;
  t->has_out = 0;
}

static inline void topk_left_out(topk* t, float s) {
  if (!t->has_out || s > t->out_s) t->out_s = s;
  t->has_out = 1;
}

static void topk_free(topk* t) { free(t->items); }

static void topk_compact(topk* t) {
  if (t->len > t->k) {
    select_nth(t->items, t->len, t->k - 1);
    for (uint32_t i = t->k; i < t->len; i++) topk_left_out(t, t->items[i].s);
    t->len = t->k;
    /* the k-th best (worst kept) becomes the admission threshold */
    item w = t->items[0];
    for (uint32_t i = 1; i < t->len; i++)
      if (better(w, t->items[i])) w = t->items[i];
    t->thr = w;
    t->has_thr = 1;
  }
}

/* Would a push of (s, id) enter? The canonical rule's order agrees with the reference's
 * `score <= threshold` rejection for the push orders the query path uses (ids rising with push
 * order); the reference rule is that rejection itself. A rejected item is recorded as left out. */
static inline int topk_admits(topk* t, float s, uint32_t id) {
  if (!t->has_thr) return 1;
  item x = {s, id};
  if (better(x, t->thr)) return 1;
  topk_left_out(t, s);
  return 0;
}

static inline void topk_push(topk* t, float s, uint32_t id) {
  if (!topk_admits(t, s, id)) return;
  t->items[t->len].s = s;
  t->items[t->len].id = id;
  t->len++;
  if (t->len >= 2 * t->k) topk_compact(t);
}

static int cmp_item_final(const void* x, const void* y) {
  item a = *(const item*)x, b = *(const item*)y;
  if (a.s != b.s) return a.s > b.s ? -1 : 1;
  return a.id < b.id ? -1 : (a.id > b.id);
}

/* into_sorted (src/topk.rs:57-61): the kept items by (score desc, id asc). A left-out item whose
 * score equals the k-th kept score means the cut at the k-th place was tied. */
static uint32_t topk_sorted(topk* t) {
  topk_compact(t);
  qsort(t->items, t->len, sizeof(item), cmp_item_final);
  if (t->len > t->k) t->len = t->k;
  if (t->has_out && t->len == t->k && t->items[t->len - 1].s == t->out_s) g_tied = 1;
  return t->len;
}

uint32_t or_topk(const float* scores, const uint32_t* ids, uint64_t n, uint32_t k,
                 float* out_scores, uint32_t* out_ids) {
  if (k == 0) return 0;
  topk t;
  topk_init(&t, k);
  for (uint64_t i = 0; i < n; i++) topk_push(&t, scores[i], ids[i]);
  uint32_t m = topk_sorted(&t);
  for (uint32_t i = 0; i < m; i++) {
    out_scores[i] = t.items[i].s;
    out_ids[i] = t.items[i].id;
  }
  topk_free(&t);
  return m;
}

/* ---- gemm_abt portable: src/blas.rs:43-54 ----------------------------------------------- */
void or_gemm_abt(const float* a, const float* b, uint64_t m, uint64_t n, uint64_t k, float* c) {
  for (uint64_t i = 0; i < m; i++)
    for (uint64_t j = 0; j < n; j++) {
      float s = NEG0;
      const float* x = a + i * k;
      const float* y = b + j * k;
      for (uint64_t t = 0; t < k; t++) s += x[t] * y[t];
      c[i * n + j] = s;
    }
}

/* ---- Index::route: src/ivf.rs:589-618 ---------------------------------------------------- */
static inline uint64_t cluster_slots(const sg_ivf_arrays* ix, uint32_t c) {
  return (ix->block_off[c + 1] - ix->block_off[c]) * SG_BLOCK;
}

uint32_t or_route(const sg_ivf_arrays* ix, const float* q256, const sg_params* p,
                  float* out_scores, uint32_t* out_clusters) {
  uint32_t K = ix->k;
  float* cent = (float*)malloc(sizeof(float) * K);
  or_gemm_abt(q256, ix->centroids, 1, K, SG_PDIM, cent);
  uint32_t np = p->nprobe < K ? p->nprobe : K;
  uint32_t m = 0;
  if (np > 0) {
    topk t;
    topk_init(&t, np);
    for (uint32_t c = 0; c < K; c++) topk_push(&t, cent[c], c);
    m = topk_sorted(&t);
    for (uint32_t i = 0; i < m; i++) {
      out_scores[i] = t.items[i].s;
      out_clusters[i] = t.items[i].id;
    }
    topk_free(&t);
  }
  if (p->has_margin && m > 0) {
    float lim = out_scores[0] - p->margin;
    uint32_t w = 0;
    for (uint32_t i = 0; i < m; i++)
      if (out_scores[i] >= lim) {
        out_scores[w] = out_scores[i];
        out_clusters[w] = out_clusters[i];
        w++;
      }
    m = w;
  }
  if (p->has_budget) {
    uint64_t used = 0;
    uint32_t keep = 0;
    for (uint32_t i = 0; i < m; i++) {
      used += cluster_slots(ix, out_clusters[i]);
      if (used <= p->budget) keep++;
      else break;
    }
    if (keep < 1) keep = 1;
    if (keep < m) m = keep;
  }
  free(cent);
  return m;
}

/* ---- View::hidden for an allow bitset: src/ivf.rs:474-483 -------------------------------- */
static inline int allowed(const uint64_t* allow, uint64_t words, uint32_t id) {
  uint64_t w = (uint64_t)id >> 6;
  return w < words && ((allow[w] >> (id & 63)) & 1);
}

/* ---- Index::candidates (RaBitQ branch): src/ivf.rs:647-729 ------------------------------ */
typedef struct {
  float est;
  uint32_t id;
  float err;
  uint32_t order; /* admission order, the tie-break of the dedup sort */
} cand3;

static inline uint32_t f32_ordered(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* sort_unstable_by(id asc, est desc by total_cmp), admission order as the final tie-break */
static int cmp_dedup(const void* x, const void* y) {
  const cand3* a = (const cand3*)x;
  const cand3* b = (const cand3*)y;
  if (a->id != b->id) return a->id < b->id ? -1 : 1;
  uint32_t ea = f32_ordered(a->est), eb = f32_ordered(b->est);
  if (ea != eb) return ea > eb ? -1 : 1;
  return a->order < b->order ? -1 : (a->order > b->order);
}

/* Index::candidates over global sign codes (the `None` branch, src/ivf.rs:700-717): Lut::new on
 * the unrotated prefix, TopK(cand) of the u16 LUT scores keyed by corpus row, then estimates
 * lut.to_float(score) and an infinite error width (pruning keeps every such candidate). */
static uint32_t candidates_global(const sg_ivf_arrays* ix, const float* q256,
                                  const uint32_t* probe_clusters, uint32_t nprobe, const sg_params* p,
                                  const uint64_t* allow, uint64_t allow_words, float* out_est,
                                  uint32_t* out_ids, float* out_err, uint64_t* scanned) {
  uint8_t tables[SG_GROUPS * 16];
  float scale, bias;
  or_lut_new(q256, SG_GROUPS, tables, &scale, &bias);
  topk cand;
  topk_init(&cand, p->cand);
  uint16_t* scores = NULL;
  size_t scores_cap = 0;
  uint64_t nscanned = 0;
  for (uint32_t pi = 0; pi < nprobe; pi++) {
    uint32_t c = probe_clusters[pi];
    uint64_t b0 = ix->block_off[c], b1 = ix->block_off[c + 1];
    size_t ns = (size_t)(b1 - b0) * SG_BLOCK;
    if (ns > scores_cap) {
      scores_cap = ns;
      scores = (uint16_t*)realloc(scores, sizeof(uint16_t) * ns);
    }
    or_scan(tables, SG_GROUPS, ix->blocks + b0 * SG_BLOCK_BYTES, b1 - b0, scores);
    nscanned += ns;
    const uint32_t* ids = ix->ids + b0 * SG_BLOCK;
    for (size_t j = 0; j < ns; j++) {
      uint32_t id = ids[j];
      if (id == SG_PAD) continue;
      if (allow && !allowed(allow, allow_words, id)) continue;
      float sc = (float)scores[j];
      if (!topk_admits(&cand, sc, id)) continue;
      topk_push(&cand, sc, id);
    }
  }
  uint32_t m = topk_sorted(&cand);
  cand3* v = (cand3*)malloc(sizeof(cand3) * (m ? m : 1));
  for (uint32_t i = 0; i < m; i++) {
    v[i].est = or_lut_to_float(scale, bias, (uint16_t)cand.items[i].s);
    v[i].id = cand.items[i].id;
    v[i].err = INFINITY;
    v[i].order = i;
  }
  qsort(v, m, sizeof(cand3), cmp_dedup);
  uint32_t w = 0;
  for (uint32_t i = 0; i < m; i++) {
    if (w > 0 && v[i].id == out_ids[w - 1]) continue;
    out_est[w] = v[i].est;
    out_ids[w] = v[i].id;
    out_err[w] = v[i].err;
    w++;
  }
  if (scanned) *scanned += nscanned;
  free(v);
  free(scores);
  topk_free(&cand);
  return w;
}

uint32_t or_candidates(const sg_ivf_arrays* ix, const float* q256, const float* probe_scores,
                       const uint32_t* probe_clusters, uint32_t nprobe, const sg_params* p,
                       const uint64_t* allow, uint64_t allow_words, float* out_est,
                       uint32_t* out_ids, float* out_err, uint64_t* scanned) {
  if (!ix->rotation || !ix->factors)
    return candidates_global(ix, q256, probe_clusters, nprobe, p, allow, allow_words, out_est, out_ids,
                             out_err, scanned);
  uint8_t tables[SG_GROUPS * 16];
  float scale, bias, a, b;
  or_query_new(ix->rotation, SG_PDIM, q256, tables, &scale, &bias, &a, &b);
  topk cand;
  topk_init(&cand, p->cand);
  size_t meta_cap = 4096, meta_len = 0;
  uint32_t* meta_id = (uint32_t*)malloc(sizeof(uint32_t) * meta_cap);
  float* meta_err = (float*)malloc(sizeof(float) * meta_cap);
  uint16_t* scores = NULL;
  size_t scores_cap = 0;
  uint64_t nscanned = 0;
  for (uint32_t pi = 0; pi < nprobe; pi++) {
    uint32_t c = probe_clusters[pi];
    float cent = probe_scores[pi];
    uint64_t b0 = ix->block_off[c], b1 = ix->block_off[c + 1];
    size_t ns = (size_t)(b1 - b0) * SG_BLOCK;
    if (ns > scores_cap) {
      scores_cap = ns;
      scores = (uint16_t*)realloc(scores, sizeof(uint16_t) * ns);
    }
    or_scan(tables, SG_GROUPS, ix->blocks + b0 * SG_BLOCK_BYTES, b1 - b0, scores);
    nscanned += ns;
    const float* f = ix->factors + b0 * SG_BLOCK * 2;
    const uint32_t* ids = ix->ids + b0 * SG_BLOCK;
    for (size_t j = 0; j < ns; j++) {
      float est = or_estimate(a, b, cent, f[2 * j], scores[j]);
      uint32_t id = ids[j];
      if (id == SG_PAD) continue;
      if (allow && !allowed(allow, allow_words, id)) continue;
      if (!topk_admits(&cand, est, (uint32_t)meta_len)) continue;
      topk_push(&cand, est, (uint32_t)meta_len);
      if (meta_len == meta_cap) {
        meta_cap *= 2;
        meta_id = (uint32_t*)realloc(meta_id, sizeof(uint32_t) * meta_cap);
        meta_err = (float*)realloc(meta_err, sizeof(float) * meta_cap);
      }
      meta_id[meta_len] = id;
      meta_err[meta_len] = f[2 * j + 1];
      meta_len++;
    }
  }
  uint32_t m = topk_sorted(&cand);
  cand3* v = (cand3*)malloc(sizeof(cand3) * (m ? m : 1));
  for (uint32_t i = 0; i < m; i++) {
    uint32_t k = cand.items[i].id;
    v[i].est = cand.items[i].s;
    v[i].id = meta_id[k];
    v[i].err = meta_err[k];
    v[i].order = k;
  }
  qsort(v, m, sizeof(cand3), cmp_dedup);
  uint32_t w = 0;
  for (uint32_t i = 0; i < m; i++) {
    if (w > 0 && v[i].id == out_ids[w - 1]) continue;
    out_est[w] = v[i].est;
    out_ids[w] = v[i].id;
    out_err[w] = v[i].err;
    w++;
  }
  if (scanned) *scanned += nscanned;
  free(v);
  free(scores);
  free(meta_id);
  free(meta_err);
  topk_free(&cand);
  return w;
}

/* prune_threshold: src/ivf.rs:540-550 (m-th largest lower bound by total_cmp) */
static int cmp_desc_total(const void* x, const void* y) {
  uint32_t a = f32_ordered(*(const float*)x), b = f32_ordered(*(const float*)y);
  return a > b ? -1 : (a < b);
}

float or_prune_threshold(const float* est, const float* err, uint32_t n, uint32_t m, float w) {
  if (m == 0 || n < m) return -INFINITY;
  float* lo = (float*)malloc(sizeof(float) * n);
  for (uint32_t i = 0; i < n; i++) lo[i] = est[i] - w * err[i];
  qsort(lo, n, sizeof(float), cmp_desc_total);
  float v = lo[m - 1];
  free(lo);
  return v;
}

/* ---- rerank: src/ivf.rs:734-832 ---------------------------------------------------------- */
static float query_weights_i8(const float* quant_scale, const float* q, uint32_t n, int8_t* wq) {
  float w[SG_DIM];
  for (uint32_t i = 0; i < n; i++) w[i] = q[i] / quant_scale[i];
  float s = or_query_i8(w, n, wq);
  return 1.0f / s;
}

/* read_and_rerank: src/ivf.rs:819-832 (every id is a base row here) */
static void read_and_rerank(const sg_ivf_arrays* ix, const float* q768, const uint32_t* ids,
                            uint32_t n, topk* out) {
  int8_t wq[SG_DIM];
  float inv = query_weights_i8(ix->quant_scale, q768, SG_DIM, wq);
  for (uint32_t i = 0; i < n; i++)
    topk_push(out, (float)or_dot_i8i8(wq, ix->rerank + (uint64_t)ids[i] * SG_DIM, SG_DIM) * inv,
              ids[i]);
}

uint32_t or_rerank(const sg_ivf_arrays* ix, const float* q768, const float* q256,
                   const float* est_in, const uint32_t* ids_in, const float* err_in, uint32_t n,
                   const sg_params* p, float* out_scores, uint32_t* out_ids,
                   uint64_t* reranked) {
  float* est = (float*)malloc(sizeof(float) * (n ? n : 1));
  uint32_t* ids = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t m = 0;
  if (p->has_prune) {
    float tau = or_prune_threshold(est_in, err_in, n, p->prune_m, p->prune_w);
    for (uint32_t i = 0; i < n; i++)
      if (est_in[i] + p->prune_w * err_in[i] >= tau) {
        est[m] = est_in[i];
        ids[m] = ids_in[i];
        m++;
      }
  } else {
    memcpy(est, est_in, sizeof(float) * n);
    memcpy(ids, ids_in, sizeof(uint32_t) * n);
    m = n;
  }
  if (reranked) *reranked += m;
  topk out;
  topk_init(&out, p->k);
  int kind = (int)p->rerank_kind;
  int have_t2 = ix->tier2_codes != NULL && ix->tier2_norm != NULL && ix->tier2_sigma != NULL;
  if (kind == SG_RERANK_NONE) {
    for (uint32_t i = 0; i < m; i++) topk_push(&out, est[i], ids[i]);
  } else if (kind == SG_RERANK_FULL) {
    read_and_rerank(ix, q768, ids, m, &out);
  } else if (kind == SG_RERANK_SSD) {
    topk best;
    topk_init(&best, p->rerank_r);
    for (uint32_t i = 0; i < m; i++) topk_push(&best, est[i], ids[i]);
    uint32_t r = p->rerank_r ? topk_sorted(&best) : 0;
    uint32_t sel[r ? r : 1];
    for (uint32_t i = 0; i < r; i++) sel[i] = best.items[i].id;
    read_and_rerank(ix, q768, sel, r, &out);
    topk_free(&best);
  } else if (kind == SG_RERANK_TIERED && have_t2) {
    float* tables = (float*)malloc(sizeof(float) * SG_TIER2_BYTES * 256);
    or_tier2_tables(ix->tier2_sigma, q256, tables);
    topk pre;
    topk_init(&pre, p->rerank_r);
    for (uint32_t i = 0; i < m; i++) {
      uint32_t id = ids[i];
      topk_push(&pre,
                or_tier2_score(tables, ix->tier2_codes + (uint64_t)id * SG_TIER2_BYTES,
                               ix->tier2_norm[id]),
                id);
    }
    uint32_t r = p->rerank_r ? topk_sorted(&pre) : 0;
    uint32_t* sel = (uint32_t*)malloc(sizeof(uint32_t) * (r ? r : 1));
    for (uint32_t i = 0; i < r; i++) sel[i] = pre.items[i].id;
    read_and_rerank(ix, q768, sel, r, &out);
    free(sel);
    free(tables);
    topk_free(&pre);
  } else { /* Prefix, or Tiered without a tier-2 file */
    int8_t wq[SG_PDIM];
    float inv = query_weights_i8(ix->quant_scale, q256, SG_PDIM, wq);
    uint32_t pk = kind == SG_RERANK_TIERED ? p->rerank_r : p->k;
    topk pre;
    topk_init(&pre, pk);
    for (uint32_t i = 0; i < m; i++) {
      uint32_t id = ids[i];
      float s = (float)or_dot_i8i8(wq, ix->rerank + (uint64_t)id * SG_DIM, SG_PDIM) * inv /
                ix->norm256[id];
      topk_push(&pre, s, id);
    }
    if (kind == SG_RERANK_PREFIX) {
      topk_free(&out);
      out = pre;
    } else {
      uint32_t r = pk ? topk_sorted(&pre) : 0;
      uint32_t* sel = (uint32_t*)malloc(sizeof(uint32_t) * (r ? r : 1));
      for (uint32_t i = 0; i < r; i++) sel[i] = pre.items[i].id;
      read_and_rerank(ix, q768, sel, r, &out);
      free(sel);
      topk_free(&pre);
    }
  }
  uint32_t k = p->k ? topk_sorted(&out) : 0;
  for (uint32_t i = 0; i < k; i++) {
    out_scores[i] = out.items[i].s;
    out_ids[i] = out.items[i].id;
  }
  topk_free(&out);
  free(est);
  free(ids);
  return k;
}

/* Index::search_view: src/ivf.rs:621-633 */
uint32_t or_search(const sg_ivf_arrays* ix, const float* q768, const float* q256,
                   const sg_params* p, const uint64_t* allow, uint64_t allow_words,
                   float* out_scores, uint32_t* out_ids, sg_timing* t) {
  uint32_t np = p->nprobe < ix->k ? p->nprobe : ix->k;
  float* ps = (float*)malloc(sizeof(float) * (np ? np : 1));
  uint32_t* pc = (uint32_t*)malloc(sizeof(uint32_t) * (np ? np : 1));
  uint32_t m = or_route(ix, q256, p, ps, pc);
  uint32_t cap = p->cand ? p->cand : 1;
  float* est = (float*)malloc(sizeof(float) * cap);
  uint32_t* ids = (uint32_t*)malloc(sizeof(uint32_t) * cap);
  float* err = (float*)malloc(sizeof(float) * cap);
  uint64_t scanned = 0, reranked = 0;
  uint32_t n = p->cand ? or_candidates(ix, q256, ps, pc, m, p, allow, allow_words, est, ids, err,
                                       &scanned)
                       : 0;
  uint32_t k = or_rerank(ix, q768, q256, est, ids, err, n, p, out_scores, out_ids, &reranked);
  if (t) {
    t->probed += m;
    t->scanned += scanned;
    t->reranked += reranked;
  }
  free(ps);
  free(pc);
  free(est);
  free(ids);
  free(err);
  return k;
}

/* ---- ivf::build: src/ivf.rs:188-395 (the index the query path reads) -------------------- */
static uint32_t soar_secondary(const float* x, const float* cents, const uint32_t* cand, uint32_t nc,
                               float lambda);

/* Corpus::prefix_f32 (src/ivf.rs:110-116): the int8 row's prefix over its scale, normalised. */
static void prefix_f32(const int8_t* rerank, const float* scale, uint64_t i, float* out) {
  for (int d = 0; d < SG_PDIM; d++) out[d] = (float)rerank[i * SG_DIM + d] / scale[d];
  or_normalize(out, SG_PDIM);
}

/* assign (src/ivf.rs:160-162): the first maximum of the sequential f32 dots. */
static uint32_t assign1(const float* x, const float* cents, uint32_t k) {
  uint32_t bj = 0;
  float bv = -FLT_MAX;
  for (uint32_t j = 0; j < k; j++) {
    float s;
    or_gemm_abt(x, cents + (uint64_t)j * SG_PDIM, 1, 1, SG_PDIM, &s);
    if (s > bv) {
      bv = s;
      bj = j;
    }
  }
  return bj;
}

/* split_large (src/ivf.rs:231-254). The reference orders clusters by size with an unstable sort,
 * which leaves equal sizes in an unspecified order; here equal sizes keep cluster order. */
static uint32_t split_large(const float* sample, uint64_t n, const uint32_t* a, const uint64_t* counts,
                            uint32_t k, float* cents, float r, uint64_t* rng) {
  float mean = (float)n / (float)k;
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * k);
  for (uint32_t c = 0; c < k; c++) order[c] = c;
  for (uint32_t i = 1; i < k; i++) { /* stable insertion sort by count desc */
    uint32_t v = order[i];
    int32_t j = (int32_t)i - 1;
    while (j >= 0 && counts[order[j]] < counts[v]) {
      order[j + 1] = order[j];
      j--;
    }
    order[j + 1] = v;
  }
  uint32_t nl = 0;
  while (nl < k && (float)counts[order[nl]] > r * mean) nl++;
  uint32_t ns = 0;
  while (ns < nl && ns < k && (float)counts[order[k - 1 - ns]] < 0.5f * mean) ns++;
  for (uint32_t t = 0; t < ns; t++) {
    uint32_t big = order[t], tiny = order[k - 1 - t];
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < n; i++) cnt += a[i] == big;
    uint64_t pick_k = or_rng_below(rng, cnt), seen = 0, pick = 0;
    for (uint64_t i = 0; i < n; i++)
      if (a[i] == big && seen++ == pick_k) {
        pick = i;
        break;
      }
    memcpy(cents + (uint64_t)tiny * SG_PDIM, sample + pick * SG_PDIM, sizeof(float) * SG_PDIM);
  }
  free(order);
  return ns;
}

/* kmeans (src/ivf.rs:194-225): spherical Lloyd on the sample. */
static void kmeans(const float* sample, uint64_t n, uint32_t k, uint32_t iters, uint64_t seed, int has_balance,
                   float balance, float* cents) {
  uint64_t rng = seed;
  for (uint32_t c = 0; c < k; c++)
    memcpy(cents + (uint64_t)c * SG_PDIM, sample + or_rng_below(&rng, n) * SG_PDIM, sizeof(float) * SG_PDIM);
  uint32_t* a = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  float* sums = (float*)malloc(sizeof(float) * k * SG_PDIM);
  uint64_t* counts = (uint64_t*)malloc(sizeof(uint64_t) * k);
  for (uint32_t it = 0; it < iters; it++) {
    for (uint64_t i = 0; i < n; i++) a[i] = assign1(sample + i * SG_PDIM, cents, k);
    memset(sums, 0, sizeof(float) * k * SG_PDIM);
    memset(counts, 0, sizeof(uint64_t) * k);
    for (uint64_t i = 0; i < n; i++) {
      counts[a[i]]++;
      for (int d = 0; d < SG_PDIM; d++) sums[(uint64_t)a[i] * SG_PDIM + d] += sample[i * SG_PDIM + d];
    }
    for (uint32_t c = 0; c < k; c++) {
      float* dst = cents + (uint64_t)c * SG_PDIM;
      if (counts[c] == 0) {
        memcpy(dst, sample + or_rng_below(&rng, n) * SG_PDIM, sizeof(float) * SG_PDIM);
      } else {
        memcpy(dst, sums + (uint64_t)c * SG_PDIM, sizeof(float) * SG_PDIM);
        or_normalize(dst, SG_PDIM);
      }
    }
    if (has_balance && it + 2 < iters) split_large(sample, n, a, counts, k, cents, balance, &rng);
  }
  free(a);
  free(sums);
  free(counts);
}

uint64_t or_build_ivf(uint64_t n, const int8_t* rerank, const float* quant_scale, uint32_t k, uint64_t sample_n,
                      uint32_t iters, int has_balance, float balance, int has_soar, float lambda, float* cents,
                      float* sigma, uint8_t* t2_codes, float* t2_norm, uint64_t* block_off, uint32_t* ids,
                      uint8_t* blocks, float* factors, uint64_t max_blocks) {
  uint64_t rng = 42;
  if (sample_n > n) sample_n = n;
  float* sample = (float*)malloc(sizeof(float) * (sample_n ? sample_n : 1) * SG_PDIM);
  for (uint64_t s = 0; s < sample_n; s++) prefix_f32(rerank, quant_scale, or_rng_below(&rng, n), sample + s * SG_PDIM);
  kmeans(sample, sample_n, k, iters, 7, has_balance, balance, cents);
  or_tier2_fit(sample, sample_n, sigma);
  free(sample);
  float signs[3 * SG_PDIM];
  or_rotation_signs(11, SG_PDIM, signs);
  float* cents_rot = (float*)malloc(sizeof(float) * k * SG_PDIM);
  memcpy(cents_rot, cents, sizeof(float) * k * SG_PDIM);
  for (uint32_t c = 0; c < k; c++) or_rotation_apply(signs, SG_PDIM, cents_rot + (uint64_t)c * SG_PDIM);
  uint64_t* cnt = (uint64_t*)calloc(k, sizeof(uint64_t));
  uint32_t* pc = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (n ? n : 1));
  uint8_t* pcode = (uint8_t*)malloc(2 * SG_CODE_BYTES * (n ? n : 1));
  float* pfac = (float*)malloc(sizeof(float) * 4 * (n ? n : 1));
  float* sc = (float*)malloc(sizeof(float) * k);
  uint32_t* cid = (uint32_t*)malloc(sizeof(uint32_t) * k);
  for (uint32_t j = 0; j < k; j++) cid[j] = j;
  for (uint64_t i = 0; i < n; i++) {
    float x[SG_PDIM], xr[SG_PDIM];
    prefix_f32(rerank, quant_scale, i, x);
    t2_norm[i] = or_tier2_encode(sigma, x, t2_codes + i * SG_TIER2_BYTES);
    uint32_t* pair = pc + 2 * i;
    if (!has_soar) {
      pair[0] = assign1(x, cents, k);
      pair[1] = SG_PAD;
    } else {
      uint32_t cand[16] = {0};
      float top[16];
      or_gemm_abt(x, cents, 1, k, SG_PDIM, sc);
      or_topk(sc, cid, k, 16, top, cand);
      pair[0] = cand[0];
      pair[1] = soar_secondary(x, cents, cand, 16, lambda);
    }
    memcpy(xr, x, sizeof xr);
    or_rotation_apply(signs, SG_PDIM, xr);
    for (int h = 0; h < 2; h++) {
      uint8_t* code = pcode + (2 * i + h) * SG_CODE_BYTES;
      float* f = pfac + 4 * i + 2 * h;
      memset(code, 0, SG_CODE_BYTES);
      f[0] = f[1] = 0.0f;
      if (pair[h] == SG_PAD) continue;
      or_rabitq_encode(xr, cents_rot + (uint64_t)pair[h] * SG_PDIM, SG_PDIM, code, f);
      cnt[pair[h]]++;
    }
  }
  uint64_t nb = 0;
  block_off[0] = 0;
  for (uint32_t c = 0; c < k; c++) {
    nb += (cnt[c] + SG_BLOCK - 1) / SG_BLOCK;
    block_off[c + 1] = nb;
  }
  if (nb <= max_blocks) {
    /* cluster-major write (src/ivf.rs:356-385): members in row order, 32 per block */
    uint64_t* fill = (uint64_t*)calloc(k, sizeof(uint64_t));
    for (uint64_t s = 0; s < nb * SG_BLOCK; s++) {
      ids[s] = SG_PAD;
      factors[2 * s] = factors[2 * s + 1] = 0.0f;
    }
    uint8_t* raw = (uint8_t*)calloc(nb * SG_BLOCK + 1, SG_CODE_BYTES);
    for (uint64_t i = 0; i < n; i++)
      for (int h = 0; h < 2; h++) {
        const uint32_t c = pc[2 * i + h];
        if (c == SG_PAD) continue;
        const uint64_t s = block_off[c] * SG_BLOCK + fill[c]++;
        ids[s] = (uint32_t)i;
        factors[2 * s] = pfac[4 * i + 2 * h];
        factors[2 * s + 1] = pfac[4 * i + 2 * h + 1];
        memcpy(raw + s * SG_CODE_BYTES, pcode + (2 * i + h) * SG_CODE_BYTES, SG_CODE_BYTES);
      }
    for (uint32_t c = 0; c < k; c++)
      for (uint64_t b = block_off[c]; b < block_off[c + 1]; b++) {
        const uint64_t s0 = b * SG_BLOCK, end = block_off[c] * SG_BLOCK + cnt[c];
        const uint64_t used = s0 + SG_BLOCK <= end ? SG_BLOCK : end - s0;
        or_pack_block(raw + s0 * SG_CODE_BYTES, (uint32_t)used, SG_GROUPS, blocks + b * SG_BLOCK_BYTES);
      }
    free(raw);
    free(fill);
  }
  free(cents_rot);
  free(cnt);
  free(pc);
  free(pcode);
  free(pfac);
  free(sc);
  free(cid);
  return nb;
}

/* Live::apply_insert's encoding of one inserted row (src/live.rs:274-350), as ivf::build encodes
 * a row: the int8 row (Int8Quantizer::encode), the prefix norm, the normalised prefix of the int8
 * row, its primary cluster and (with SOAR) its secondary among the 16 nearest (assign_top,
 * soar_secondary, src/ivf.rs:138-186), the RaBitQ residual code and factors of the rotated
 * prefix against each rotated centroid (rabitq::encode), and the 2-bit tier code and norm.
 * pair[1] = PAD without SOAR; its code and factors are then zero. */
static float dot16(const float* a, const float* b, uint32_t n) { return or_dot_f32(a, b, n); }

static uint32_t soar_secondary(const float* x, const float* cents, const uint32_t* cand, uint32_t nc,
                               float lambda) {
  const float* c1 = cents + (uint64_t)cand[0] * SG_PDIM;
  float x_c1 = dot16(x, c1, SG_PDIM);
  float r2 = fmaxf(2.0f - 2.0f * x_c1, 1e-12f);
  float r_x = 1.0f - x_c1;
  float best = FLT_MAX;
  uint32_t best_c = cand[1];
  for (uint32_t i = 1; i < nc; i++) {
    const float* cv = cents + (uint64_t)cand[i] * SG_PDIM;
    float x_c = dot16(x, cv, SG_PDIM);
    float r_c = x_c - dot16(c1, cv, SG_PDIM);
    float along = r_x - r_c;
    float loss = (2.0f - 2.0f * x_c) + lambda * along * along / r2;
    if (loss < best) {
      best = loss;
      best_c = cand[i];
    }
  }
  return best_c;
}

void or_live_encode(const sg_ivf_arrays* ix, const float* cents_rot, int soar, float lambda, const float* v,
                    int8_t* row, float* norm256, uint32_t* pair, uint8_t* codes, float* factors, uint8_t* t2,
                    float* t2_norm) {
  or_int8_encode(ix->quant_scale, v, row);
  float nn = NEG0;
  for (int i = 0; i < SG_PDIM; i++) nn += v[i] * v[i];
  *norm256 = sqrtf(nn);
  float x[SG_PDIM];
  for (int i = 0; i < SG_PDIM; i++) x[i] = (float)row[i] / ix->quant_scale[i];
  or_normalize(x, SG_PDIM);
  const uint32_t K = ix->k;
  float* sc = (float*)malloc(sizeof(float) * K);
  or_gemm_abt(x, ix->centroids, 1, K, SG_PDIM, sc);
  if (!soar) {
    uint32_t bj = 0;
    float bv = -FLT_MAX;
    for (uint32_t j = 0; j < K; j++)
      if (sc[j] > bv) {
        bv = sc[j];
        bj = j;
      }
    pair[0] = bj;
    pair[1] = SG_PAD;
  } else {
    uint32_t cand[16] = {0};
    uint32_t* ids = (uint32_t*)malloc(sizeof(uint32_t) * K);
    for (uint32_t j = 0; j < K; j++) ids[j] = j;
    float top_s[16];
    uint32_t m = or_topk(sc, ids, K, 16, top_s, cand);
    free(ids);
    (void)m;  /* fewer than 16 clusters leave the rest of cand at cluster 0, as assign_top does */
    pair[0] = cand[0];
    pair[1] = soar_secondary(x, ix->centroids, cand, 16, lambda);
  }
  free(sc);
  float xr[SG_PDIM];
  memcpy(xr, x, sizeof xr);
  or_rotation_apply(ix->rotation, SG_PDIM, xr);
  for (int h = 0; h < 2; h++) {
    if (pair[h] == SG_PAD) {
      memset(codes + h * SG_CODE_BYTES, 0, SG_CODE_BYTES);
      factors[2 * h] = factors[2 * h + 1] = 0.0f;
      continue;
    }
    or_rabitq_encode(xr, cents_rot + (uint64_t)pair[h] * SG_PDIM, SG_PDIM, codes + h * SG_CODE_BYTES,
                     factors + 2 * h);
  }
  if (ix->tier2_sigma) *t2_norm = or_tier2_encode(ix->tier2_sigma, x, t2);
}

/* The flat Hamming baseline of the search binary (src/bin/search.rs:251-269): the query's sign code
 * against every corpus code (hamming, src/lut.rs:156-165), TopK(cand) of PDIM - distance keyed by
 * row, then the rows' float-weight int8 dot (quant::dot_i8 with Int8Quantizer::query_weights)
 * into TopK(k), best first. */
uint32_t or_flat_hamming(const uint8_t* codes, uint64_t n, const int8_t* rerank, const float* quant_scale,
                         const float* q768, const float* q256, uint32_t cand, uint32_t k, float* out_scores,
                         uint32_t* out_ids) {
  uint8_t qc[SG_CODE_BYTES];
  or_sign_code(q256, qc);
  topk top;
  topk_init(&top, cand);
  for (uint64_t i = 0; i < n; i++) {
    float s = (float)(uint16_t)(SG_PDIM - or_hamming(qc, codes + i * SG_CODE_BYTES, SG_CODE_BYTES));
    if (topk_admits(&top, s, (uint32_t)i)) topk_push(&top, s, (uint32_t)i);
  }
  uint32_t m = cand ? topk_sorted(&top) : 0;
  float w[SG_DIM];
  or_int8_query_weights(quant_scale, q768, SG_DIM, w);
  topk out;
  topk_init(&out, k);
  for (uint32_t j = 0; j < m; j++) {
    uint32_t id = top.items[j].id;
    float s = or_dot_i8(w, rerank + (uint64_t)id * SG_DIM, SG_DIM);
    if (topk_admits(&out, s, id)) topk_push(&out, s, id);
  }
  uint32_t r = k ? topk_sorted(&out) : 0;
  for (uint32_t j = 0; j < r; j++) {
    out_scores[j] = out.items[j].s;
    out_ids[j] = out.items[j].id;
  }
  topk_free(&top);
  topk_free(&out);
  return r;
}

uint64_t or_search_batch(const sg_ivf_arrays* ix, uint32_t nq, const float* q768,
                         const float* q256, const sg_params* p, const uint64_t* allow,
                         uint64_t allow_words, int threads, float* out_scores,
                         uint32_t* out_ids, uint32_t* out_counts, uint8_t* out_tied) {
  uint64_t scanned = 0;
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads) reduction(+ : scanned)
  for (int64_t i = 0; i < (int64_t)nq; i++) {
    sg_timing t;
    memset(&t, 0, sizeof t);
    g_tied = 0;
    out_counts[i] =
        or_search(ix, q768 + (uint64_t)i * SG_DIM, q256 + (uint64_t)i * SG_PDIM, p, allow,
                  allow_words, out_scores + (uint64_t)i * p->k, out_ids + (uint64_t)i * p->k, &t);
    if (out_tied) out_tied[i] = (uint8_t)g_tied;
    scanned += t.scanned;
  }
  return scanned;
}

int or_last_tied(void) { return g_tied; }
void or_clear_tied(void) { g_tied = 0; }

/* ---- filter.rs: src/filter.rs:27-110 ----------------------------------------------------- */
void or_filter_per_cluster(const sg_ivf_arrays* ix, const uint64_t* allow, uint64_t words,
                           uint32_t* per_cluster) {
  for (uint32_t c = 0; c < ix->k; c++) {
    uint32_t cnt = 0;
    for (uint64_t s = ix->block_off[c] * SG_BLOCK; s < ix->block_off[c + 1] * SG_BLOCK; s++) {
      uint32_t id = ix->ids[s];
      if (id != SG_PAD && allowed(allow, words, id)) cnt++;
    }
    per_cluster[c] = cnt;
  }
}

int or_plan_resolve(int plan, uint64_t allowed_rows, uint64_t n) {
  if (plan != 3) return plan;
  if (allowed_rows <= 250000) return 2;
  if ((double)allowed_rows >= 0.3 * (double)n) return 0;
  return 1;
}

uint32_t or_filter_search(const sg_ivf_arrays* ix, const uint64_t* allow, uint64_t words,
                          const uint32_t* rows, uint64_t nrows, const uint32_t* per_cluster,
                          int plan, uint64_t expand_target, const float* q768,
                          const float* q256, const sg_params* p, float* out_scores,
                          uint32_t* out_ids) {
  int resolved = or_plan_resolve(plan, nrows, ix->n);
  if (plan == 3 && resolved == 1) expand_target = 200000;
  if (resolved == 0) return or_search(ix, q768, q256, p, allow, words, out_scores, out_ids, 0);
  if (resolved == 2) {
    int8_t wq[SG_DIM];
    float inv = query_weights_i8(ix->quant_scale, q768, SG_DIM, wq);
    topk top;
    topk_init(&top, p->k);
    for (uint64_t i = 0; i < nrows; i++)
      topk_push(&top, (float)or_dot_i8i8(wq, ix->rerank + (uint64_t)rows[i] * SG_DIM, SG_DIM) * inv,
                rows[i]);
    uint32_t k = p->k ? topk_sorted(&top) : 0;
    for (uint32_t i = 0; i < k; i++) {
      out_scores[i] = top.items[i].s;
      out_ids[i] = top.items[i].id;
    }
    topk_free(&top);
    return k;
  }
  /* Expand: route over every cluster, keep clusters with allowed slots until the target is
   * covered (the cluster that crosses it is kept). */
  sg_params all = *p;
  all.nprobe = ix->k;
  all.has_margin = 0;
  all.has_budget = 0;
  float* ps = (float*)malloc(sizeof(float) * ix->k);
  uint32_t* pc = (uint32_t*)malloc(sizeof(uint32_t) * ix->k);
  uint32_t m = or_route(ix, q256, &all, ps, pc);
  uint32_t w = 0;
  uint64_t covered = 0;
  for (uint32_t i = 0; i < m; i++) {
    uint32_t c = pc[i];
    if (per_cluster[c] == 0) continue;
    if (covered >= expand_target) break;
    covered += per_cluster[c];
    ps[w] = ps[i];
    pc[w] = c;
    w++;
  }
  uint32_t cap = p->cand ? p->cand : 1;
  float* est = (float*)malloc(sizeof(float) * cap);
  uint32_t* ids = (uint32_t*)malloc(sizeof(uint32_t) * cap);
  float* err = (float*)malloc(sizeof(float) * cap);
  uint32_t n = p->cand ? or_candidates(ix, q256, ps, pc, w, p, allow, words, est, ids, err, 0) : 0;
  uint32_t k = or_rerank(ix, q768, q256, est, ids, err, n, p, out_scores, out_ids, 0);
  free(ps);
  free(pc);
  free(est);
  free(ids);
  free(err);
  return k;
}

/* ---- eval::recall_at: src/eval.rs:7-10 --------------------------------------------------- */
double or_recall_at(uint32_t k, const uint32_t* got, uint32_t ngot, const uint32_t* truth,
                    uint32_t ntruth) {
  uint32_t tk = ntruth < k ? ntruth : k;
  /* distinct truth ids among the first k */
  uint32_t distinct = 0;
  for (uint32_t i = 0; i < tk; i++) {
    int dup = 0;
    for (uint32_t j = 0; j < i; j++)
      if (truth[j] == truth[i]) dup = 1;
    if (!dup) distinct++;
  }
  uint32_t gk = ngot < k ? ngot : k, hit = 0;
  for (uint32_t i = 0; i < gk; i++)
    for (uint32_t j = 0; j < tk; j++)
      if (got[i] == truth[j]) {
        hit++;
        break;
      }
  uint32_t den = k < distinct ? k : distinct;
  return (double)hit / (double)(den > 0 ? den : 1);
}

/* ---- bigann.rs: L2 search over int8 rows ------------------------------------------------- */
#define BG_D SG_BG_DIM
#define BG_PD SG_BG_PDIM
#define BG_CODE SG_BG_CODE
#define BG_BB SG_BG_BLOCK_BYTES

uint32_t or_bg_extra(uint32_t bits) { return bits > 1 ? (bits - 1) * BG_CODE + 4 : 0; }

/* refine_encode: src/bigann.rs:65-108 (extended-RaBitQ step search over 24 deltas). */
static inline uint32_t bg_level(float v, float delta, float h, uint32_t top) {
  float x = floorf(v / delta + h + 0.5f);
  float hi = (float)(2 * top - 1);
  if (x < 0.0f) x = 0.0f;
  if (x > hi) x = hi;
  uint32_t u = (uint32_t)x;
  return v > 0.0f ? (u | top) : (u & (top - 1));
}

float or_bg_refine_encode(const float* r, uint32_t bits, uint8_t* planes) {
  memset(planes, 0, (SG_BG_MAX_BITS - 1) * BG_CODE);
  const uint32_t top = 1u << (bits - 1);
  const float h = (float)(2 * top - 1) / 2.0f;
  float amax = 0.0f;
  for (int i = 0; i < BG_PD; i++) amax = fmaxf(amax, fabsf(r[i]));
  if (amax < 1e-12f) return 0.0f;
  float best = -FLT_MAX, best_delta = amax / h;
  for (int s = 0; s < 24; s++) {
    const float delta = amax / h * (0.3f + 0.035f * (float)s);
    float dot = 0.0f, n2 = 0.0f;
    for (int i = 0; i < BG_PD; i++) {
      const float w = (float)bg_level(r[i], delta, h, top) - h;
      dot += r[i] * w;
      n2 += w * w;
    }
    const float cosv = dot / sqrtf(n2);
    if (cosv > best) {
      best = cosv;
      best_delta = delta;
    }
  }
  float rr = 0.0f, dot = 0.0f;
  for (int i = 0; i < BG_PD; i++) {
    const uint32_t u = bg_level(r[i], best_delta, h, top);
    for (uint32_t p = 0; p + 1 < bits; p++)
      planes[p * BG_CODE + (i >> 3)] |= (uint8_t)(((u >> p) & 1u) << (i & 7));
    rr += r[i] * r[i];
    dot += r[i] * ((float)u - h);
  }
  return dot > 0.0f ? rr / dot : 0.0f;
}

/* Refiner::new / plane / estimate: src/bigann.rs:568-602. tab is [16][256]. */
void or_bg_refiner_new(const float* qr, uint32_t bits, float* tab, float* off) {
  for (int k = 0; k < BG_CODE; k++) {
    float* t = tab + k * 256;
    t[0] = 0.0f;
    for (int v = 1; v < 256; v++) t[v] = t[v & (v - 1)] + qr[8 * k + __builtin_ctz((unsigned)v)];
  }
  const float h = (float)((1u << bits) - 1) / 2.0f;
  float sum = NEG0;
  for (int i = 0; i < BG_PD; i++) sum += qr[i];
  *off = h * sum;
}

static float bg_plane(const float* tab, const uint8_t* p) {
  float s = NEG0;
  for (int k = 0; k < BG_CODE; k++) s += tab[k * 256 + p[k]];
  return s;
}

float or_bg_refiner_estimate(const float* tab, float off, uint32_t bits, const uint8_t* sign,
                             const uint8_t* planes, float f) {
  float u = (float)(1u << (bits - 1)) * bg_plane(tab, sign);
  for (uint32_t p = 0; p + 1 < bits; p++) u += (float)(1u << p) * bg_plane(tab, planes + p * BG_CODE);
  return f * (u - off);
}

/* The rotated, padded query: pad_rotate(rot, q as f32) (src/bigann.rs:243-248). */
static void bg_rotated_query(const sg_bigann_arrays* ix, const int8_t* q, float* qr) {
  for (int i = 0; i < BG_PD; i++) qr[i] = i < BG_D ? (float)q[i] : 0.0f;
  or_rotation_apply(ix->rotation, BG_PD, qr);
}

/* Index::route: src/bigann.rs:660-678. Returns the probe count; dots gets <q, c> of every leaf. */
uint32_t or_bg_route(const sg_bigann_arrays* ix, const int8_t* q, const sg_bigann_params* p,
                     uint32_t* out_probe, float* out_probe_scores, float* dots) {
  const uint32_t K = ix->k;
  float qf[BG_D];
  for (int i = 0; i < BG_D; i++) qf[i] = (float)q[i];
  or_gemm_abt(qf, ix->leaves, 1, K, BG_D, dots);
  uint32_t np = p->nprobe < K ? p->nprobe : K;
  if (np == 0) return 0;
  topk t;
  topk_init(&t, np);
  for (uint32_t c = 0; c < K; c++) {
    float n = NEG0;
    for (int i = 0; i < BG_D; i++) n += ix->leaves[(uint64_t)c * BG_D + i] * ix->leaves[(uint64_t)c * BG_D + i];
    topk_push(&t, 2.0f * dots[c] - n, c);
  }
  uint32_t m = topk_sorted(&t);
  uint32_t keep = m;
  if (p->margin > 0.0f && m > 0) {
    float qq = NEG0;
    for (int i = 0; i < BG_D; i++) qq += qf[i] * qf[i];
    const float lim = (qq - t.items[0].s) * (1.0f + p->margin);
    keep = 0;
    for (uint32_t i = 0; i < m; i++)
      if (qq - t.items[i].s <= lim) t.items[keep++] = t.items[i];
  }
  for (uint32_t i = 0; i < keep; i++) {
    out_probe[i] = t.items[i].id;
    if (out_probe_scores) out_probe_scores[i] = t.items[i].s;
  }
  topk_free(&t);
  return keep;
}

/* Index::candidates: src/bigann.rs:683-732, the leaves scanned in probe order (every record
 * resident). Out: (id, estimate, |x|^2) best first. */
uint32_t or_bg_candidates(const sg_bigann_arrays* ix, const int8_t* q, const uint32_t* probe,
                          uint32_t nprobe, const float* dots, const sg_bigann_params* p,
                          uint32_t* out_ids, float* out_est, float* out_nx, uint64_t* scanned) {
  float qp[BG_PD], qr[BG_PD];
  for (int i = 0; i < BG_PD; i++) qp[i] = i < BG_D ? (float)q[i] : 0.0f;
  uint8_t tables[SG_BG_GROUPS * 16];
  float scale, bias, a, b;
  or_query_new(ix->rotation, BG_PD, qp, tables, &scale, &bias, &a, &b);
  const uint32_t bits = ix->bits;
  const int refine = bits > 1 && p->refine > 0;
  float* rtab = NULL;
  float roff = 0.0f;
  if (refine) {
    bg_rotated_query(ix, q, qr);
    rtab = (float*)malloc(sizeof(float) * BG_CODE * 256);
    or_bg_refiner_new(qr, bits, rtab, &roff);
  }
  const uint32_t extra = or_bg_extra(bits);
  /* info: (id, estimate, |x|^2) of every admitted slot, indexed by admission order */
  uint64_t info_cap = 1024, ninfo = 0;
  uint32_t* info_id = (uint32_t*)malloc(sizeof(uint32_t) * info_cap);
  float* info_est = (float*)malloc(sizeof(float) * info_cap);
  float* info_nx = (float*)malloc(sizeof(float) * info_cap);
  const uint32_t kc = refine ? (p->refine > p->cand ? p->refine : p->cand) : p->cand;
  topk cand, best;
  topk_init(&cand, kc);
  topk_init(&best, p->cand);
  uint64_t sc_total = 0;
  uint8_t sign[BG_CODE];
  for (uint32_t i = 0; i < nprobe; i++) {
    const uint32_t c = probe[i];
    const float cent = dots[c];
    const uint64_t b0 = ix->block_off[c], b1 = ix->block_off[c + 1];
    for (uint64_t blk = b0; blk < b1; blk++) {
      uint16_t scores[SG_BLOCK];
      or_scan(tables, SG_BG_GROUPS, ix->blocks + blk * BG_BB, 1, scores);
      for (uint32_t j = 0; j < SG_BLOCK; j++) {
        const uint64_t s = blk * SG_BLOCK + j;
        const uint32_t id = ix->ids[s];
        if (id == SG_PAD) continue;
        const float mul = ix->factors[2 * s], nx = ix->factors[2 * s + 1];
        const float est = 2.0f * (cent + mul * (a * (float)scores[j] + b)) - nx;
        if (!topk_admits(&cand, est, (uint32_t)ninfo)) continue;
        topk_push(&cand, est, (uint32_t)ninfo);
        float e = est;
        if (refine) {
          or_unpack_slot(ix->blocks + blk * BG_BB, SG_BG_GROUPS, j, sign);
          const uint8_t* ex = ix->ext + s * extra;
          float fs;
          memcpy(&fs, ex + extra - 4, 4);
          e = 2.0f * (cent + or_bg_refiner_estimate(rtab, roff, bits, sign, ex, fs)) - nx;
          topk_push(&best, e, (uint32_t)ninfo);
        }
        if (ninfo == info_cap) {
          info_cap *= 2;
          info_id = (uint32_t*)realloc(info_id, sizeof(uint32_t) * info_cap);
          info_est = (float*)realloc(info_est, sizeof(float) * info_cap);
          info_nx = (float*)realloc(info_nx, sizeof(float) * info_cap);
        }
        info_id[ninfo] = id;
        info_est[ninfo] = e;
        info_nx[ninfo] = nx;
        ninfo++;
      }
    }
    sc_total += (b1 - b0) * SG_BLOCK;
  }
  topk* top = refine ? &best : &cand;
  uint32_t m = p->cand ? topk_sorted(top) : 0;
  for (uint32_t i = 0; i < m; i++) {
    const uint32_t x = top->items[i].id;
    out_ids[i] = info_id[x];
    out_est[i] = info_est[x];
    out_nx[i] = info_nx[x];
  }
  if (scanned) *scanned = sc_total;
  topk_free(&cand);
  topk_free(&best);
  free(info_id);
  free(info_est);
  free(info_nx);
  free(rtab);
  return m;
}

/* Index::rerank: src/bigann.rs:735-747: 2 <q, x> - |x|^2 from the base rows, TopK(k). */
uint32_t or_bg_rerank(const sg_bigann_arrays* ix, const int8_t* q, const uint32_t* ids,
                      const float* nx, uint32_t n, const sg_bigann_params* p, float* out_scores,
                      uint32_t* out_ids) {
  if (p->k == 0) return 0;
  topk t;
  topk_init(&t, p->k);
  for (uint32_t i = 0; i < n; i++) {
    const int32_t dot = or_dot_i8i8(q, ix->base + (uint64_t)ids[i] * BG_D, BG_D);
    topk_push(&t, 2.0f * (float)dot - nx[i], ids[i]);
  }
  uint32_t m = topk_sorted(&t);
  for (uint32_t i = 0; i < m; i++) {
    out_scores[i] = t.items[i].s;
    out_ids[i] = t.items[i].id;
  }
  topk_free(&t);
  return m;
}

/* Index::search: src/bigann.rs:653-657. */
uint32_t or_bg_search(const sg_bigann_arrays* ix, const int8_t* q, const sg_bigann_params* p,
                      float* out_scores, uint32_t* out_ids, sg_bigann_timing* t) {
  uint32_t* probe = (uint32_t*)malloc(sizeof(uint32_t) * (ix->k ? ix->k : 1));
  float* dots = (float*)malloc(sizeof(float) * (ix->k ? ix->k : 1));
  const uint32_t np = or_bg_route(ix, q, p, probe, NULL, dots);
  const uint32_t cap = p->cand ? p->cand : 1;
  uint32_t* cid = (uint32_t*)malloc(sizeof(uint32_t) * cap);
  float* cest = (float*)malloc(sizeof(float) * cap);
  float* cnx = (float*)malloc(sizeof(float) * cap);
  uint64_t scanned = 0;
  const uint32_t n = or_bg_candidates(ix, q, probe, np, dots, p, cid, cest, cnx, &scanned);
  const uint32_t k = or_bg_rerank(ix, q, cid, cnx, n, p, out_scores, out_ids);
  if (t) {
    t->probes += np;
    t->scanned += scanned;
  }
  free(probe);
  free(dots);
  free(cid);
  free(cest);
  free(cnx);
  return k;
}

uint64_t or_bg_search_batch(const sg_bigann_arrays* ix, uint32_t nq, const int8_t* q,
                            const sg_bigann_params* p, int threads, float* out_scores,
                            uint32_t* out_ids, uint32_t* out_counts) {
  uint64_t scanned = 0;
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads) reduction(+ : scanned)
  for (int64_t i = 0; i < (int64_t)nq; i++) {
    sg_bigann_timing t;
    memset(&t, 0, sizeof t);
    out_counts[i] = or_bg_search(ix, q + (uint64_t)i * BG_D, p, out_scores + (uint64_t)i * p->k,
                                 out_ids + (uint64_t)i * p->k, &t);
    scanned += t.scanned;
  }
  return scanned;
}
