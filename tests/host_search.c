/* host_search.c — a C host of the drop-in boundary: opens an index from the reference's files
 * (sg_open_ivf), searches a batch from a binary query file through sg_search and through
 * per-thread search contexts (sg_context_open + sg_search_ctx on two threads), and writes the
 * results. The test that builds it (tests/test_c_host.py) compares them with the Python API.
 *
 *   host_search <ingest_dir> <index_dir> <queries.f32 [nq x 768]> <nq> <out.bin>
 *
 * out.bin: for each of the three runs, nq counts (u32), nq*K scores (f32), nq*K ids (u32). */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sieve_gpu.h"

#define K 10

struct job {
  sg_context* ctx;
  const float* q;
  uint32_t nq;
  const sg_params* p;
  float* sc;
  uint32_t* ids;
  uint32_t* cnt;
  int rc;
};

static void* run_ctx(void* arg) {
  struct job* j = (struct job*)arg;
  j->rc = sg_search_ctx(j->ctx, j->nq, j->q, NULL, j->p, NULL, 0, j->sc, j->ids, j->cnt, NULL);
  return NULL;
}

static int fail(const char* what, int rc) {
  fprintf(stderr, "%s: status %d: %s\n", what, rc, sg_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s ingest_dir index_dir queries.f32 nq out.bin\n", argv[0]);
    return 2;
  }
  const uint32_t nq = (uint32_t)strtoul(argv[4], NULL, 10);
  float* q = (float*)malloc((size_t)nq * SG_DIM * sizeof(float));
  FILE* f = fopen(argv[3], "rb");
  if (!f || fread(q, sizeof(float), (size_t)nq * SG_DIM, f) != (size_t)nq * SG_DIM) return 2;
  fclose(f);
  sg_index* ix = NULL;
  int rc = sg_open_ivf(argv[1], argv[2], 0, &ix);
  if (rc) return fail("sg_open_ivf", rc);
  sg_params p;
  memset(&p, 0, sizeof p);
  p.nprobe = 16;
  p.cand = 500;
  p.rerank_kind = SG_RERANK_FULL;
  p.k = K;
  float* sc = (float*)calloc((size_t)3 * nq * K, sizeof(float));
  uint32_t* ids = (uint32_t*)calloc((size_t)3 * nq * K, sizeof(uint32_t));
  uint32_t* cnt = (uint32_t*)calloc((size_t)3 * nq, sizeof(uint32_t));
  /* run 0: the index's default context */
  rc = sg_search(ix, nq, q, NULL, &p, NULL, 0, sc, ids, cnt, NULL);
  if (rc) return fail("sg_search", rc);
  /* runs 1 and 2: two threads, each with its own context, each searching half of the batch */
  for (int run = 1; run <= 2; run++) {
    struct job jobs[2];
    pthread_t th[2];
    const uint32_t half = nq / 2;
    for (int t = 0; t < 2; t++) {
      const uint32_t q0 = t ? half : 0, n = t ? nq - half : half;
      jobs[t].q = q + (size_t)q0 * SG_DIM;
      jobs[t].nq = n;
      jobs[t].p = &p;
      jobs[t].sc = sc + (size_t)run * nq * K + (size_t)q0 * K;
      jobs[t].ids = ids + (size_t)run * nq * K + (size_t)q0 * K;
      jobs[t].cnt = cnt + (size_t)run * nq + q0;
      if ((rc = sg_context_open(ix, &jobs[t].ctx))) return fail("sg_context_open", rc);
    }
    for (int t = 0; t < 2; t++) pthread_create(&th[t], NULL, run_ctx, &jobs[t]);
    for (int t = 0; t < 2; t++) pthread_join(th[t], NULL);
    for (int t = 0; t < 2; t++) {
      if (jobs[t].rc) return fail("sg_search_ctx", jobs[t].rc);
      sg_context_close(jobs[t].ctx);
    }
  }
  FILE* o = fopen(argv[5], "wb");
  if (!o) return 2;
  for (int run = 0; run < 3; run++) {
    fwrite(cnt + (size_t)run * nq, sizeof(uint32_t), nq, o);
    fwrite(sc + (size_t)run * nq * K, sizeof(float), (size_t)nq * K, o);
    fwrite(ids + (size_t)run * nq * K, sizeof(uint32_t), (size_t)nq * K, o);
  }
  fclose(o);
  sg_close(ix);
  free(q);
  free(sc);
  free(ids);
  free(cnt);
  return 0;
}
