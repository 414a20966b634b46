/*
 * common.c — oracle threading helper (TEST INFRASTRUCTURE ONLY).
 *
 * The reference spreads independent work units over scoped threads and its
 * results do not depend on the thread count (src/arnr.rs:551-590,
 * src/loop_filter.rs:2097-2127). vo_parallel_for does the same: an atomic
 * work counter over `n` units, so outputs are identical for any `threads`.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>

#include "vp8a_oracle.h"

typedef struct {
  atomic_uint next;
  uint32_t n;
  vo_task_fn fn;
  void* arg;
} pf_state;

static void* pf_worker(void* p) {
  pf_state* s = (pf_state*)p;
  for (;;) {
    uint32_t i = atomic_fetch_add(&s->next, 1u);
    if (i >= s->n) break;
    s->fn(s->arg, i);
  }
  return NULL;
}

void vo_parallel_for(uint32_t n, uint32_t threads, vo_task_fn fn, void* arg) {
  pf_state s;
  atomic_init(&s.next, 0u);
  s.n = n;
  s.fn = fn;
  s.arg = arg;
  if (threads <= 1 || n <= 1) {
    pf_worker(&s);
    return;
  }
  if (threads > n) threads = n;
  pthread_t* tids = (pthread_t*)malloc(sizeof(pthread_t) * (threads - 1));
  uint32_t started = 0;
  for (uint32_t t = 0; t + 1 < threads; t++) {
    if (pthread_create(&tids[t], NULL, pf_worker, &s) == 0) started++;
    else break;
  }
  pf_worker(&s);
  for (uint32_t t = 0; t < started; t++) pthread_join(tids[t], NULL);
  free(tids);
}

/* sizeof of the shared ABI records, as this C compiler lays them out
 * (lets the tests pin the Python mirrors of include/vp8a.h). */
size_t vo_type_size(int which) {
  switch (which) {
    case 0: return sizeof(vp8a_mv);
    case 1: return sizeof(vp8a_search_result);
    case 2: return sizeof(vp8a_luma_ref);
    case 3: return sizeof(vp8a_i420);
    case 4: return sizeof(vp8a_planes);
    case 5: return sizeof(vp8a_mv_contexts);
    case 6: return sizeof(vp8a_mb_decision);
    case 7: return sizeof(vp8a_ref_search);
    case 8: return sizeof(vp8a_mb_lf_info);
    case 9: return sizeof(vp8a_filter_config);
    case 10: return sizeof(vp8a_source);
    case 11: return sizeof(vp8a_mb_info);
    case 12: return sizeof(vp8a_rd_inter);
    case 13: return sizeof(vp8a_quant_indices);
    case 14: return sizeof(vp8a_analysis_job);
    case 15: return sizeof(vp8a_arnr_job);
    case 16: return sizeof(vp8a_recon_job);
    case 17: return sizeof(vp8a_sweep_job);
    case 18: return sizeof(vp8a_frame_header);
    case 19: return sizeof(vp8a_arnr_planes_job);
    default: return 0;
  }
}
