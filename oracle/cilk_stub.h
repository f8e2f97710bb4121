/* Single-worker stand-ins for the four Cilk runtime calls that the reference's non-OpenMP
 * build references (lib/utilities.h:38-49, lib/counting_sort.h:110,185, lib/histogram.h:65).
 * With them the reference compiles serially, which is the only build that includes its
 * HIST/AHIST aggregators (the OpenMP build exits at butterfly_count.h:574-576).
 * Test infrastructure only: used by oracle/Makefile for oracle/_ref/ref_harness_ser. */
#ifndef PB_CILK_STUB_H
#define PB_CILK_STUB_H
static inline int __cilkrts_get_nworkers(void) { return 1; }
static inline int __cilkrts_get_worker_number(void) { return 0; }
static inline void __cilkrts_end_cilk(void) {}
static inline int __cilkrts_set_param(const char* a, const char* b) { (void)a; (void)b; return 0; }
#endif
