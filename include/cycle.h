/* cycle.h -- the tick counter header the reference's drivers include before mdcore.h
 * (examples/argon/argon.c: `ticks`, getticks(), elapsed()), so that such a driver compiles
 * unchanged against libmdcore_b200.  ticks counts the processor's time-stamp counter. */
#ifndef MDCORE_CYCLE_H_B200
#define MDCORE_CYCLE_H_B200
#include <x86intrin.h>
typedef unsigned long long ticks;
static inline ticks getticks(void) { return (ticks)__rdtsc(); }
static inline double elapsed(ticks t1, ticks t0) { return (double)t1 - (double)t0; }
#endif
