// Test infrastructure, force-included (g++ -include) when the reference sources are built
// as an oracle.  Random.cpp:31 seeds every per-thread mt19937 with time(0) + cnt^2*23 +
// 3571*rank, so two runs never share a stream.  This header pins the value time(0) returns
// to $MPSQMC_REF_SEED (default 20131015) without editing the reference: <time.h> is
// included first, then a function-like macro replaces later calls of time(...).
// It also provides the declarations the reference takes for granted: sleep()
// (Random.cpp:63, <unistd.h>), sprintf() (MPSQMC2.cpp:452, <cstdio>) and
// std::cout (Random.cpp:84, <iostream>).
#ifndef MPSQMC_COMPAT_PIN_SEED_H
#define MPSQMC_COMPAT_PIN_SEED_H

#include <time.h>
#include <ctime>
#include <cstdio>
#include <cstdlib>
#include <unistd.h>
#include <iostream>

static inline time_t mpsqmc_pinned_time_(time_t *out) {
  const char *s = getenv("MPSQMC_REF_SEED");
  time_t v = s ? (time_t)strtoll(s, 0, 10) : (time_t)20131015;
  if (out) *out = v;
  return v;
}
#define time(x) mpsqmc_pinned_time_(x)

#endif
