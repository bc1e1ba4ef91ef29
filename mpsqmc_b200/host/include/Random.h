// Random: the walk's random stream.  Interface of the reference's include/Random.h:9-27
// (rand() returns uniforms on [0,1) from a 32-bit Mersenne Twister, one engine output per
// draw).  The reference seeds one engine per OpenMP thread with time(0) + cnt^2*23 +
// 3571*rank; this build uses one engine (the walk runs on the GPU), seeded with time(0) or
// $MPSQMC_SEED, and counts its draws so the device can continue the same stream.
#ifndef RANDOM_H
#define RANDOM_H

#include <stdint.h>
#include <random>

class Random {
 public:
  Random();
  ~Random();
  double rand();
  void test();
  // stream position, for handing the stream to the device engine and taking it back
  uint32_t gSeed() const;
  unsigned long long gDraws() const;
  void discard(unsigned long long n);

 private:
  std::mt19937 gen;
  uint32_t seed;
  unsigned long long draws;
};

#endif
