// Test infrastructure: stand-in for Boost.Random's mt19937, used only to build the
// reference sources as an oracle. Nothing in the product links this file.
//
// Boost's mt19937 is the standard 32-bit Mersenne Twister (Matsumoto & Nishimura 1998:
// n=624, m=397, matrix 0x9908b0df, tempering b=0x9d2c5680 c=0xefc60000, seeded by the
// standard init_genrand recurrence), which is exactly std::mt19937.  The wrapper counts
// the 32-bit outputs drawn so the oracle harness can report how many uniforms the
// reference consumed during setup (Random.cpp:28-36 seeds, MPStensor.cpp:77 draws).
#ifndef MPSQMC_COMPAT_BOOST_MT19937_HPP
#define MPSQMC_COMPAT_BOOST_MT19937_HPP

#include <random>
#include <stdint.h>

namespace mpsqmc_compat {
inline unsigned long long &mt_draw_count() {
  static unsigned long long count = 0;
  return count;
}
inline uint32_t &mt_last_seed() {
  static uint32_t seed = 5489u;
  return seed;
}
}  // namespace mpsqmc_compat

namespace boost {
namespace random {

class mt19937 {
 public:
  typedef uint32_t result_type;
  mt19937() : engine_() {}
  explicit mt19937(result_type value) : engine_(value) {}
  void seed(result_type value) {
    mpsqmc_compat::mt_last_seed() = value;
    engine_.seed(value);
  }
  result_type operator()() {
    ++mpsqmc_compat::mt_draw_count();
    return engine_();
  }
  static result_type min() { return 0u; }
  static result_type max() { return 0xffffffffu; }
  std::mt19937 &engine() { return engine_; }

 private:
  std::mt19937 engine_;
};

}  // namespace random
}  // namespace boost

#endif
