// Test infrastructure: stand-in for Boost.Random's uniform_real_distribution, used only
// to build the reference sources as an oracle.
//
// Boost (>= 1.47, the reference's makefile points at 1.49.0) draws a real uniform from an
// integral engine with ONE engine output per value:
//     u = (x - eng.min()) / ((eng.max() - eng.min()) + 1) * (b - a) + a,
// retried only if u >= b.  For mt19937 this is x / 2^32 on [0,1).  This differs from
// std::uniform_real_distribution (which uses two 32-bit outputs per double), so the
// standard one cannot be used here.
#ifndef MPSQMC_COMPAT_BOOST_UNIFORM_REAL_HPP
#define MPSQMC_COMPAT_BOOST_UNIFORM_REAL_HPP

namespace boost {
namespace random {

template <class RealType = double>
class uniform_real_distribution {
 public:
  typedef RealType result_type;
  explicit uniform_real_distribution(RealType a = RealType(0), RealType b = RealType(1))
      : a_(a), b_(b) {}
  template <class Engine>
  RealType operator()(Engine &eng) const {
    for (;;) {
      const RealType numerator = static_cast<RealType>(eng() - (eng.min)());
      const RealType divisor = static_cast<RealType>((eng.max)() - (eng.min)()) + RealType(1);
      const RealType r = numerator / divisor * (b_ - a_) + a_;
      if (r < b_) return r;
    }
  }
  RealType a() const { return a_; }
  RealType b() const { return b_; }

 private:
  RealType a_, b_;
};

}  // namespace random
}  // namespace boost

#endif
