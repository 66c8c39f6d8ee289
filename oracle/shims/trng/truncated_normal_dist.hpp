// Interface shim: normal(mu, sigma) truncated to [a, b) by rejection, normal
// draws by the Box-Muller transform.
#pragma once
#include <cmath>
#include "trng/uniform01_dist.hpp"

namespace trng {

template <typename T = double>
class truncated_normal_dist {
 public:
  using result_type = T;
  truncated_normal_dist(T mu, T sigma, T a, T b) : mu_(mu), s_(sigma), a_(a), b_(b) {}
  template <typename R>
  T operator()(R &r) {
    for (int it = 0; it < 1000; ++it) {
      double u1 = u_(r), u2 = u_(r);
      if (u1 <= 0.0) continue;
      double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      T x = T(mu_ + s_ * z);
      if (x >= a_ && x < b_) return x;
    }
    return a_;
  }

 private:
  T mu_, s_, a_, b_;
  uniform01_dist<double> u_;
};

}  // namespace trng
