// Interface shim: uniform real in [a, b).
#pragma once
#include "trng/uniform01_dist.hpp"

namespace trng {

template <typename T = double>
class uniform_dist {
 public:
  using result_type = T;
  uniform_dist(T a, T b) : a_(a), b_(b) {}
  template <typename R>
  T operator()(R &r) { return a_ + (b_ - a_) * u_(r); }

 private:
  T a_, b_;
  uniform01_dist<double> u_;
};

}  // namespace trng
