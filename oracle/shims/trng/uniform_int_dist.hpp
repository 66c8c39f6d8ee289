// Interface shim: uniform integer in [a, b) by scaling a 53-bit uniform.
#pragma once
#include <cstdint>

namespace trng {

class uniform_int_dist {
 public:
  using result_type = long;
  uniform_int_dist(long a, long b) : a_(a), d_(b - a) {}
  template <typename R>
  long operator()(R &r) {
    double u = double(uint64_t(r() >> 11)) * (1.0 / 9007199254740992.0);
    long v = a_ + long(u * double(d_));
    return v < a_ + d_ ? v : a_ + d_ - 1;
  }

 private:
  long a_, d_;
};

}  // namespace trng
