// Interface shim: uniform real in [0, 1) from the top mantissa bits of one draw.
#pragma once
#include <cstdint>

namespace trng {

template <typename T = double>
class uniform01_dist {
 public:
  using result_type = T;
  template <typename R>
  T operator()(R &r) {
    if constexpr (sizeof(T) <= 4)
      return T(uint32_t(r() >> 40)) * T(1.0 / 16777216.0);
    else
      return T(uint64_t(r() >> 11)) * T(1.0 / 9007199254740992.0);
  }
};

}  // namespace trng
