// Interface shim for the trng4 "lcg64" engine, written for this project so the
// reference's CPU code compiles without trng4 (not available offline).  It is
// NOT trng4: only the interface (seed / split / operator()) matches.
//   state update : x <- a*x + c (mod 2^64), Knuth's MMIX constants
//                  (TAOCP vol. 2, 3rd ed., sec. 3.3.4: a = 6364136223846793005,
//                  c = 1442695040888963407)
//   split(s, i)  : leapfrog partition -- the stream keeps elements i, i+s, ...
//                  (a' = a^s, c' = c (1 + a + ... + a^(s-1)), x advanced i steps)
//   output       : murmur3 fmix64 finalizer of the pre-update state
//                  (Appleby, MurmurHash3), so low state bits do not leak.
#pragma once
#include <cstdint>
#include <stdexcept>

namespace trng {

class lcg64 {
 public:
  using result_type = unsigned long long;
  static constexpr result_type min() { return 0ull; }
  static constexpr result_type max() { return ~0ull; }

  lcg64() = default;
  explicit lcg64(unsigned long long s) { seed(s); }

  void seed(unsigned long long s) { x_ = s; }

  result_type operator()() {
    uint64_t out = x_;
    x_ = a_ * x_ + c_;
    out ^= out >> 33;
    out *= 0xff51afd7ed558ccdull;
    out ^= out >> 33;
    out *= 0xc4ceb9fe1a85ec53ull;
    out ^= out >> 33;
    return out;
  }

  void split(unsigned int s, unsigned int i) {
    if (s < 1 || i >= s) throw std::invalid_argument("invalid argument for trng::lcg64::split");
    if (s == 1) return;
    for (unsigned int j = 0; j < i; ++j) x_ = a_ * x_ + c_;
    uint64_t as = 1, cs = 0;  // compose the update s times
    for (unsigned int j = 0; j < s; ++j) {
      cs = a_ * cs + c_;
      as = a_ * as;
    }
    a_ = as;
    c_ = cs;
  }

  void jump(unsigned long long n) {
    for (unsigned long long j = 0; j < n; ++j) x_ = a_ * x_ + c_;
  }

 private:
  uint64_t a_ = 6364136223846793005ull;
  uint64_t c_ = 1442695040888963407ull;
  uint64_t x_ = 0;
};

}  // namespace trng
