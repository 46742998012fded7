// Checks gann::FastDiv (the record-addressing division of the batched walk)
// against integer division on the host: every numerator below 2^20 for divisors
// 1..300, and for divisors up to 4096 the numerators next to each multiple near
// the top of the range, 2^31 - 1, and a pseudo-random sample.
#include <cstdint>
#include <cstdio>

#include "../gustann_b200/csrc/gann_internal.h"

int main() {
  uint64_t checked = 0;
  auto check = [&](uint32_t d, uint32_t n) {
    const gann::FastDiv f(d);
    if (f.div(n) != n / d) {
      std::printf("mismatch d=%u n=%u got %u want %u\n", d, n, f.div(n), n / d);
      return false;
    }
    checked++;
    return true;
  };
  for (uint32_t d = 1; d <= 300; d++)
    for (uint32_t n = 0; n < (1u << 20); n++)
      if (!check(d, n)) return 1;
  uint64_t x = 88172645463325252ull;
  for (uint32_t d = 1; d <= 4096; d++) {
    const uint32_t top = 0x7fffffffu;
    for (uint32_t q = top / d - 2; q <= top / d && q != 0xffffffffu; q++)
      for (int64_t off = -1; off <= 1; off++) {
        const int64_t n = (int64_t)q * d + off;
        if (n >= 0 && n <= top && !check(d, (uint32_t)n)) return 1;
      }
    if (!check(d, top)) return 1;
    for (int i = 0; i < 2000; i++) {
      x ^= x << 13;
      x ^= x >> 7;
      x ^= x << 17;
      if (!check(d, (uint32_t)(x & 0x7fffffffu))) return 1;
    }
  }
  std::printf("ok %llu\n", (unsigned long long)checked);
  return 0;
}
