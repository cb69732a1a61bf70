// xoshiro256** seeded through splitmix64: the random stream of the CPU oracle (test infrastructure only).
#ifndef RASPA_ORACLE_RNG_H
#define RASPA_ORACLE_RNG_H

#include <cstdint>

namespace oracle_rng
{
struct Rng
{
  uint64_t s[4];
  explicit Rng(uint64_t seed)
  {
    for (int i = 0; i < 4; ++i)
    {
      seed += 0x9e3779b97f4a7c15ULL;
      uint64_t z = seed;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s[i] = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next()
  {
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
};
}  // namespace oracle_rng

#endif
