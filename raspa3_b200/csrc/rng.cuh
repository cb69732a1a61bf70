// Counter-based random numbers of the device-resident Monte Carlo kernels: Philox-4x32-10 (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11). A draw is a pure function of (seed, stream, move,
// slot), so any thread, block or cluster rank can reproduce any number without shared generator state.
#pragma once

#include <cstdint>

namespace rgd
{
__device__ __forceinline__ void philox(uint32_t ctr[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
  for (int r = 0; r < 10; ++r)
  {
    const uint32_t hi0 = __umulhi(0xD2511F53u, ctr[0]), lo0 = 0xD2511F53u * ctr[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, ctr[2]), lo1 = 0xCD9E8D57u * ctr[2];
    const uint32_t n0 = hi1 ^ ctr[1] ^ k0, n1 = lo1, n2 = hi0 ^ ctr[3] ^ k1, n3 = lo0;
    ctr[0] = n0;
    ctr[1] = n1;
    ctr[2] = n2;
    ctr[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Two uniform doubles in [0,1) (53 random bits each) for (stream, move, slot).
__device__ __forceinline__ double2 uniform2(unsigned long long seed, int stream, long long move, uint32_t slot)
{
  uint32_t c[4] = {slot, static_cast<uint32_t>(move), static_cast<uint32_t>(move >> 32),
                   static_cast<uint32_t>(stream)};
  philox(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
  const unsigned long long a = (static_cast<unsigned long long>(c[0]) << 32) | c[1];
  const unsigned long long b = (static_cast<unsigned long long>(c[2]) << 32) | c[3];
  return make_double2(static_cast<double>(a >> 11) * 0x1.0p-53, static_cast<double>(b >> 11) * 0x1.0p-53);
}
}  // namespace rgd
