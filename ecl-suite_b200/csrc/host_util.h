// Small host-side helpers shared by the generators and the runtime.
#pragma once
#include <cstdint>

namespace ecl {
namespace host {

// SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014): a bijective 64-bit mixer used as a
// counter-based random number source.
inline uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// Uniform double in [0, 1) from the top 53 bits.
inline double unit_double(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace host
}  // namespace ecl
