// Internal host-side helpers of libmce.so: seeded RNG, CSR building.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <vector>

#include "../../include/mce.h"

namespace mce {

// SplitMix64 (Steele, Lea, Flood 2014): used to derive independent seeds.
inline uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// xoshiro256** (Blackman, Vigna 2018): the generators' random stream.
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed, uint64_t stream = 0) {
    uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  inline uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform double in [0, 1) from the top 53 bits
  inline double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform integer in [0, bound) (Lemire's multiply-shift; bias < 2^-32 for
  // bound < 2^32, which is irrelevant for graph generation)
  inline uint64_t below(uint64_t bound) {
    return (uint64_t)(((unsigned __int128)next() * bound) >> 64);
  }
  inline int64_t range(int64_t lo, int64_t hi) {  // inclusive
    return lo + (int64_t)below((uint64_t)(hi - lo + 1));
  }
};

// Undirected edge list -> normalised CSR (both directions, no loops, sorted
// rows, unique).  Pairs are (src[i], dst[i]).  Fails with MCE_ELIMIT if the
// result has 2^31 or more arcs.
int build_csr(const std::vector<std::pair<int64_t, int64_t>> &pairs, int64_t n,
              mce_hgraph_t *out);

// Allocate the arrays of a single-graph mce_hgraph_t.
int hgraph_alloc(mce_hgraph_t *g, int64_t n, int64_t m, int32_t num_graphs);

// Choose k distinct values from [0, n) (Floyd's algorithm), ascending.
std::vector<int64_t> sample_distinct(Rng &rng, int64_t n, int64_t k);

}  // namespace mce
