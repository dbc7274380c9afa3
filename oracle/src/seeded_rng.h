/*
 * Test infrastructure: the seeded input generator shared by the oracle and
 * the reference-side drivers. Counter-based SplitMix64 (Steele, Lea, Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014): the k-th
 * output of the generator seeded with `seed` is mix(seed + (k+1)*GAMMA).
 * Being counter-based, a value depends only on (seed, k), so a cell's input
 * does not depend on the order cells are visited. The product side
 * (ops_b200/seeded.py) implements the same function with numpy uint64
 * arithmetic; a CPU test checks the two agree bit for bit.
 */
#ifndef ORACLE_SEEDED_RNG_H
#define ORACLE_SEEDED_RNG_H
#include <stdint.h>
#include <math.h>

#define SM64_GAMMA 0x9E3779B97F4A7C15ULL

static inline uint64_t sm64_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* k-th raw 64-bit output of the stream `seed` (k = 0, 1, ...). */
static inline uint64_t sm64_at(uint64_t seed, uint64_t k) {
  return sm64_mix(seed + (k + 1) * SM64_GAMMA);
}

/* Uniform double in [0, 1): top 53 bits of the k-th output. */
static inline double sm64_u01(uint64_t seed, uint64_t k) {
  return (double)(sm64_at(seed, k) >> 11) * (1.0 / 9007199254740992.0);
}

/* Uniform double in [lo, hi). */
static inline double sm64_uniform(uint64_t seed, uint64_t k, double lo, double hi) {
  return lo + (hi - lo) * sm64_u01(seed, k);
}

#endif
