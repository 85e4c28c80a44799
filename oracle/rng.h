/*
 * ORACLE (test infrastructure): the reference's counter-based random numbers, restated.
 *
 * src/lumen/_core/rng.py:71-97 draws every random number through JAX's threefry PRNG:
 *   photon_key(key, id) = fold_in(key, id); vertex_key(pkey, v) = fold_in(pkey, v)         (rng.py:71-78)
 *   uniforms(key, n)[i] = ((bits_i >> 9) + 0.5) 2^-23, bits_i in threefry's partitionable mode (rng.py:81-95)
 * JAX's published algorithm (jax/_src/prng.py): fold_in(k, d) = threefry2x32(k, (0, d)); PRNGKey(s) = (0, s) for a
 * 32-bit seed; partitionable bits(k, (n,))[i] = y0 ^ y1 with (y0, y1) = threefry2x32(k, (0, i)).
 * threefry2x32 is Threefry-2x32 with 20 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
 * 1, 2, 3", SC'11), pinned by the Random123 known-answer vectors in tests/test_rng.py.
 */
#ifndef LUMEN_ORACLE_RNG_H
#define LUMEN_ORACLE_RNG_H
#include <stdint.h>

typedef struct { uint32_t k0, k1; } OKey;

static inline uint32_t o_rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

static inline void o_threefry(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1, uint32_t* y0, uint32_t* y1) {
  const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
  static const int R0[4] = {13, 15, 26, 6};
  static const int R1[4] = {17, 29, 16, 24};
  x0 += k0; x1 += k1;
#define O_ROUNDS(R) for (int j = 0; j < 4; ++j) { x0 += x1; x1 = o_rotl(x1, R[j]); x1 ^= x0; }
  O_ROUNDS(R0); x0 += k1; x1 += k2 + 1u;
  O_ROUNDS(R1); x0 += k2; x1 += k0 + 2u;
  O_ROUNDS(R0); x0 += k0; x1 += k1 + 3u;
  O_ROUNDS(R1); x0 += k1; x1 += k2 + 4u;
  O_ROUNDS(R0); x0 += k2; x1 += k0 + 5u;
#undef O_ROUNDS
  *y0 = x0; *y1 = x1;
}

static inline OKey o_fold_in(OKey k, uint32_t d) {
  OKey r;
  o_threefry(k.k0, k.k1, 0u, d, &r.k0, &r.k1);
  return r;
}

/* uniform i of key k, in (0, 1): (k + 1/2) 2^-23 with k the top 23 bits */
static inline float o_uniform(OKey k, uint32_t i) {
  uint32_t y0, y1;
  o_threefry(k.k0, k.k1, 0u, i, &y0, &y1);
  uint32_t b = (y0 ^ y1) >> 9;
  return ((float)b + 0.5f) * 1.1920928955078125e-7f;
}

#endif
