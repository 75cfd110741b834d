/*
 * ORACLE (test infrastructure only): Philox-4x32-10 counter-based generator on the
 * CPU, restated from Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11 (the Random123 paper), section 4 ("Philox").  The product keeps
 * its own device copy; this one exists so the oracle draws the SAME uniforms as the
 * GPU from the same (key, counter) and so it can be checked against published
 * known-answer vectors independently of the product.
 */
#pragma once
#include <cstdint>

namespace oracle {

static inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t n0 = hi1 ^ c[1] ^ k[0];
  const uint32_t n2 = hi0 ^ c[3] ^ k[1];
  c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
}

/* 10 rounds, key bumped by the Weyl constants between rounds. */
static inline void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  uint32_t k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    if (r) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
    philox_round(c, k);
  }
  out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}

/* Uniform on the open interval (0,1): the top 23 bits plus half a step, i.e.
 * (2k+1) * 2^-24 with k < 2^23.  That needs 24 significant bits, so every value is
 * exactly representable in binary32 and binary64: an FP32 consumer and an FP64
 * consumer see the identical number, and it is never 0 or 1. */
static inline double u01(uint32_t x) { return ((double)(x >> 9) + 0.5) * (1.0 / 8388608.0); }

/* Stream tags (counter word 3).  Word 0 = particle / sample index, word 1 = draw
 * block (event number in transport), word 2 = time-step index. */
enum : uint32_t {
  TAG_TRANSPORT = 0x10000000u,
  TAG_BOUNDARY  = 0x20000000u,  /* | side (0..3) */
  TAG_SOURCE    = 0x30000000u,
  TAG_EMISSION  = 0x40000000u,
  TAG_IC        = 0x50000000u,
  TAG_COMB      = 0x60000000u,
};

struct Draw4 { double u[4]; };

static inline Draw4 draw(uint64_t seed, uint32_t idx, uint32_t block, uint32_t step, uint32_t tag) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t ctr[4] = {idx, block, step, tag};
  uint32_t o[4];
  philox4x32_10(ctr, key, o);
  return Draw4{{u01(o[0]), u01(o[1]), u01(o[2]), u01(o[3])}};
}

}  // namespace oracle
