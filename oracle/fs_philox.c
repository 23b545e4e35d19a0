/*
 * fs_philox.c — CPU restatement of the production modes' external drive
 * draws.  TEST INFRASTRUCTURE ONLY: tests/ and the smoke check load it as the
 * checker of the device code; nothing in the product links or calls it.
 *
 * What it restates:
 *  - Philox-4x32-10, the counter-based generator of Salmon, Moraes, Dror and
 *    Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds
 *    of two 32x32->64 multiplications (multipliers 0xD2511F53, 0xCD9E8D57)
 *    with the key bumped by the Weyl constants 0x9E3779B9 / 0xBB67AE85
 *    between rounds.  Pinned against an independent implementation
 *    (cuRAND's host Philox4_32_10 generator) by tests/test_philox.py.
 *  - The per-(step, neuron) drive draws of the production kernel
 *    (draw_inputs in flysim_b200/csrc/fs_prod.cu), which replace the
 *    reference's sequential std::mt19937 draws of EqsGnl2::BgInit
 *    (code/EqsGnl2.cpp:284-337: one uniform per receptor in the order AMPA,
 *    GABA, ACh, GluCl, NMDA; a hit when the uniform is below the receptor's
 *    per-step probability) and its ziggurat injection noise
 *    (code/EqsGnl2.cpp:335, code/StiExt.h:214-218) by a Box-Muller normal:
 *      block 0 = Philox(key, (t_lo, t_hi, neuron, 0)): word r is receptor
 *        r's uniform for r = AMPA, GABA, ACh, GluCl (hit: pb > u24(word));
 *      block 1 = Philox(key, (t_lo, t_hi, neuron, 1)), drawn only when the
 *        neuron's NMDA drive is on with pb > 0 or its injection is on:
 *        word 0 is the NMDA uniform, words 1 and 2 the Box-Muller inputs
 *        u1 = (w1 >> 8 + 1) 2^-24 in (0, 1], u2 = (w2 >> 8) 2^-24,
 *        z = sqrt(-2 ln u1) cos(2 pi u2), current = mean + std z (one fused
 *        multiply-add in the state type);
 *    u24(w) = (w >> 8) 2^-24, exact in float.
 *  - The stream key of a reset: key0 = low word of the user key XOR the
 *    run seed, key1 = high word XOR 0x5eed5eed (prod_reset in fs_prod.cu).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void oracle_drive_key(uint64_t user_key, uint32_t seed, uint32_t key[2]) {
  key[0] = (uint32_t)user_key ^ seed;
  key[1] = (uint32_t)(user_key >> 32) ^ 0x5eed5eedu;
}

static float u24(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

/* cos(pi x) with the argument reduced exactly (every reduction step below is
 * an exact floating-point subtraction), so only the final cos / sin rounds */
static double cospi_ref(double x) {
  double y = fmod(fabs(x), 2.0);
  if (y > 1.0) y = 2.0 - y;
  double sign = 1.0;
  if (y > 0.5) { y = 1.0 - y; sign = -1.0; }
  const double pi = 3.141592653589793238462643383279502884;
  return sign * (y > 0.25 ? sin(pi * (0.5 - y)) : cos(pi * y));
}

/* Draws of steps [t0, t0 + nsteps) for neurons [first, first + count) of an
 * n-neuron network: hits[j * count + q] bit r = receptor r hit; gauss[j *
 * count + q] = the injection current (state type: fp64 != 0 double, else
 * float), 0 where the neuron's injection is off.  pb is receptor-major
 * [5][n]; act holds the ActCtr bits (AMPA 1, GABA 2, NMDA 4, INJ 128). */
void oracle_drive_draws(const uint32_t key[2], uint64_t t0, uint32_t nsteps, uint32_t first, uint32_t count,
                        uint32_t n, const float *pb, const uint32_t *act, const float *inj_mean,
                        const float *inj_std, int fp64, uint8_t *hits, double *gauss) {
  for (uint32_t j = 0; j < nsteps; j++) {
    const uint64_t t = t0 + j;
    for (uint32_t q = 0; q < count; q++) {
      const uint32_t p = first + q;
      const uint32_t a = act[p];
      uint32_t c[4] = {(uint32_t)t, (uint32_t)(t >> 32), p, 0u}, r1[4], r2[4];
      oracle_philox4x32_10(c, key, r1);
      uint32_t h = 0;
      for (int r = 0; r < 4; r++)
        if (pb[(size_t)r * n + p] > u24(r1[r])) h |= 1u << r;
      double gv = 0.0;
      const float pbn = pb[(size_t)4 * n + p];
      if (((a & 4u) && pbn > 0.0f) || (a & 128u)) {
        c[3] = 1u;
        oracle_philox4x32_10(c, key, r2);
        if (pbn > u24(r2[0])) h |= 1u << 4;
        if (a & 128u) {
          const double u1 = ((double)(r2[1] >> 8) + 1.0) * 5.9604644775390625e-08;
          const double u2 = (double)(r2[2] >> 8) * 5.9604644775390625e-08;
          const double z = sqrt(-2.0 * log(u1)) * cospi_ref(2.0 * u2);
          if (fp64) gv = fma((double)inj_std[p], z, (double)inj_mean[p]);
          else gv = (double)fmaf(inj_std[p], (float)z, inj_mean[p]);
        }
      }
      hits[(size_t)j * count + q] = (uint8_t)h;
      gauss[(size_t)j * count + q] = gv;
    }
  }
}
