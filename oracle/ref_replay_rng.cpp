/*
 * oracle/ref_replay_rng.cpp -- TEST INFRASTRUCTURE, linked only into the
 * reference build under oracle/_ref/.
 *
 * Replaces the reference's random number generators (Src/mersenne.cpp and
 * the Normal() of Src/stoc1.cpp) with the counter stream of irbc_rng.h, so
 * that the unmodified reference step functions consume the same draws as the
 * oracle and the CUDA library.  The class layouts come from the reference's
 * own headers (Include/randomc.h, Include/stocc.h); only the member
 * functions the reference calls are defined here.
 */
#include <stdint.h>
#include "Include/randomc.h"
#include "Include/stocc.h"
#include "irbc_rng.h"

static uint64_t g_seed = 0;
static uint32_t g_ustream = ORC_STREAM_INIT, g_nstream = ORC_STREAM_COLLIDE_N;
static uint64_t g_uepoch = 0, g_nepoch = 0, g_ucur = 0, g_ncur = 0;

extern "C" void ref_rng_seed(uint64_t seed) { g_seed = seed; }
extern "C" void ref_rng_set_uniform(uint32_t stream, uint64_t epoch) {
  g_ustream = stream; g_uepoch = epoch; g_ucur = 0;
}
extern "C" void ref_rng_set_normal(uint32_t stream, uint64_t epoch) {
  g_nstream = stream; g_nepoch = epoch; g_ncur = 0;
}
extern "C" uint64_t ref_rng_uniform_cursor() { return g_ucur; }
extern "C" uint64_t ref_rng_normal_cursor() { return g_ncur; }

void CRandomMersenne::RandomInit(int) { mti = 0; }

uint32_t CRandomMersenne::BRandom() {
  uint32_t o[4];
  orc_block(g_seed, g_ustream, g_uepoch, g_ucur >> 2, o);
  return o[(g_ucur++) & 3u];
}

// Random(): 32 random bits times 2^-32 (Src/mersenne.cpp:108-112)
double CRandomMersenne::Random() { return (double)BRandom() * (1. / (65536. * 65536.)); }

// IRandom (Src/mersenne.cpp:115-125), same formula over the replaced bits
int CRandomMersenne::IRandom(int min, int max) {
  if (max <= min) {
    if (max == min) return min; else return (int)0x80000000;
  }
  int r = int((double)(uint32_t)(max - min + 1) * Random() + min);
  if (r > max) r = max;
  return r;
}

StochasticLib1::StochasticLib1(int seed) : STOC_BASE(seed) { normal_x2_valid = 0; }

double StochasticLib1::Normal(double m, double s) {
  return orc_normal(g_seed, g_nstream, g_nepoch, g_ncur++) * s + m;
}
