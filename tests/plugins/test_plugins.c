/* Test plugins for the propaq plugin ABI, compiled into several shared
 * libraries with -D switches (see tests/test_api.py).  Each variant is a
 * small, deliberately minimal implementation of the ABI contract. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double damping; } Ctx;

static double parse(const char* json, const char* key, double dflt) {
  if (!json) return dflt;
  const char* p = strstr(json, key);
  if (!p) return dflt;
  p = strchr(p, ':');
  return p ? atof(p + 1) : dflt;
}

#ifdef BAD_ABI
uint32_t propaq_noise_abi_version(void) { return 2; }
#else
uint32_t propaq_noise_abi_version(void) { return 1; }
#endif

#ifdef UNKNOWN_DEPENDS
uint32_t propaq_noise_depends(void) { return 4; }
#endif
#ifdef LAYERED
uint32_t propaq_noise_depends(void) { return 2; }
#endif
#ifdef KEYED
uint32_t propaq_noise_depends(void) { return 1; }
#endif

void* propaq_noise_create(const char* json) {
  Ctx* c = (Ctx*)malloc(sizeof(Ctx));
  c->damping = parse(json, "\"damping\"", 0.0);
  return c;
}
#ifndef NO_DESTROY
void propaq_noise_destroy(void* c) { free(c); }
#endif

#ifndef NO_FACTOR
double propaq_noise_factor(void* ctx, uint32_t kind, const uint64_t* words, size_t n_words, uint32_t n_units,
                           uint32_t weight, uint32_t layer, uint32_t n_layers) {
  (void)kind; (void)n_units; (void)n_layers;
  double d = ((Ctx*)ctx)->damping;
#ifdef LAYERED
  d *= 1.0 + 0.25 * (double)layer;
#else
  (void)layer;
#endif
#ifdef KEYED
  /* damp only terms touching unit 0 */
  if (!words || n_words == 0 || !(words[0] & 3u)) return 1.0;
#else
  (void)words; (void)n_words;
#endif
  return exp(-d * (double)weight);
}
#endif
