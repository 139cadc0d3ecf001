/* A weight-only truncator plugin for the propaq truncator ABI. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint32_t max_weight; } Ctx;

uint32_t propaq_truncator_abi_version(void) { return 1; }

void* propaq_truncator_create(const char* json) {
  Ctx* c = (Ctx*)malloc(sizeof(Ctx));
  c->max_weight = 1000;
  if (json) {
    const char* p = strstr(json, "\"max_weight\"");
    if (p && (p = strchr(p, ':'))) c->max_weight = (uint32_t)strtoul(p + 1, NULL, 10);
  }
  return c;
}
void propaq_truncator_destroy(void* c) { free(c); }

int32_t propaq_truncator_keep(void* ctx, uint32_t kind, const uint64_t* words, size_t n_words, uint32_t n_units,
                              uint32_t weight, double mag, uint32_t layer, uint32_t n_layers) {
  (void)kind; (void)words; (void)n_words; (void)n_units; (void)mag; (void)layer; (void)n_layers;
  return weight <= ((Ctx*)ctx)->max_weight;
}
