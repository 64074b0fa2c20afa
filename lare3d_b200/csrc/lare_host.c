/*
 * lare_host.c - host-side helpers of the user-deck layer.
 *
 * KISS random numbers exactly as src/core/random_generator.f90 produces them
 * (32-bit two's-complement wrap-around, logical shifts), used to seed the
 * synthetic initial states the same way a Lare3d deck would.
 */
#include <stdint.h>

typedef struct {
  uint32_t x, y, z, w;
} kiss_state;

/* random_generator.f90:31-53 */
static double kiss_next(kiss_state* s) {
  s->x = 69069u * s->x + 1327217885u;
  uint32_t a1 = s->y;
  uint32_t a2 = a1 ^ (a1 << 13);
  uint32_t a3 = a2 ^ (a2 >> 17);
  s->y = a3 ^ (a3 << 5);
  s->z = 18000u * (s->z & 65535u) + (s->z >> 16);
  s->w = 30903u * (s->w & 65535u) + (s->w >> 16);
  int32_t kiss = (int32_t)(s->x + s->y + (s->z << 16) + s->w);
  return ((double)kiss + 2147483648.0) / 4294967296.0;
}

/* random_init_local (random_generator.f90:57-73) followed by n draws. */
void lare_kiss_fill(int seed, long n, double* out) {
  kiss_state s = {123456789u, 362436069u, 521288629u, 916191069u};
  uint32_t sd = (uint32_t)seed;
  s.x += sd; s.y += sd; s.z += sd; s.w += sd;
  for (int i = 0; i < 1000; ++i) (void)kiss_next(&s);
  for (long i = 0; i < n; ++i) out[i] = kiss_next(&s);
}
