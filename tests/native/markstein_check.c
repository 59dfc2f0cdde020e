/* The dot-step kernels divide by T1 and T2 through a precomputed
 * reciprocal and one Markstein correction (q0 = x*y; r = fma(-q0, t, x);
 * q = fma(r, y, q0)).  This program checks, in IEEE binary64 on the host
 * (the same operations the GPU performs, all correctly rounded), that the
 * result equals x / t bit for bit on random operands over 64 binades, on
 * divisors with all-ones, near-power-of-two and short significands, and on a
 * grid of decay-time-like divisors.  Exit status 1 on any mismatch. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static uint64_t state = 0x9E3779B97F4A7C15ull;

static uint64_t next_u64(void)
{
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double make_double(int exponent, uint64_t significand)
{
  const uint64_t bits = ((uint64_t)(exponent + 1023) << 52) | (significand & ((1ull << 52) - 1));
  double d;
  memcpy(&d, &bits, 8);
  return d;
}

static double div_by(double x, double t, double y)
{
  const double q0 = x * y;
  const double r = fma(-q0, t, x);
  return r == 0.0 ? q0 : fma(r, y, q0);
}

int main(int argc, char **argv)
{
  long long samples = 20000000LL, bad = 0, n = 0;
  if(argc > 1) sscanf(argv[1], "%lld", &samples);
  for(long long i = 0; i < samples; ++i) {
    const uint64_t a = next_u64(), b = next_u64();
    const int ex = (int)(a >> 58) - 32, et = (int)(b >> 58) - 32;
    uint64_t mt = b;
    switch(i & 7) {
    case 1: mt = (1ull << 52) - 1 - (b & 0xFF); break; /* significand near all ones */
    case 2: mt = b & 0xFF; break;                      /* near a power of two */
    case 3: mt = (b & 0xFFFF) << 36; break;            /* few significant bits */
    default: break;
    }
    double x = make_double(ex, a);
    const double t = make_double(et, mt);
    if(a & (1ull << 57)) x = -x;
    const double q = div_by(x, t, 1.0 / t), e = x / t;
    ++n;
    if(memcmp(&q, &e, 8) != 0) {
      if(bad < 10) printf("mismatch x=%a t=%a got=%a want=%a\n", x, t, q, e);
      ++bad;
    }
  }
  for(int i = -2000; i <= 2000; ++i)
    for(int j = 1; j <= 1000; ++j) {
      const double x = i * 0.001, t = j * 0.01;
      const double q = div_by(x, t, 1.0 / t), e = x / t;
      ++n;
      if(memcmp(&q, &e, 8) != 0) {
        if(bad < 20) printf("mismatch x=%a t=%a\n", x, t);
        ++bad;
      }
    }
  printf("checked %lld, mismatches %lld\n", n, bad);
  return bad != 0;
}
