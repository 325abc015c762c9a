/* Regenerates the approximation tables of the x86 `rcpss` / `rsqrtss` instructions by executing them on the host.
 *
 * Lux.Engine reproduces Intel's approximate reciprocal and reciprocal square root bit for bit
 * (Lux.Engine/Imaging/IntelApprox.cs:21-45). Those results are a table function of the top 12 mantissa bits, scaled by a
 * power of two. This program executes the instructions on 1.m (exponent 127) for the reciprocal and on 1.m / 2.m
 * (exponents 127 / 128) for the reciprocal square root, and prints a C header with the three 4096-entry tables.
 * It must run on an Intel CPU: AMD processors implement different approximations.
 *
 * Build and run:  gcc -O1 -msse gen_intel_tables.c -o gen && ./gen > intel_approx_tables.h
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <xmmintrin.h>

static uint32_t bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float from_bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

static void table(const char* name, uint32_t exp_bits, int rsqrt) {
  printf("static const uint32_t %s[4096] = {\n", name);
  for (int i = 0; i < 4096; i++) {
    float x = from_bits(exp_bits | ((uint32_t)i << 11));
    __m128 v = _mm_set_ss(x);
    float r = _mm_cvtss_f32(rsqrt ? _mm_rsqrt_ss(v) : _mm_rcp_ss(v));
    printf("0x%08xu,%s", bits(r), (i % 8 == 7) ? "\n" : " ");
  }
  printf("};\n");
}

int main(void) {
  printf("/* Generated by gen_intel_tables.c from the rcpss / rsqrtss instructions of an Intel CPU. Do not edit. */\n");
  printf("#pragma once\n#include <stdint.h>\n");
  table("lux_rcp_table", 0x3f800000u, 0);        /* input exponent 127 */
  table("lux_rsqrt_table_e127", 0x3f800000u, 1); /* input exponent 127 (odd biased exponent) */
  table("lux_rsqrt_table_e128", 0x40000000u, 1); /* input exponent 128 (even biased exponent) */
  return 0;
}
