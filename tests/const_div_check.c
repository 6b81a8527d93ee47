/* Exhaustive check of hicar_b200/csrc/const_div.h: for every non-negative
 * float x (zero, subnormals, normals and +infinity), the double-product
 * quotient (float)((double)x * ICAR_RCP{d}_D) must equal the IEEE quotient
 * x/d bit for bit, d = 12 and 60.  Negative x follow by symmetry (both
 * sides are odd functions under round-to-nearest-even).  Prints the number
 * of x checked and of mismatches per divisor; exit status 1 on any
 * mismatch.  Build: cc -O2 -ffp-contract=off -fopenmp const_div_check.c */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../hicar_b200/csrc/const_div.h"

static float from_bits(uint32_t u)
{
    float f;
    memcpy(&f, &u, 4);
    return f;
}
static uint32_t to_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

int main(void)
{
    const float d[2] = {12.0f, 60.0f};
    const double r[2] = {ICAR_RCP12_D, ICAR_RCP60_D};
    const long long last = 0x7f800000LL;  /* +infinity */
    int fail = 0;
    for (int t = 0; t < 2; t++) {
        long long bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
        for (long long u = 0; u <= last; u++) {
            const float x = from_bits((uint32_t)u);
            volatile float ref = x / d[t];
            const float q = (float)((double)x * r[t]);
            bad += to_bits(q) != to_bits(ref);
        }
        printf("d=%g checked=%lld mismatches=%lld\n", d[t], last + 1, bad);
        fail |= bad != 0;
    }
    return fail;
}
