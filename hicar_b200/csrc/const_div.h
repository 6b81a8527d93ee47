/* Correctly rounded division of a float by the constant divisors of the
 * high-order flux formulas (flux3, src/physics/advect.f90:149-185: /12 and
 * /60) without the general division sequence: one double-precision product
 * with the double nearest to 1/d, rounded back to float,
 *
 *     x / d  ==  (float)((double)x * ICAR_RCP{d}_D).
 *
 * The product carries a relative error of at most about 2^-52, far inside
 * the distance from a non-midpoint quotient to the nearest float rounding
 * boundary, and a quotient that is exactly a float or a midpoint is a
 * short binary fraction that the double product reproduces exactly, so the
 * final rounding agrees with IEEE division.  tests/const_div_check.c
 * verifies the identity bit for bit for every non-negative float (zero,
 * subnormals and infinity included; negative x follow by symmetry, NaN
 * stays NaN), and tests/test_const_division.py checks the constants.
 *
 * Plain C so that the exhaustive check can include it. */
#ifndef ICAR_CONST_DIV_H
#define ICAR_CONST_DIV_H

#define ICAR_RCP12_D 0x1.5555555555555p-4
#define ICAR_RCP60_D 0x1.1111111111111p-6

#endif
