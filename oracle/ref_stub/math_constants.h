// math_constants.h stand-in for the host build of the reference's device
// program: the one constant it uses, single-precision infinity.
// TEST INFRASTRUCTURE ONLY.
#ifndef G4B_REF_MATH_CONSTANTS_H
#define G4B_REF_MATH_CONSTANTS_H

#define CUDART_INF_F __builtin_huge_valf()

#endif
