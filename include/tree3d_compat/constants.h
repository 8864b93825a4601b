/*
 * constants.h for programs written against the reference (ongbw/bit): the constants of
 * the reference's src/constants.h:8-38, the ones the drop-in uses taken from
 * tree3d_b200.h, plus the remaining physical constants under the reference's names.
 */
#ifndef constants_h
#define constants_h 1

#include "../tree3d_b200.h"

const double mu = 4e-7 * pi;
const double c = 3.0e8;
const double Bfield = 10.0;
const double endcap = -50.0;

#endif
