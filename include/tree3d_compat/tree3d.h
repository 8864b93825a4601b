/*
 * tree3d.h for programs written against the reference (ongbw/bit).
 *
 * Put include/tree3d_compat first on the include path and link -ltree3d_b200 -lbit_b200:
 * a program that includes "tree3d.h" (and "constants.h", "problem.h") then compiles
 * unchanged and runs on the GPU.  This header gives the caller what the reference's
 * src/tree3d.h gives it: the standard headers that header includes, its
 * `using namespace std`, the constants, and the treecode declarations (here those of
 * tree3d_b200.h).
 *
 * The reference compiles DEL and KERNEL_ORDER into its library from the program's
 * problem.h (src/problem.h:11-13).  The drop-in reads them at run time, so when a
 * problem.h is on the include path its values are copied into bit_tree3d_del,
 * bit_tree3d_mac_del and bit_tree3d_kernel_order when the program starts.
 */
#ifndef tree3D_h
#define tree3D_h 1

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>

#include "constants.h"
#include "../tree3d_b200.h"

using namespace std;

#if defined(__has_include)
#if __has_include("problem.h")
#include "problem.h"
namespace {
const int bit_tree3d_problem_constants_ =
    (bit_tree3d_del = DEL, bit_tree3d_mac_del = DEL, bit_tree3d_kernel_order = KERNEL_ORDER, 0);
}
#endif
#endif

#endif
