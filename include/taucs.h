/* Drop-in header for programs written against the reference's public header
 * (src/taucs.h with src/taucs_private.h): this library declares the same
 * types, flags, error codes and function names and signatures for the
 * multifrontal Cholesky path in taucs_b200.h, so such a program compiles
 * unchanged with -I<this directory> and links against libtaucs_b200.so. */
#ifndef TAUCS_H
#define TAUCS_H
#include "taucs_b200.h"
#endif
