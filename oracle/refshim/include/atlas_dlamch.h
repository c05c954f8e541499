/* Stand-in for the generated FP64 machine parameters (ATLAS probes them at
 * configure time; these are the IEEE-754 binary64 values it finds on x86-64
 * with round-to-nearest). */
#ifndef ATLAS_DLAMCH_H
#define ATLAS_DLAMCH_H
#include <float.h>
#define ATL_dlaROUND 1
#define ATL_dlaSAFMIN DBL_MIN
#define ATL_dlaOVERTHRESH DBL_MAX
#define ATL_dlaUNDERTHRESH DBL_MIN
#define ATL_dlaMAXEXP DBL_MAX_EXP
#define ATL_dlaMINEXP DBL_MIN_EXP
#define ATL_dlaMANTDIG DBL_MANT_DIG
#define ATL_dlaPRECISION (DBL_EPSILON)
#define ATL_dlaBASE 2.0
#define ATL_dlaEPSILON (DBL_EPSILON * 0.5)
#endif
