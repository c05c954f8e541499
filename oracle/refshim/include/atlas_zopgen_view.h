/* Stand-in for the generated amm "opgen" view of a tuned build: a table of
 * K-blockings 8, 16, ..., 64.  It sets only the QR blocking and the
 * recursion split points (rounding, not semantics). */
#ifndef ATL_VWopgen_MAX_KB
#define ATL_VWopgen_MAX_KB 64
#define ATL_VWopgen_100IDX 7
#define ATL_VWopgen_100KB 64
#define ATL_VWopgen_100LCMMN 8
#define ATL_VWopgen_99KB 56
#define ATL_VWopgen_99LCMMN 8
#define ATL_VWopgen_98KB 48
#define ATL_VWopgen_98LCMMN 8
#define ATL_GetVWopgenKB(i_) (((i_) + 1) * 8)
#endif
