/* Stand-in for the generated cache description: a 32 KiB L1 data cache
 * (4096 doubles), the size below which getrfC / geqrr stop recursing. */
#ifndef ATLAS_CACHE_H
#define ATLAS_CACHE_H
#define L1C_ELTS 4096
#endif
