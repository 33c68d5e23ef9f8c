/* Hand-written stand-in for the header LELA's configure script would
 * generate.  It fixes the integer widths for x86-64 Linux (LP64) and turns
 * every optional dependency off (no GMP beyond the stand-in in ../gmpxx.h,
 * no CBLAS, no M4RI, no libpng).  Test infrastructure only: used to build
 * the reference's own CPU path as the oracle under oracle/_ref. */
#ifndef ORACLE_SHIM_LELA_CONFIG_H
#define ORACLE_SHIM_LELA_CONFIG_H
#define __LELA_INT8 char
#define __LELA_INT16 short
#define __LELA_INT32 int
#define __LELA_INT64 long long
#define __LELA_UINT128 unsigned __int128
#define __LELA_HAVE_LITTLE_ENDIAN 1
#define __LELA_SIZEOF_CHAR 1
#define __LELA_SIZEOF_SHORT 2
#define __LELA_SIZEOF_INT 4
#define __LELA_SIZEOF_LONG 8
#define __LELA_SIZEOF_LONG_LONG 8
#endif
