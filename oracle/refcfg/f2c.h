/* Shadow f2c.h for the reference's vendored AMD / GENMMD (f2c output).  The
 * reference passes 32-bit int* to these routines, so integer and logical must
 * be 32-bit here; the vendored header's 64-bit long makes them read past the
 * ends of their arrays. */
#ifndef ORACLE_F2C_SHADOW_H
#define ORACLE_F2C_SHADOW_H
/* pre-included with -include; defining the vendored header's guard turns the
 * vendored copy (found first by its quoted #include) into a no-op */
#define F2C_INCLUDE
typedef int integer;
typedef unsigned int uinteger;
typedef int logical;
typedef short shortint;
typedef float real;
typedef double doublereal;
typedef char *address;
typedef struct { real r, i; } complex;
typedef struct { doublereal r, i; } doublecomplex;
typedef short shortlogical;
typedef char logical1;
typedef char integer1;
typedef int ftnlen;
typedef int flag;
typedef int ftnint;
#define TRUE_ (1)
#define FALSE_ (0)
#define abs(x) ((x) >= 0 ? (x) : -(x))
#define min(a,b) ((a) <= (b) ? (a) : (b))
#define max(a,b) ((a) >= (b) ? (a) : (b))
#endif
