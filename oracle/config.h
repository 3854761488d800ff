/* Hand-written configuration header for compiling the snogray reference
 * renderer's C++ core as a CPU oracle.  It stands in for the header that the
 * reference's autoconf script would generate (configure.ac), with the
 * features of this toolchain (GCC 13, libstdc++, glibc) switched on and the
 * optional image libraries (libpng, libjpeg, OpenEXR, netpbm) switched off,
 * since their headers are absent.
 *
 * HAVE_FEENABLEEXCEPT is deliberately left undefined: the reference enables
 * FE_DIVBYZERO|FE_INVALID traps around rendering when it is available
 * (util/float-excepts-guard.h:38-66); without it the guard is a no-op and the
 * oracle's arithmetic results are unchanged.
 */
#ifndef SNOGRAY_ORACLE_CONFIG_H
#define SNOGRAY_ORACLE_CONFIG_H

#define PACKAGE_NAME "snogray"
#define PACKAGE_VERSION "0.6-oracle"
#define PACKAGE_STRING "snogray 0.6-oracle"

#define USE_THREADS 1
#define USE_STD_THREAD 1
#define USE_STD_RANDOM 1

#define HAVE_STD_UNIQUE_PTR 1
#define HAVE_STD_TRUNC 1
#define HAVE_STD_COPYSIGN 1
#define HAVE_INTPTR_T 1
#define HAVE_STDINT_H 1
#define HAVE_STDLIB_H 1
#define HAVE_FENV_H 1
#define HAVE_EXTERN_TEMPLATE 1
#define EXTERN_TEMPLATE_EXTENSION

#endif
