/* Test infrastructure only.  Configuration of libsc for the serial build of
 * the reference's vendored p4est-1.1 that oracle/build_ref.sh compiles
 * directly with gcc (no MPI, no BLAS/LAPACK, no zlib, no Lua, no threads);
 * written for this recipe in place of the header p4est's configure would
 * generate. */
#ifndef SC_CONFIG_H
#define SC_CONFIG_H
#define SC_PACKAGE_STRING "libsc (serial build for the oracle)"
#define SC_VERSION "1.1"
#define SC_CC "gcc"
#define SC_CFLAGS "-O2"
#define SC_CPP "gcc -E"
#define SC_CPPFLAGS ""
#define SC_F77 "none"
#define SC_FFLAGS ""
#define SC_LDFLAGS ""
#define SC_LIBS "-lm"
#define SC_HAVE_SIGNAL_H 1
#define SC_HAVE_SYS_TIME_H 1
#define SC_HAVE_SYS_TYPES_H 1
#define SC_HAVE_TIME_H 1
#define SC_HAVE_STRTOLL 1
#define SC_HAVE_EXECINFO_H 1
#define SC_HAVE_BACKTRACE 1
#define SC_HAVE_BACKTRACE_SYMBOLS 1
#define SC_F77_FUNC(name, NAME) name##_
#endif
