/* Test infrastructure only.  Configuration of p4est for the serial build of
 * the reference's vendored p4est-1.1 that oracle/build_ref.sh compiles
 * directly with gcc; written for this recipe in place of the header p4est's
 * configure would generate. */
#ifndef P4EST_CONFIG_H
#define P4EST_CONFIG_H
#define P4EST_PACKAGE_STRING "p4est (serial build for the oracle)"
#define P4EST_VERSION "1.1"
#define P4EST_PACKAGE_VERSION "1.1"
#define P4EST_HAVE_UNISTD_H 1
#define P4EST_HAVE_NETINET_IN_H 1
#define P4EST_VERSION_MAJOR 1
#define P4EST_VERSION_MINOR 1
#define P4EST_CC "gcc"
#define P4EST_CFLAGS "-O2"
#define P4EST_CPP "gcc -E"
#define P4EST_CPPFLAGS ""
#define P4EST_LDFLAGS ""
#define P4EST_LIBS "-lm"
#endif
