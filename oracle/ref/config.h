/* Configuration header for building the reference's fermion-solve subset as a
 * test oracle.  The reference's own build generates this file with autoconf;
 * this hand-written stand-in selects the single-rank build with the improved
 * Wilson kernel (the only kernel variant of the reference that compiles) and
 * the default message verbosity. */
#ifndef IROIRO_ORACLE_REF_CONFIG_H
#define IROIRO_ORACLE_REF_CONFIG_H
#define IMPROVED_WILSON 1
#define VERBOSITY 1
#define HAVE_SQRT 1
#define STDC_HEADERS 1
#endif
/* The package macros sit outside the include guard: include/iroiro_config.h
   undefines them and includes this file again to define them afresh. */
#ifndef PACKAGE
#define PACKAGE "iroiro"
#define PACKAGE_BUGREPORT ""
#define PACKAGE_NAME "IroIro"
#define PACKAGE_STRING "IroIro 1.0.9"
#define PACKAGE_TARNAME "iroiro"
#define PACKAGE_URL ""
#define PACKAGE_VERSION "1.0.9"
#define VERSION "1.0.9"
#endif
