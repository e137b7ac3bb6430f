/* Stand-in for GSL's header, for compiling the reference's tune.c in the
 * oracle recipe (GSL is not installed here); tune.c uses nothing from it. */
#ifndef ORACLE_STUB_GSL_ERRNO_H
#define ORACLE_STUB_GSL_ERRNO_H
#endif
