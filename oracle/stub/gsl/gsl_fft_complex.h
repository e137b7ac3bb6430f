/* Stand-in for GSL's header, for compiling the reference's tune.c in the
 * oracle recipe.  tune.c declares the one function it calls itself
 * (gsl_fft_real_radix2_transform); oracle/gsl_fft_stub.c provides it. */
#ifndef ORACLE_STUB_GSL_FFT_COMPLEX_H
#define ORACLE_STUB_GSL_FFT_COMPLEX_H
#endif
