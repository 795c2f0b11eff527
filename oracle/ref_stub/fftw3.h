/* Minimal stand-in for <fftw3.h> so that the reference's header-only Array
 * containers compile without FFTW installed.  Only the typedefs and the
 * allocation functions the containers use are provided; no transform is
 * available (the CPU FFT field path is not built by the harness). */
#ifndef ASD_REF_STUB_FFTW3_H
#define ASD_REF_STUB_FFTW3_H
#include <stdlib.h>
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef void* fftw_plan;
typedef void* fftwf_plan;
static inline void* fftw_malloc(size_t n) { return malloc(n); }
static inline void fftw_free(void* p) { free(p); }
static inline void* fftwf_malloc(size_t n) { return malloc(n); }
static inline void fftwf_free(void* p) { free(p); }
#endif
