/* Stand-in for <fftw3.h> for the reference's time-series analysis tool: the typedefs and
 * allocators of ../ref_stub/fftw3.h plus the two transform calls the tool makes
 * (fftw_plan_dft_1d, fftw_execute), backed by the direct DFT in ../ref_dft.cpp.
 * Test infrastructure only. */
#ifndef ASD_REF_STUB_DFT_FFTW3_H
#define ASD_REF_STUB_DFT_FFTW3_H
#include "../ref_stub/fftw3.h"
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
#endif
