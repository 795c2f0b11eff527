// Direct O(n^2) discrete Fourier transform behind the fftw_plan_dft_1d / fftw_execute calls of
// the reference's time-series analysis tool (FFTW itself is not installed).  The transform is
// X_k = sum_j x_j exp(sign 2 pi i j k / n), FFTW's definition, accumulated in long double with
// the phase reduced exactly as (j k) mod n.  Test infrastructure only.
#include "ref_stub_dft/fftw3.h"
#include <cmath>
#include <vector>

namespace {
struct Plan {
    int n, sign;
    fftw_complex *in, *out;
};
}  // namespace

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    return new Plan{n, sign, in, out};
}

void fftw_execute(const fftw_plan p) {
    const Plan* q = static_cast<const Plan*>(p);
    const int n = q->n;
    const long double two_pi = 6.283185307179586476925286766559L;
    std::vector<long double> c(n), s(n);
    for (int m = 0; m < n; m++) {
        c[m] = cosl(two_pi * m / n);
        s[m] = sinl(two_pi * m / n);
    }
    std::vector<long double> re(n), im(n);
    for (int k = 0; k < n; k++) {
        long double a = 0.0L, b = 0.0L;
        for (int j = 0; j < n; j++) {
            const int m = (int)(((long long)j * k) % n);
            const long double cr = c[m], ci = q->sign * s[m];
            a += q->in[j][0] * cr - q->in[j][1] * ci;
            b += q->in[j][0] * ci + q->in[j][1] * cr;
        }
        re[k] = a;
        im[k] = b;
    }
    for (int k = 0; k < n; k++) {
        q->out[k][0] = (double)re[k];
        q->out[k][1] = (double)im[k];
    }
}
