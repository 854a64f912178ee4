// Hand-written shared-memory FFT Poisson solver (see fft.cu).
#pragma once

#include "mzb_common.cuh"

namespace mzb {

struct FftPoisson {
    int n = 0, nh = 0;
    double L = 0, h = 0;
    double2* spec = nullptr;  // [n][n][n/2+1]
    double2* W = nullptr;     // twiddles exp(-2 pi i t/n)
    double* freq = nullptr;   // [n]
    double* rfreq = nullptr;  // [n/2+1]

    void init(int n, double L, double h);
    void release();
    // phi = unnormalised-IFFT(FFT(q) * ig2), DC term passed through (fftw_wrap.c:166-189)
    void solve(const double* q, double* phi, cudaStream_t s) const;
};

}  // namespace mzb
