// Double-precision FFT used by the CPU oracle (test infrastructure only).
//
// The reference calls cuFFT (a closed library) for every transform
// (Markerfree/src/method/Cufft1&2.cu:32,42,50,67,95,103,121,143,163).  The oracle
// restates the published discrete Fourier transform with cuFFT's conventions:
//   forward  X[k] = sum_n x[n] exp(-2 pi i k n / N)   (unnormalised)
//   inverse  x[n] = sum_k X[k] exp(+2 pi i k n / N)   (unnormalised)
//   R2C keeps bins 0..N/2, C2R reads bins 0..N/2 and assumes Hermitian symmetry.
// Sizes with only factors 2,3,5,7 use mixed-radix Cooley-Tukey; other prime
// factors use Bluestein's chirp-z algorithm (Bluestein 1970).
#pragma once
#include <complex>
#include <vector>

namespace oc {

typedef std::complex<double> cd;

// In-place complex transform of length n; sign = -1 forward, +1 inverse.
void fft_c2c(cd* data, int n, int sign);

// Real-to-complex 1-D: in[n] -> out[n/2+1].
void fft_r2c_1d(const double* in, cd* out, int n);
// Complex-to-real 1-D (unnormalised): in[n/2+1] -> out[n].
void fft_c2r_1d(const cd* in, double* out, int n);

// 2-D R2C on an ny x nx real image (row stride in_stride doubles) into an
// ny x (nx/2+1) complex array (row stride nx/2+1).
void fft_r2c_2d(const double* in, int in_stride, cd* out, int nx, int ny);
// 2-D C2R (unnormalised): ny x (nx/2+1) complex -> ny x nx real (row stride out_stride).
void fft_c2r_2d(const cd* in, double* out, int out_stride, int nx, int ny);

}  // namespace oc
