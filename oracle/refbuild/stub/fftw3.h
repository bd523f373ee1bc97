// Minimal FFTW3 interface for building the reference's CPU accumulators without FFTW.
//
// Test infrastructure only (the reference build recipe under oracle/refbuild).  The
// declarations follow FFTW 3's public API as documented at fftw.org ("The Basic Interface",
// "One-Dimensional DFTs of Real Data").  fftw_naive.cpp implements the few entry points the
// reference's Dnfft1D calls (dnfft_1d.hpp:447 r2c forward, :506 c2c backward) by the DFT
// definition; nothing else is implemented.
#ifndef ORACLE_REFBUILD_STUB_FFTW3_H
#define ORACLE_REFBUILD_STUB_FFTW3_H

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

extern "C" {
fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in,
                             const int* inembed, int istride, int idist, fftw_complex* out,
                             const int* onembed, int ostride, int odist, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
}

#endif  // ORACLE_REFBUILD_STUB_FFTW3_H
