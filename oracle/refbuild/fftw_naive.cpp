// DFT-by-definition implementation of the FFTW 3 entry points that the reference's Dnfft1D
// uses (include/dca/math/nfft/dnfft_1d.hpp:447-455 and :506-515).
//
// Test infrastructure only: lets the reference's own SpAccumulator<CPU> run in this container,
// which has no FFTW.  Semantics follow FFTW's documented definitions:
//   r2c (forward):  out[k] = sum_j in[j] exp(-2 pi i j k / n),  k = 0 .. n/2
//   c2c:            out[k] = sum_j in[j] exp(sign * 2 pi i j k / n)
// The phase index j*k is reduced modulo n in integers before the sine/cosine, so twiddles are
// exact to double rounding for every n.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fftw3.h"

struct fftw_plan_s {
  int kind;  // 0: r2c, 1: c2c
  int n;
  int sign;
  double* rin;
  fftw_complex* cin;
  fftw_complex* out;
};

extern "C" {

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned) {
  return new fftw_plan_s{0, n, FFTW_FORWARD, in, nullptr, out};
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
  return new fftw_plan_s{1, n, sign, nullptr, in, out};
}

fftw_plan fftw_plan_many_dft(int, const int*, int, fftw_complex*, const int*, int, int,
                             fftw_complex*, const int*, int, int, int, unsigned) {
  std::fprintf(stderr, "fftw_plan_many_dft is not provided by the test stub\n");
  std::abort();
}

void fftw_execute(const fftw_plan p) {
  const int n = p->n;
  std::vector<double> c(n), s(n);
  for (int m = 0; m < n; ++m) {
    const double arg = 2.0 * M_PI * static_cast<double>(m) / static_cast<double>(n);
    c[m] = std::cos(arg);
    s[m] = std::sin(arg);
  }
  if (p->kind == 0) {
    std::vector<double> re(n / 2 + 1), im(n / 2 + 1);
    for (int k = 0; k <= n / 2; ++k) {
      double acc_r = 0, acc_i = 0;
      for (int j = 0; j < n; ++j) {
        const int m = static_cast<int>((static_cast<long long>(j) * k) % n);
        acc_r += p->rin[j] * c[m];
        acc_i -= p->rin[j] * s[m];
      }
      re[k] = acc_r;
      im[k] = acc_i;
    }
    for (int k = 0; k <= n / 2; ++k) {
      p->out[k][0] = re[k];
      p->out[k][1] = im[k];
    }
  }
  else {
    const double sg = p->sign > 0 ? 1.0 : -1.0;
    std::vector<double> re(n), im(n);
    for (int k = 0; k < n; ++k) {
      double acc_r = 0, acc_i = 0;
      for (int j = 0; j < n; ++j) {
        const int m = static_cast<int>((static_cast<long long>(j) * k) % n);
        const double xr = p->cin[j][0], xi = p->cin[j][1];
        acc_r += xr * c[m] - sg * xi * s[m];
        acc_i += xi * c[m] + sg * xr * s[m];
      }
      re[k] = acc_r;
      im[k] = acc_i;
    }
    for (int k = 0; k < n; ++k) {
      p->out[k][0] = re[k];
      p->out[k][1] = im[k];
    }
  }
}

void fftw_destroy_plan(fftw_plan p) {
  delete p;
}
}
