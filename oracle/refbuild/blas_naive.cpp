// Column-major ZGEMM with the reference-BLAS (netlib) semantics:
//   C <- alpha * op(A) * op(B) + beta * C,  op(X) in {X, X^T, X^H} selected by 'N', 'T', 'C'.
//
// Test infrastructure only: the container has no system BLAS, and the reference's CPU
// accumulators call zgemm_ through include/dca/linalg/blas/blas3.hpp:29-32.  This is a plain
// triple loop (j, l, i order, unit stride over i), single threaded, so that one reference
// accumulator instance uses exactly one core.
#include <complex>

using zcomplex = std::complex<double>;

extern "C" void zgemm_(const char* transa, const char* transb, const int* m_, const int* n_,
                       const int* k_, const zcomplex* alpha_, const zcomplex* a, const int* lda_,
                       const zcomplex* b, const int* ldb_, const zcomplex* beta_, zcomplex* c,
                       const int* ldc_) {
  const int m = *m_, n = *n_, k = *k_, lda = *lda_, ldb = *ldb_, ldc = *ldc_;
  const zcomplex alpha = *alpha_, beta = *beta_;
  const char ta = *transa, tb = *transb;
  const bool a_n = (ta == 'N' || ta == 'n'), a_c = (ta == 'C' || ta == 'c');
  const bool b_n = (tb == 'N' || tb == 'n'), b_c = (tb == 'C' || tb == 'c');

  auto A = [&](int i, int l) -> zcomplex {
    if (a_n)
      return a[i + static_cast<long>(lda) * l];
    const zcomplex v = a[l + static_cast<long>(lda) * i];
    return a_c ? std::conj(v) : v;
  };
  auto B = [&](int l, int j) -> zcomplex {
    if (b_n)
      return b[l + static_cast<long>(ldb) * j];
    const zcomplex v = b[j + static_cast<long>(ldb) * l];
    return b_c ? std::conj(v) : v;
  };

  for (int j = 0; j < n; ++j) {
    zcomplex* cj = c + static_cast<long>(ldc) * j;
    if (beta == zcomplex(0))
      for (int i = 0; i < m; ++i)
        cj[i] = 0;
    else if (beta != zcomplex(1))
      for (int i = 0; i < m; ++i)
        cj[i] *= beta;
    for (int l = 0; l < k; ++l) {
      const zcomplex t = alpha * B(l, j);
      if (t == zcomplex(0))
        continue;
      if (a_n) {
        const zcomplex* al = a + static_cast<long>(lda) * l;
        for (int i = 0; i < m; ++i)
          cj[i] += t * al[i];
      }
      else {
        for (int i = 0; i < m; ++i)
          cj[i] += t * A(i, l);
      }
    }
  }
}
