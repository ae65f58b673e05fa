/* TEST INFRASTRUCTURE ONLY.  Stand-in for the blaspp interface that GA's ga_linalg.h
 * exposes to TAMM (blas::gemm / axpy / copy, as called at kernels/cpu_blas.cpp:8 and
 * multop.hpp:509).  Real double GEMM forwards to OpenBLAS's ILP64 CBLAS entry point
 * (the libscipy_openblas64_ build shipped with numpy); other types use plain loops. */
#pragma once
#include <complex>
#include <cstdint>
#include <type_traits>

extern "C" void scipy_cblas_dgemm64_(int order, int ta, int tb, int64_t m, int64_t n, int64_t k,
                                     double alpha, const double* A, int64_t lda, const double* B,
                                     int64_t ldb, double beta, double* C, int64_t ldc);

namespace blas {
enum class Layout { RowMajor, ColMajor };
enum class Op { NoTrans, Trans, ConjTrans };

template<typename TS, typename TA, typename TB, typename TC>
void gemm(Layout layout, Op ta, Op tb, int64_t m, int64_t n, int64_t k, TS alpha, const TA* A,
          int64_t lda, const TB* B, int64_t ldb, TS beta, TC* C, int64_t ldc) {
  if constexpr(std::is_same_v<TS, double> && std::is_same_v<TA, double> &&
               std::is_same_v<TB, double> && std::is_same_v<TC, double>) {
    scipy_cblas_dgemm64_(layout == Layout::RowMajor ? 101 : 102, ta == Op::NoTrans ? 111 : 112,
                         tb == Op::NoTrans ? 111 : 112, m, n, k, alpha, A, lda, B, ldb, beta, C,
                         ldc);
  }
  else {
    for(int64_t i = 0; i < m; i++)
      for(int64_t j = 0; j < n; j++) {
        TC acc{0};
        for(int64_t p = 0; p < k; p++) {
          auto a = ta == Op::NoTrans ? A[i * lda + p] : A[p * lda + i];
          auto b = tb == Op::NoTrans ? B[p * ldb + j] : B[j * ldb + p];
          acc += TC(a) * TC(b);
        }
        C[i * ldc + j] = beta == TS{0} ? TC(alpha) * acc : TC(alpha) * acc + TC(beta) * C[i * ldc + j];
      }
  }
}

template<typename T>
void axpy(int64_t n, T alpha, const T* x, int64_t incx, T* y, int64_t incy) {
  for(int64_t i = 0; i < n; i++) y[i * incy] += alpha * x[i * incx];
}

template<typename T, typename U>
void copy(int64_t n, const T* x, int64_t incx, U* y, int64_t incy) {
  for(int64_t i = 0; i < n; i++) y[i * incy] = x[i * incx];
}
} // namespace blas
