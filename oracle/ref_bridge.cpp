// TEST INFRASTRUCTURE ONLY — the oracle's link to the reference.
//
// Compiles TAMM's own src/tamm/kernels/multiply.hpp (block_multiply, CPU branch),
// src/tamm/kernels/assign.hpp (kernels::assign) and src/tamm/kernels/cpu_blas.cpp
// from the TAMM tree, with the stand-in third-party headers in oracle/ref_shim/, and
// exposes them through a C ABI so tests can pin the C restatement (tamm_oracle.c)
// against the reference and bench.py can time the reference's CPU path.
// Built by oracle/Makefile into oracle/_ref/libtamm_ref.so; never shipped.
#include "tamm/kernels/multiply.hpp"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace tamm {
// errors.cpp needs GA/MPI; a single-process stand-in for tamm_terminate.
void tamm_terminate(std::string msg) {
  std::fprintf(stderr, "%s ... terminating program.\n", msg.c_str());
  std::abort();
}
} // namespace tamm

extern "C" void scipy_openblas_set_num_threads64_(int);

namespace {
tamm::SizeVec to_sizes(const int64_t* d, int n) {
  tamm::SizeVec v;
  for(int i = 0; i < n; i++) v.push_back(tamm::Size{static_cast<uint64_t>(d[i])});
  return v;
}
tamm::IntLabelVec to_labels(const int* l, int n) { return tamm::IntLabelVec(l, l + n); }
} // namespace

extern "C" {

// tamm::kernels::block_multiply<double,double,double,double>(..., ExecutionHW::CPU, ...)
// (multiply.hpp:212-220).  Returns 0, or 1 when the reference raised EXPECTS /
// NOT_IMPLEMENTED.
int ref_block_multiply(double alpha, const double* abuf, const int64_t* adims, const int* alabels,
                       int na, const double* bbuf, const int64_t* bdims, const int* blabels, int nb,
                       double beta, double* cbuf, const int64_t* cdims, const int* clabels, int nc,
                       int is_assign) {
  try {
    tamm::gpuStream_t h{};
    double*           cdev = nullptr;
    double*           ctmp = nullptr;
    tamm::kernels::block_multiply<double, double, double, double>(
      h, alpha, abuf, to_sizes(adims, na), to_labels(alabels, na), bbuf, to_sizes(bdims, nb),
      to_labels(blabels, nb), beta, cbuf, to_sizes(cdims, nc), to_labels(clabels, nc),
      tamm::ExecutionHW::CPU, is_assign != 0, cdev, ctmp);
  } catch(std::string&) { return 1; } catch(std::exception&) {
    return 1;
  }
  return 0;
}

// tamm::kernels::assign<double> (assign.hpp:467-485).
int ref_assign(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
               const double* src, const int64_t* sdims, const int* slabels, int ns, int is_assign) {
  try {
    tamm::kernels::assign<double>(dst, to_sizes(ddims, nd), to_labels(dlabels, nd), scale, src,
                                  to_sizes(sdims, ns), to_labels(slabels, ns), is_assign != 0);
  } catch(std::string&) { return 1; } catch(std::exception&) {
    return 1;
  }
  return 0;
}

// Thread count of the OpenBLAS GEMM behind blas::gemm.
void ref_set_blas_threads(int n) { scipy_openblas_set_num_threads64_(n); }

} // extern "C"
