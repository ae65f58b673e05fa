/* TEST INFRASTRUCTURE ONLY.  Stand-in for the HPTT tensor-transpose library (not part
 * of the TAMM tree).  It implements the interface TAMM calls
 * (kernels/assign.hpp:396-400, ip_hptt.hpp:53-57) with HPTT's documented semantics:
 * row-major when rowMajor is set, sizeB[j] = sizeA[perm[j]], and
 * B = alpha * permute(A) + beta * B, B not read when beta == 0. */
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

namespace hptt {
enum SelectionMethod { ESTIMATE, MEASURE, PATIENT, CRAZY };

template<typename T>
class Transpose {
public:
  std::vector<int> perm_, size_a_;
  T                alpha_, beta_;
  const T*         a_;
  T*               b_;
  bool             row_major_;

  void execute() {
    const int        d = static_cast<int>(size_a_.size());
    std::vector<int> pa(perm_), sa(size_a_);
    if(!row_major_) { /* column-major input: view it as row-major with reversed modes */
      for(int j = 0; j < d; j++) pa[j] = d - 1 - perm_[d - 1 - j];
      for(int j = 0; j < d; j++) sa[j] = size_a_[d - 1 - j];
    }
    std::vector<int64_t> sb(d), ia(d, 0);
    int64_t              n = 1;
    for(int j = 0; j < d; j++) {
      sb[j] = sa[pa[j]];
      n *= sa[j];
    }
    for(int64_t lin = 0; lin < n; lin++) {
      int64_t ob = 0;
      for(int j = 0; j < d; j++) ob = ob * sb[j] + ia[pa[j]];
      b_[ob] = beta_ == T{0} ? alpha_ * a_[lin] : alpha_ * a_[lin] + beta_ * b_[ob];
      for(int q = d - 1; q >= 0; q--) {
        if(++ia[q] < sa[q]) break;
        ia[q] = 0;
      }
    }
  }
};

template<typename T>
std::shared_ptr<Transpose<T>> create_plan(const int* perm, int dim, T alpha, const T* A,
                                          const int* sizeA, const int* /*outerSizeA*/, T beta,
                                          T* B, const int* /*outerSizeB*/, SelectionMethod,
                                          int /*numThreads*/, const int* /*threadIds*/,
                                          bool useRowMajor) {
  auto p        = std::make_shared<Transpose<T>>();
  p->perm_      = std::vector<int>(perm, perm + dim);
  p->size_a_    = std::vector<int>(sizeA, sizeA + dim);
  p->alpha_     = alpha;
  p->beta_      = beta;
  p->a_         = A;
  p->b_         = B;
  p->row_major_ = useRowMajor;
  return p;
}
} // namespace hptt
