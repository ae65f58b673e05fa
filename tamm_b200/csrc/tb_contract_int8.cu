// Split-INT8 (Ozaki-style) contraction on the tcgen05 INT8 tensor cores.
#include "tb_internal.hpp"

namespace tb {

void contract_int8(Plan&, const WorkList&, double, const double*, const double*, double*,
                   cudaStream_t) {
  fail(TB_ERR_NOT_IMPLEMENTED, "split-INT8 contraction is not built yet");
}

void contract_bf16x3(Plan&, const WorkList&, double, const double*, const double*, double*,
                     cudaStream_t) {
  fail(TB_ERR_NOT_IMPLEMENTED, "BF16x3 contraction is not built yet");
}

} // namespace tb
