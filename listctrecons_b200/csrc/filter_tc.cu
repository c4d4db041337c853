// Stage 3 on the tensor cores: the Toeplitz GEMM form of the row convolution.
#include "lct_internal.h"

namespace lct {

int launch_filter_bf16x3(int ns, const float* d_h, float* d_rows, long long nrows,
                         cudaStream_t s) {
  (void)ns; (void)d_h; (void)d_rows; (void)nrows; (void)s;
  return LCT_ERR_UNSUPPORTED;
}

}  // namespace lct
