// lu_tc.cu -- tcgen05 tensor-core trailing update of the mixed-precision LU.
#include "lu.cuh"

namespace uvlm {

bool gemm_tc_available() { return false; }

Error gemm_update_tc(float*, int, const float*, int, const float*, int, int, int, int, LuUpdate, LuWork*,
                     cudaStream_t) {
  return fail(kErrUnsupported, "tensor-core update not built");
}

}  // namespace uvlm
