// pairwise_tc.cu -- tensor-core forms of the pairwise RMSD matrix (pending).
#include "../../include/warpmd_rmsd.h"
#include "pairwise_tc.h"

namespace wmd {

int pairwise_tc_run(PairwiseWorkspace&, int, const float*, int64_t, int64_t, int, const uint32_t*, int64_t, int, int,
                    float*, int*, cudaStream_t, std::string* msg) {
  *msg = "tensor-core pairwise modes are not built in this version";
  return WMD_ERR_UNSUPPORTED;
}

}  // namespace wmd
