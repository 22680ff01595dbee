// The final stage on the tcgen05 tensor cores (sm_100a). Not built yet: the plain float32 final stage
// (final_fp32.cu) is the one that runs.
#include "kernels.h"

namespace ffbp {

cudaError_t launch_final_tc(const FinalLaunch &, int, cudaStream_t, const char **why)
{
    *why = "the tensor-core final stage is not built in this version";
    return cudaErrorNotSupported;
}

}  // namespace ffbp
