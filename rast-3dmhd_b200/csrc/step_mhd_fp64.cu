// step_mhd_fp64.cu - placeholder until the MHD stage kernel lands.
#include "r3d_kernels.h"
namespace r3dk {
cudaError_t launch_stage_mhd_fp64(int, const Geometry&, const Physics&, const Lines&,
                                  const FieldSet&, Scalars*, int, cudaStream_t) {
    return cudaErrorNotSupported;
}
}  // namespace r3dk
