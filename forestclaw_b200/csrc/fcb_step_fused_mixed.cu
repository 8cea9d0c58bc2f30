// Ghost-exchange-fused mixed FP32/FP64 form of the pipelined step kernel
// (fcb_step_pipe.cuh, FUSED; the arithmetic of fcb_step_mixed.cu).
#include "fcb_step_pipe.cuh"

namespace fcb {

cudaError_t launch_step_pipe_fused_mixed(int solver, int aux_kind, int mwaves, int mx, int my, int mbc,
                                         int claw_version, const StepArgs& a, cudaStream_t st) {
    return launch_step_pipe_t<float, true>(solver, aux_kind, mwaves, mx, my, mbc, claw_version, a, st);
}

}  // namespace fcb
