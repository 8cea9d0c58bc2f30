// Mixed FP32/FP64 form of the pipelined step kernel (fcb_step_pipe.cuh):
// Riemann solves, limiters and transverse parts in FP32; the flux sums that
// form fm, fp, gm, gp, the conservative update and the stored state in FP64.
#include "fcb_step_pipe.cuh"

namespace fcb {

cudaError_t launch_step_pipe_mixed(int solver, int aux_kind, int mwaves, int mx, int my, int mbc,
                                   int claw_version, const StepArgs& a, cudaStream_t st) {
    return launch_step_pipe_t<float, false>(solver, aux_kind, mwaves, mx, my, mbc, claw_version, a, st);
}

}  // namespace fcb
