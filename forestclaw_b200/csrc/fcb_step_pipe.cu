// FP64 form of the pipelined step kernel (fcb_step_pipe.cuh), compiled with
// -fmad=false so that every product and sum is rounded as in the reference.
#include "fcb_step_pipe.cuh"

namespace fcb {

cudaError_t launch_step_pipe(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, int claw_version, const StepArgs& a,
                             cudaStream_t st) {
    return launch_step_pipe_t<double, false>(solver, aux_kind, mwaves, mx, my, mbc, claw_version, a, st);
}

}  // namespace fcb
