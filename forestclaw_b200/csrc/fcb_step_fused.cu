// Ghost-exchange-fused FP64 form of the pipelined step kernel
// (fcb_step_pipe.cuh, FUSED): on a mesh of one level the step reads its ghost
// cells from the neighbours' interiors in the arena of the previous step and
// writes the updated interiors to the other arena.  Compiled with
// -fmad=false, as the unfused FP64 form.
#include "fcb_step_pipe.cuh"

namespace fcb {

cudaError_t launch_step_pipe_fused(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, int claw_version,
                                   const StepArgs& a, cudaStream_t st) {
    return launch_step_pipe_t<double, true>(solver, aux_kind, mwaves, mx, my, mbc, claw_version, a, st);
}

}  // namespace fcb
