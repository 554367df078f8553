// Fused stage kernels in the reference's expression order (built with
// --fmad=false): FP64 results equal the reference's routine chain bit for bit.
#define STAGE_FAST false
#define STAGE_LAUNCH_FN launch_stage_strict
#include "stage_impl.cuh"
