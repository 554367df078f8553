// Fused stage kernels with FMA and the single-reciprocal WENO5 weights
// (weno_fast.cuh); FP64 within 1e-12 relative of the reference.
#define STAGE_FAST true
#define STAGE_LAUNCH_FN launch_stage_fast
#define STAGE_BAND_FN launch_stage_band
#include "stage_impl.cuh"
