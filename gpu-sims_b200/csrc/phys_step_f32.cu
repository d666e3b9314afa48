// Physics-mode step kernels with f32 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_f32, LBM_PREC_F32, false)
