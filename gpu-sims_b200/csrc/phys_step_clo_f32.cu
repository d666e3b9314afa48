// Physics-mode step kernels with the learned closure, f32 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_clo_f32, LBM_PREC_F32, true)
