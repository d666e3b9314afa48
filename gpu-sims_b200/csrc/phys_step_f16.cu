// Physics-mode step kernels with f16 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_f16, LBM_PREC_F16S, false)
