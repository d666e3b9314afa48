// Physics-mode step kernels with bf16 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_bf16, LBM_PREC_BF16S, false)
