// Physics-mode step kernels with the learned closure, bf16 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_clo_bf16, LBM_PREC_BF16S, true)
