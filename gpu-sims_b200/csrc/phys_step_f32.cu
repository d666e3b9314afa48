// Physics-mode step kernels with f32 population storage.
#include "phys_step_launch.cuh"

LBM_DEFINE_PHYS_STEP(phys_step_f32, LBM_PREC_F32, false)

namespace lbm {

uint32_t phys_cons_slots(const PhysGeom& g) {
  const uint32_t nyz = (uint32_t)g.ny * (uint32_t)g.nz;
  return (uint32_t)((g.nx + 31) / 32) * nyz + 2u * 4u * ((nyz + 127u) / 128u);
}

// The slots the moment-writing launch of the step as configured fills:
// one per warp of the row kernel (two- or one-node rows), one per warp of
// the face kernel.  Four nodes per thread and the tensor-core closure write
// no partials.
bool phys_cons_layout(const Ctx& c, uint32_t* rows, uint32_t* faces) {
  if (!c.pp.cons || c.d.mode != LBM_MODE_PHYSICS) return false;
  if (c.closure && c.step_variant == 8) return false;
  if (!c.closure && c.d.precision != LBM_PREC_F32 && use_quads(c)) return false;
  const PhysGeom& G = c.pp.g;
  const uint32_t tiles = use_pairs(c) ? (uint32_t)((G.nx + 63) / 64) : (uint32_t)((G.nx + 31) / 32);
  const uint32_t nyz = (uint32_t)G.ny * (uint32_t)G.nz;
  *rows = tiles * nyz;
  *faces = c.pp.any_open ? 2u * 4u * ((nyz + 127u) / 128u) : 0u;
  return true;
}

}  // namespace lbm
