// Headless C++ host of the D3Q19 step, written the way the reference sim's
// frame loop drives its compute path (volumetric-grid/lattice-boltzmann/
// src/main.cpp), but through the C ABI of include/lbm.h:
//
//   allocate_tier_images (:835-846)      -> lbm_create
//   apply_preset (:1167-1211)            -> lbm_set_flags_naca + lbm_init_equilibrium
//   per-frame uniform upload (:1523-1537)-> lbm_get_params / lbm_set_params when a slider moved
//   substep chain (:1554-1591)           -> lbm_step(substeps)
//   VDB export (:1767-1790)              -> lbm_vdb_export
//
// plus the fp64 mass / momentum sums every frame.  No window, no Vulkan: the
// final moments and mask are written as raw files for whoever checks them.
//
//   lbm_frame_loop NX NY NZ NACA AOA_DEG TAU UX UY UZ FRAMES SUBSTEPS
//                  CHANGE_FRAME TAU2 UX2 UY2 UZ2 OUT_PREFIX [VDB_DIR]
//
// At frame CHANGE_FRAME the tau and u_inf "sliders" move to TAU2 / U*2.
// Writes OUT_PREFIX.rho.bin (float[N]), .u.bin (float[N][3]) and
// .mask.bin (uint8[N]); prints one JSON line (per-frame sums, the last
// iteration, the wall time of the frame loop).  Exit status 1 on any error,
// with the library's message on stderr.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "lbm.h"

namespace {

lbm_ctx* g_ctx = nullptr;

void check(int rc, const char* what) {
  if (rc == LBM_OK) return;
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, lbm_last_error(g_ctx));
  if (g_ctx) lbm_destroy(g_ctx);
  std::exit(1);
}

bool write_file(const std::string& path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
  return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 18 && argc != 19) {
    std::fprintf(stderr,
                 "usage: %s NX NY NZ NACA AOA_DEG TAU UX UY UZ FRAMES SUBSTEPS CHANGE_FRAME "
                 "TAU2 UX2 UY2 UZ2 OUT_PREFIX [VDB_DIR]\n",
                 argv[0]);
    return 2;
  }
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  const char* naca = argv[4];
  const float aoa = std::strtof(argv[5], nullptr), tau = std::strtof(argv[6], nullptr);
  const float u_inf[3] = {std::strtof(argv[7], nullptr), std::strtof(argv[8], nullptr),
                          std::strtof(argv[9], nullptr)};
  const int frames = std::atoi(argv[10]), substeps = std::atoi(argv[11]), change = std::atoi(argv[12]);
  const float tau2 = std::strtof(argv[13], nullptr);
  const float u_inf2[3] = {std::strtof(argv[14], nullptr), std::strtof(argv[15], nullptr),
                           std::strtof(argv[16], nullptr)};
  const std::string out = argv[17];
  const char* vdb_dir = argc == 19 ? argv[18] : nullptr;

  // the tier's context (reference mode: the reference's own step semantics)
  lbm_desc d;
  check(lbm_desc_default(&d), "lbm_desc_default");
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.tau = tau;
  for (int a = 0; a < 3; ++a) d.u_inf[a] = u_inf[a];
  check(lbm_create(&d, &g_ctx), "lbm_create");

  // apply_preset: the airfoil mask made on the device, then the equilibrium
  check(lbm_set_flags_naca(g_ctx, naca, 0.25f, 0.25f, aoa), "lbm_set_flags_naca");
  check(lbm_init_equilibrium(g_ctx, 1.0f, u_inf), "lbm_init_equilibrium");

  std::vector<double> sums(4 * (size_t)frames);
  const auto t0 = std::chrono::steady_clock::now();
  for (int f = 0; f < frames; ++f) {
    if (f == change) {  // a slider moved: the next frame's uniforms change
      lbm_params p;
      p.struct_size = sizeof p;
      check(lbm_get_params(g_ctx, &p), "lbm_get_params");
      p.tau = tau2;
      for (int a = 0; a < 3; ++a) p.u_inf[a] = u_inf2[a];
      check(lbm_set_params(g_ctx, &p), "lbm_set_params");
    }
    check(lbm_step(g_ctx, substeps), "lbm_step");
    check(lbm_conservation(g_ctx, &sums[4 * (size_t)f]), "lbm_conservation");
  }
  check(lbm_sync(g_ctx), "lbm_sync");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  const size_t n = (size_t)nx * ny * nz;
  std::vector<float> rho(n), u(3 * n);
  std::vector<uint8_t> mask(n);
  check(lbm_read_moments(g_ctx, rho.data(), u.data(), LBM_U_F32X3), "lbm_read_moments");
  check(lbm_read_mask(g_ctx, mask.data(), n), "lbm_read_mask");
  if (!write_file(out + ".rho.bin", rho.data(), n * sizeof(float)) ||
      !write_file(out + ".u.bin", u.data(), 3 * n * sizeof(float)) ||
      !write_file(out + ".mask.bin", mask.data(), n)) {
    std::fprintf(stderr, "cannot write %s.*.bin\n", out.c_str());
    lbm_destroy(g_ctx);
    return 1;
  }
  if (vdb_dir) {
    const int rc = lbm_vdb_export(g_ctx, vdb_dir, (uint32_t)(frames - 1), 0);
    if (rc != LBM_OK) {
      std::fprintf(stderr, "lbm_vdb_export failed (%d): %s\n", rc, lbm_vdb_last_error());
      lbm_destroy(g_ctx);
      return 1;
    }
  }
  lbm_info info;
  info.struct_size = sizeof info;
  check(lbm_get_info(g_ctx, &info), "lbm_get_info");

  std::printf("{\"frames\": %d, \"substeps\": %d, \"iteration\": %llu, \"seconds\": %.6f, \"sums\": [", frames,
              substeps, (unsigned long long)info.iteration, secs);
  for (int f = 0; f < frames; ++f)
    std::printf("%s[%.17g, %.17g, %.17g, %.17g]", f ? ", " : "", sums[4 * (size_t)f], sums[4 * (size_t)f + 1],
                sums[4 * (size_t)f + 2], sums[4 * (size_t)f + 3]);
  std::printf("]}\n");
  check(lbm_destroy(g_ctx), "lbm_destroy");
  return 0;
}
