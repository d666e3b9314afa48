/*
 * lbm.h -- C ABI of the B200 D3Q19 lattice-Boltzmann step.
 *
 * This is the drop-in boundary for the `volumetric-grid/lattice-boltzmann`
 * sim of GPU-Sims.  The reference has no plugin or FFI API: its step is wired
 * directly into `main()` through Vulkan compute pipelines.  Each entry point
 * below names the reference code it replaces (paths relative to
 * `volumetric-grid/lattice-boltzmann/` unless stated otherwise).
 *
 * Conventions
 *  - Every call returns an int status: LBM_OK (0) or a negative LBM_ERR_*.
 *    No C++ exception crosses the ABI.  lbm_last_error() gives the message.
 *  - A context owns all of its device memory.  Host pointers passed in are
 *    borrowed for the duration of the call only.
 *  - Grids are linearised x-fastest: index = x + Nx*(y + Ny*z), exactly as
 *    the reference's obstacle mask (src/main.cpp:307) and capture buffers.
 *  - One context is driven by one host thread at a time, on one CUDA stream
 *    (lbm_set_stream; default: a stream the context creates).
 *  - Work is enqueued asynchronously on that stream; calls that return host
 *    data (read_*, conservation, sync) synchronise the stream first.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

#define LBM_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define LBM_OK                 0
#define LBM_ERR_INVALID_ARG   -1  /* bad pointer, size, enum or range        */
#define LBM_ERR_CUDA          -2  /* a CUDA runtime call failed               */
#define LBM_ERR_NO_DEVICE     -3  /* no CUDA device visible to this process   */
#define LBM_ERR_OUT_OF_MEMORY -4  /* device allocation failed                 */
#define LBM_ERR_STATE         -5  /* call out of order (e.g. step before init)*/
#define LBM_ERR_UNSUPPORTED   -6  /* option combination not built             */
#define LBM_ERR_TIMEOUT       -7  /* a bounded device-side wait gave up       */
#define LBM_ERR_NONFINITE     -8  /* NaN/Inf or rho<=0 found at a fluid node  */
#define LBM_ERR_IO            -9  /* capture file could not be read/written   */

/* ---- enums ------------------------------------------------------------- */
/* Semantics of the step.
 *  REFERENCE: the reference's four-pass step, reproduced literally:
 *    collide (shaders/collide.comp.glsl:39-61) with the lagged moments and
 *    velocity rounded to fp16 (the rgba16f image, src/main.cpp:843);
 *    clamp-to-edge pull stream (shaders/stream.comp.glsl:29-47);
 *    apply_boundaries (shaders/apply_boundaries.comp.glsl:57-169): solid
 *    zeroing, post-stream bounce-back against the mask with out-of-bounds
 *    counted as solid, equilibrium inlet/outlet, inverted free-slip;
 *    compute_moments (shaders/compute_moments.comp.glsl:29-50).
 *  PHYSICS: textbook stream-collide: periodic or half-way bounce-back faces,
 *    momentum-corrected moving walls, BGK or TRT, optional Smagorinsky and
 *    Guo body force.  Not present in the reference. */
enum lbm_mode      { LBM_MODE_REFERENCE = 0, LBM_MODE_PHYSICS = 1 };
/* Population storage.  F16S/BF16S store f_i - w_i (physics mode only);
 * collision arithmetic is fp32 in every case. */
enum lbm_precision { LBM_PREC_F32 = 0, LBM_PREC_F16S = 1, LBM_PREC_BF16S = 2 };
enum lbm_collision { LBM_COLL_BGK = 0, LBM_COLL_TRT = 1 };
/* Rounding applied to u between moments and the next collide (reference
 * mode).  Vulkan allows RTE or RTZ for float->half image stores. */
enum lbm_u_round   { LBM_UROUND_NONE = 0, LBM_UROUND_RTE = 1, LBM_UROUND_RTZ = 2 };
/* Host velocity formats for init/readback. */
enum lbm_u_format  { LBM_U_F32X3 = 0,   /* float[N][3]                        */
                     LBM_U_F16X4 = 1,   /* uint16 half[N][4], w=0: rgba16f    */
                     LBM_U_F32X4 = 2 }; /* float[N][4], w=0                   */
/* Open x faces (physics mode, x not periodic): the populations entering
 * through the face are rebuilt by the non-equilibrium bounce-back of Zou & He
 * (1997) in its D3Q19 form (Hecht & Harting 2010) instead of being bounced
 * back.  VELOCITY prescribes u = wall_velocity[face]; PRESSURE prescribes
 * rho = open_rho[x side] with zero tangential velocity.  The reference's
 * -X inlet / +X outlet (shaders/apply_boundaries.comp.glsl:86-130) write
 * equilibria; these are the Zou-He faces its notes plan as the upgrade
 * (docs/notes.md:5-7, 23-24). */
enum lbm_open      { LBM_OPEN_NONE = 0, LBM_OPEN_VELOCITY = 1, LBM_OPEN_PRESSURE = 2 };
/* Faces, for per-face wall velocities: x-, x+, y-, y+, z-, z+. */
enum lbm_face { LBM_FACE_XM = 0, LBM_FACE_XP, LBM_FACE_YM, LBM_FACE_YP,
                LBM_FACE_ZM, LBM_FACE_ZP };

/* ---- descriptor -------------------------------------------------------- */
typedef struct lbm_desc {
    uint32_t struct_size;       /* sizeof(lbm_desc), for ABI growth          */
    int32_t  nx, ny, nz;        /* lattice nodes; each in [2, 65535]         */
    int32_t  mode;              /* enum lbm_mode                             */
    int32_t  precision;         /* enum lbm_precision                        */
    int32_t  collision;         /* enum lbm_collision (physics mode)         */
    int32_t  periodic[3];       /* physics mode: 1 = periodic axis, 0 = wall */
    float    tau;               /* BGK relaxation time (> 0.5)               */
    float    trt_magic;         /* TRT Lambda; default 3/16                  */
    float    smagorinsky_cs;    /* 0 = off                                   */
    float    body_accel[3];     /* Guo force density F = rho * body_accel    */
    float    wall_velocity[6][3]; /* physics mode: moving-wall velocity per
                                   face (enum lbm_face); 0 = resting wall    */
    /* reference-mode knobs (src/main.cpp:1523-1537 uniforms) */
    float    u_inf[3];          /* inlet / init velocity (BoundariesUniforms) */
    float    rho0;              /* boundary density, RHO_0 = 1 (:90)          */
    int32_t  ref_inlet_outlet;  /* regime 3 of apply_boundaries: 1 = on       */
    int32_t  ref_free_slip;     /* regime 4 of apply_boundaries: 1 = on       */
    int32_t  ref_u_round;       /* enum lbm_u_round, default RTE              */
    /* physics mode: open x faces, [0] = x-, [1] = x+ (enum lbm_open) */
    int32_t  open_x[2];
    float    open_rho[2];       /* density of a PRESSURE face                */
} lbm_desc;

typedef struct lbm_info {
    uint32_t struct_size;
    int32_t  nx, ny, nz;
    int32_t  mode, precision;
    uint64_t iteration;          /* steps taken since the last init          */
    uint64_t device_bytes;       /* device memory the context owns           */
    double   bytes_per_node;     /* algorithmic HBM bytes of one node update */
    int32_t  layout;             /* 0 = two-buffer pull, 1 = esoteric pull   */
    int32_t  device;             /* CUDA ordinal                             */
} lbm_info;

/* Solver parameters that may change between lbm_step calls without touching
 * the flow state (lbm_get_params / lbm_set_params).  The reference rebuilds
 * CollideUniforms.tau_inv / omtau_inv and BoundariesUniforms.u_inf every frame
 * (src/main.cpp:1523-1537) from its tau and |u_inf| / angle-of-attack sliders
 * (src/main.cpp:1648, 1657-1661). */
typedef struct lbm_params {
    uint32_t struct_size;       /* sizeof(lbm_params)                        */
    float    tau;               /* relaxation time (> 0.5)                   */
    float    u_inf[3];          /* reference mode: inlet velocity            */
    float    body_accel[3];     /* physics mode: Guo force, F = rho * accel  */
    float    wall_velocity[6][3]; /* physics mode: per-face wall velocity
                                   (open x faces: the inlet velocity)        */
    float    smagorinsky_cs;    /* physics mode: 0 = off                     */
    float    trt_magic;         /* physics mode: TRT Lambda                  */
    float    open_rho[2];       /* physics mode: density of a PRESSURE face  */
} lbm_params;

typedef struct lbm_ctx lbm_ctx;

/* Fills *d with the reference defaults: 64^3, reference mode, fp32, BGK,
 * tau = TAU_DEFAULT 0.6 (src/main.cpp:84), rho0 = 1, all regimes on,
 * u rounding RTE, TRT Lambda 3/16, no force, resting walls. */
LBM_API int lbm_desc_default(lbm_desc* d);

/* Allocates a context on the current CUDA device.
 * Replaces allocate_tier_images (src/main.cpp:835-846) and the pipeline
 * creation that follows it.  The lattice starts all-fluid. */
LBM_API int lbm_create(const lbm_desc* desc, lbm_ctx** out);
LBM_API int lbm_destroy(lbm_ctx* ctx);

/* Uses `stream` (a cudaStream_t) for all later work; NULL = the context's
 * own stream. */
LBM_API int lbm_set_stream(lbm_ctx* ctx, void* stream);

/* Uploads the obstacle mask (uint8, Nx*Ny*Nz bytes, x-fastest; value 1 =
 * solid, any other value = fluid, as `mask_at(c) == 1u` in
 * shaders/apply_boundaries.comp.glsl:52-55,62) and classifies every node.
 * Replaces obstacle_mask.upload (src/main.cpp:1190, :1366). */
LBM_API int lbm_set_flags(lbm_ctx* ctx, const uint8_t* mask, size_t n);

/* lbm_set_flags with the NACA preset mask made on the device
 * (lbm_voxelize_naca_device into the context's mask, then classification):
 * the same mask and classification as lbm_set_flags of the host mask of
 * lbm_voxelize_naca with the context's Nx, Ny, Nz, without the host mask or
 * its upload.  Replaces the voxelize_into + obstacle_mask.upload pair of
 * apply_preset (src/main.cpp:1180-1190). */
LBM_API int lbm_set_flags_naca(lbm_ctx* ctx, const char* designation, float chord_frac,
                               float center_x_frac, float angle_of_attack_deg);

/* Reads the per-node classification word: bit 0 = node is solid; bit i
 * (1..18) = mask at x + c_i is solid, out-of-bounds counting as solid on
 * non-periodic axes (shaders/apply_boundaries.comp.glsl:52-55,76-79). */
LBM_API int lbm_read_classification(lbm_ctx* ctx, uint32_t* out, size_t n);

/* Equilibrium initialisation.  Replaces the init_equilibrium dispatch
 * (shaders/init_equilibrium.comp.glsl:35-47; src/main.cpp:1193-1206):
 * f_i = feq_i(rho0, u0) at every node, moments = (rho0, u0). */
LBM_API int lbm_init_equilibrium(lbm_ctx* ctx, float rho0, const float u0[3]);

/* Initialises f = feq(rho(x), u(x)) from host moment fields.  This is the
 * capture resume that the reference's F9 path intends (src/main.cpp:1359-
 * 1383) but does not do: its init shader ignores the uploaded moments.
 * u_fmt: LBM_U_F32X3, LBM_U_F32X4 or LBM_U_F16X4 (capture `velocity`). */
LBM_API int lbm_init_from_moments(lbm_ctx* ctx, const float* rho, const void* u,
                          int u_fmt);

/* Advances nsteps steps.  Replaces the substep dispatch chain
 * collide -> stream -> boundaries -> moments (src/main.cpp:1554-1591).
 * The moments of the last step are written for readback. */
LBM_API int lbm_step(lbm_ctx* ctx, int nsteps);

/* Physics mode: kernel variant of the step.  0 = automatic (two nodes per
 * thread when nx is even and the rows fill 64-wide warps, else one); 1, 2 or
 * 4 nodes per thread (4: nx % 4 == 0; one 16-byte access per slot quad for
 * fp32 storage, 8-byte for fp16/bf16); 8 = one node per
 * thread with the learned closure's hidden layer on the tensor cores (tcgen05;
 * without a closure the same as 1).  The 1-, 2- and 4-node variants agree bit
 * for bit except with a body force, where the one-node kernel's force terms
 * differ in the last place in a few per cent of values.  A tuning and testing
 * knob; LBM_ERR_UNSUPPORTED for a variant the grid or precision cannot use. */
LBM_API int lbm_set_step_variant(lbm_ctx* ctx, int nodes_per_thread);

/* The parameters in effect (from the descriptor, or the last lbm_set_params). */
LBM_API int lbm_get_params(lbm_ctx* ctx, lbm_params* params);

/* Changes the solver parameters between steps; populations, moments and the
 * step counter are kept.  Replaces the per-frame uniform upload of
 * src/main.cpp:1523-1537 driven by the sliders at :1648 and :1657-1661.
 * The new values apply from the next collision and the next boundary pass,
 * as a uniform upload before the next frame's dispatches does in the
 * reference.  Reference mode: the stored state between launches is the
 * post-collision population of the next step, so a tau change recomputes
 * that collision with the new tau (one extra launch; bit-identical to the
 * reference's four-pass step with the change made between frames).  After
 * lbm_write_populations or an lbm_set_flags since the last step, the pending
 * collision cannot be recomputed and keeps the old tau (the reference cannot
 * be in that state).  Reference mode accepts only tau and u_inf (the other
 * fields must equal the current ones); physics mode ignores u_inf.  The
 * validation rules of lbm_create apply; with a learned closure installed,
 * body_accel must stay 0 and smagorinsky_cs > 0. */
LBM_API int lbm_set_params(lbm_ctx* ctx, const lbm_params* params);

/* Waits for the context's stream; returns LBM_ERR_NONFINITE if a NaN/Inf or
 * non-positive density was seen at a fluid node since the last sync, and
 * LBM_ERR_TIMEOUT if a learned-closure step's bounded wait for its
 * tensor-core MMA gave up (those nodes used plain Smagorinsky). */
LBM_API int lbm_sync(lbm_ctx* ctx);

/* Copies rho (float[N]) and u (format u_fmt) to host memory; either pointer
 * may be NULL.  Solid nodes read rho = 0, u = 0
 * (shaders/compute_moments.comp.glsl:45-47).  Replaces the rho/velocity
 * Image::readback in capture_save and the VDB export (src/main.cpp:1290-
 * 1296, :1771-1779). */
LBM_API int lbm_read_moments(lbm_ctx* ctx, float* rho, void* u, int u_fmt);

/* Device pointers of the moment fields (rho float[N]; u float[3][N],
 * planes x, y, z) for on-device consumers.  Headless replacement of the
 * `velocity_image` texture bindings (src/main.cpp:1106-1114). */
LBM_API int lbm_device_moments(lbm_ctx* ctx, const float** d_rho, const float** d_u);

/* out[0] = sum rho, out[1..3] = sum rho*u over fluid nodes, in fp64. */
LBM_API int lbm_conservation(lbm_ctx* ctx, double out[4]);

/* lbm_conservation without the wait: queues the sums and their copy into
 * out (pinned host or device memory, four doubles) on the context's stream
 * and returns.  out holds the sums of the moments as they stand at this point
 * of the stream once the stream gets there (lbm_sync, or an event); it must
 * stay valid until then.  Lets a caller read every step's metric without
 * stalling the step pipeline.  No counterpart in the reference. */
LBM_API int lbm_conservation_async(lbm_ctx* ctx, double* out);

/* Full population state, natural layout float[19][N] (direction-major),
 * post-collision populations of the current step.  For checkpoints. */
LBM_API int lbm_read_populations(lbm_ctx* ctx, float* f, size_t n);
LBM_API int lbm_write_populations(lbm_ctx* ctx, const float* f, size_t n);
/* The same in physics mode as stored: g = f - w (fp32 values of the fp32,
 * fp16-shifted or bf16-shifted store), which round-trips bit for bit (f does
 * not: f - w + w is rounded).  Reference mode: LBM_ERR_UNSUPPORTED. */
LBM_API int lbm_read_populations_shifted(lbm_ctx* ctx, float* g, size_t n);
LBM_API int lbm_write_populations_shifted(lbm_ctx* ctx, const float* g, size_t n);

LBM_API int lbm_get_info(lbm_ctx* ctx, lbm_info* info);

/* Message of the last failed call on ctx (or on this thread if ctx is
 * NULL).  Never NULL. */
LBM_API const char* lbm_last_error(lbm_ctx* ctx);

/* Conservation sums of moment fields the caller already holds on the device
 * (d_rho float[n], d_u float[3][n] planes, e.g. from lbm_device_moments),
 * written to host out[4] as lbm_conservation does, but with no device
 * allocation at all.  This entry point has no counterpart in the reference.
 * It is for callers that may not allocate: a frame loop that cannot stall on
 * the device-wide synchronisation of cudaMalloc/cudaFree, or a host whose
 * memory arena owns the whole device budget.  Its scratch is a static
 * 131,104-byte device array that every GPU loading the library keeps until
 * exit; n is limited to 33,554,432 nodes (LBM_ERR_INVALID_ARG beyond).  Every
 * call looks the array's address up for the current device (no allocation).
 * All calls share the one array: calls that overlap on the GPU race.  Runs on
 * `stream` (NULL = the legacy default stream), copies the sums to pageable
 * host memory and synchronises the stream, so it cannot be called while that
 * stream (or the legacy stream) is being captured into a CUDA graph. */
LBM_API int lbm_conservation_noalloc(const float* d_rho, const float* d_u, size_t n,
                                     double out[4], void* stream);

/* The obstacle mask as last uploaded by lbm_set_flags (all zero = all fluid
 * before any upload).  Replaces obstacle_mask.readback in capture_save
 * (src/main.cpp:1296). */
LBM_API int lbm_read_mask(lbm_ctx* ctx, uint8_t* mask, size_t n);

/* The descriptor the context was created with, with the parameters of the
 * last lbm_set_params. */
LBM_API int lbm_get_desc(lbm_ctx* ctx, lbm_desc* desc);

/* Sets the step counter reported by lbm_get_info (a capture resume restores
 * the captured iteration, as capture_load does with rt.iteration,
 * src/main.cpp:1357). */
LBM_API int lbm_set_iteration(lbm_ctx* ctx, uint64_t iteration);

/* ---- capture directories ----------------------------------------------- */
/* The capture layout of the reference's F5 / F9 handlers
 * (src/main.cpp:1267-1390) and its StateWriter / StateReader
 * (common/common-cpp/src/state_writer.cpp:26-85, state_reader.cpp:12-85):
 * <root>/capture_%04u/state.json with {"frame", "meta": {"latticeBoltzmann":
 * {...}}, "buffers": [...]} and one raw <name>.bin per buffer:
 *   density        r32f     float[N]
 *   velocity       rgba16f  uint16 half[N][4], w = 0
 *   obstacle_mask  r8uint   uint8[N], "frame_invariant": true
 *   populations    r32f     float[19][N], shape [19, Nx, Ny, Nz],
 *                           post-collision f, or in physics mode f - w
 *                           ("values": "f - w" in its entry) (full-state
 *                           checkpoint; not in the reference, which cannot
 *                           resume exactly, docs/tier1-capture-format-
 *                           reference.md:124-134)
 * N = Nx*Ny*Nz, x fastest.  state.json is written as nlohmann's dump(2)
 * writes it (sorted keys, two-space indent). */
typedef struct lbm_capture_info {
    uint32_t struct_size;
    int32_t  nx, ny, nz;
    uint32_t frame;
    uint64_t iteration;            /* latticeBoltzmann.iteration, 0 if absent */
    int32_t  has_populations;
    int32_t  mask_frame_invariant;
} lbm_capture_info;

#define LBM_CAPTURE_LOAD_MASK    1  /* upload the captured obstacle mask      */
#define LBM_CAPTURE_MOMENTS_ONLY 2  /* ignore populations: f = feq(rho, u),
                                       the reference's F9 intent              */

/* Writes <root>/capture_<frame>/ from host arrays (no device needed).
 * meta_json: the latticeBoltzmann object as JSON text (NULL: a minimal one
 * with schemaVersion, Nx, Ny, Nz, iteration, substeps); pops may be NULL. */
LBM_API int lbm_capture_write(const char* root, uint32_t frame, const char* meta_json,
                              int32_t nx, int32_t ny, int32_t nz, const float* rho,
                              const uint16_t* vel, const uint8_t* mask, const float* pops);
/* Parses a capture directory; fills info and copies whichever buffers have a
 * non-NULL destination (sizes from info's dimensions).  LBM_ERR_IO for a
 * missing or malformed state.json, a missing required buffer or a file whose
 * size is not what its dimensions give. */
LBM_API int lbm_capture_read(const char* dir, lbm_capture_info* info, float* rho,
                             uint16_t* vel, uint8_t* mask, float* pops);
/* Lexicographically last capture_* directory under root (StateReader::
 * findLatest, state_reader.cpp:12-28), as a path in out[cap]. */
LBM_API int lbm_capture_latest(const char* root, char* out, size_t cap);
/* F5: reads the lattice's moments (rgba16f velocity), mask and, with
 * full_state, its populations, and writes a capture (meta_json as above;
 * NULL: the minimal meta with the context's iteration and tau). */
LBM_API int lbm_capture_save(lbm_ctx* ctx, const char* root, uint32_t frame,
                             const char* meta_json, int full_state);
/* F9: restores a capture into a lattice of the same dimensions: the mask
 * (with LBM_CAPTURE_LOAD_MASK), then the populations if the capture has them
 * (an exact resume) or else f = feq(rho, u) from the stored moments; the
 * iteration counter from the meta. */
LBM_API int lbm_capture_load(lbm_ctx* ctx, const char* dir, int flags);
LBM_API const char* lbm_capture_last_error(void);

/* ---- VDB export --------------------------------------------------------- */
/* The reference's optional VDB export (src/main.cpp:1767-1790) writes
 * vdb_export/velocity_%06u.vdb through gpusims::vdb::writeVec3Grid
 * (common/common-cpp/src/vdb_writer.cpp:96-141, which needs OpenVDB).  These
 * write the same grid in the OpenVDB file layout (format version 224) with no
 * OpenVDB dependency: a Vec3SGrid ("Tree_vec3s_5_4_3") named grid_name
 * (NULL: "velocity"), class "staggered", linear transform of voxel_size (a
 * translation by origin if origin is non-NULL and nonzero), every voxel of
 * the Nx x Ny x Nz box active and stored in a leaf, values uncompressed.
 * xyz: float[N][3], x-fastest.  LBM_ERR_IO when the file cannot be written;
 * lbm_vdb_last_error gives the message. */
LBM_API int lbm_vdb_write_vec3(const char* path, const float* xyz, int32_t nx, int32_t ny,
                               int32_t nz, float voxel_size, const float origin[3],
                               const char* grid_name);
#define LBM_VDB_F32 1  /* the fp32 velocity instead of its rgba16f rounding */
/* The frame-loop export: reads the lattice's velocity as the reference does
 * (rgba16f, then half -> float; with LBM_VDB_F32 the fp32 field itself) and
 * writes <dir>/velocity_<frame_idx, 6 digits>.vdb with voxel size 1 at the
 * origin, grid "velocity". */
LBM_API int lbm_vdb_export(lbm_ctx* ctx, const char* dir, uint32_t frame_idx, int flags);
LBM_API const char* lbm_vdb_last_error(void);

/* ---- streamlines ------------------------------------------------------- */
/* Streamline advection over the device velocity field, the reference's
 * streamline_advect compute pass (shaders/streamline_advect.comp.glsl:34-91,
 * dispatched from src/main.cpp:1596-1623) without the draw.  Positions are
 * float4 (x, y, z, age) in lattice units, `history` per streamline in a
 * ring (streamline s, slot h at s*history + h); domain [0, N] per axis.
 * Per call and streamline: read slot (head_index - 1) mod history; if its
 * age >= reseed_age or it left the domain, reseed it into the inlet slab
 * x in [Nx/16, Nx/8] (xorshift32 seeded by s*2654435761 ^ frame*1597334677)
 * and fill every slot; else take one RK2 step of dt_render with trilinear,
 * clamp-to-edge velocity (texel centres at i + 1/2; fp32 with every
 * operation rounded on its own; u rounded to binary16 first when round_f16,
 * as the rgba16f image holds it) and write slot head_index.  The caller
 * advances head_index = (head_index + 1) mod history after each call, as
 * src/main.cpp:1621 does.  d_u: float[3][N] planes (lbm_device_moments);
 * d_positions 16-byte aligned. */
LBM_API int lbm_streamline_advect(const float* d_u, int32_t nx, int32_t ny, int32_t nz,
                                  float* d_positions, uint32_t count, uint32_t history,
                                  uint32_t head_index, uint32_t frame_count, float dt_render,
                                  uint32_t reseed_age, int32_t round_f16, void* stream);
/* Host seeding of the ring (src/main.cpp:1126-1152): std::mt19937(seed) and
 * std::uniform_real_distribution<float>(0, 1); per streamline an initial age
 * u*reseed_age, then x in [Nx/16, Nx/8], y in [0, Ny], z in [0, Nz]; every
 * slot holds the seed.  The reference uses seed 12345, reseed_age 256,
 * count 10000, history 64. */
LBM_API int lbm_streamline_seed(float* positions, uint32_t count, uint32_t history,
                                int32_t nx, int32_t ny, int32_t nz, uint32_t seed,
                                uint32_t reseed_age);

/* ---- velocity-magnitude raymarch ---------------------------------------- */
/* The reference's velmag volume pass (shaders/velmag.frag.glsl:44-96, drawn
 * by src/main.cpp:1720-1740) into a headless float RGBA buffer
 * d_rgba[height][width][4] (row 0 at the top), no graphics API: per pixel a
 * ray from camera_pos through the far-plane point of its fragment
 * (inv_view_proj applied to ((px+1/2)/W*2-1, (py+1/2)/H*2-1, 1, 1)),
 * clipped to the volume box, `steps` samples with blue-noise jitter (the
 * reference's 256x256 LCG jitter LUT, src/main.cpp:565-573), |u| mapped to
 * [velmag_min, velmag_max] and the colour LUT (src/main.cpp:529-563),
 * front-to-back emission-absorption; alpha = 1 - transmittance.  Samplers,
 * sqrt and exp are evaluated with separately rounded fp32 operations (see
 * gpu-sims_b200/csrc/render.cu). */
typedef struct lbm_velmag_params {
    uint32_t struct_size;
    float    inv_view_proj[16];   /* column-major, as glm::mat4 in memory   */
    float    camera_pos[3];
    float    volume_min[3];       /* default (0, 0, 0)                      */
    float    volume_max[3];       /* default (-1, -1, -1) = (Nx, Ny, Nz)    */
    int32_t  steps;               /* raymarchSteps, default 128             */
    float    absorption;          /* velmagAbsorption, default 4            */
    float    velmag_min;          /* default 0                              */
    float    velmag_max;          /* default 0.1 (presets: 1.5 |u_inf|)     */
    float    exposure;            /* default 1.5                            */
    int32_t  round_f16;           /* sample u rounded to binary16 (rgba16f) */
} lbm_velmag_params;

LBM_API int lbm_velmag_params_default(lbm_velmag_params* p);
LBM_API int lbm_render_velmag(const float* d_u, int32_t nx, int32_t ny, int32_t nz,
                              const lbm_velmag_params* p, int32_t width, int32_t height,
                              float* d_rgba, void* stream);
/* The reference's LUTs (host): colour rgba8 [4][256][4] (build_colormap_lut,
 * src/main.cpp:529-563) and jitter r8 [256][256] (build_jitter_lut,
 * src/main.cpp:565-573). */
LBM_API int lbm_colormap_lut(uint8_t* out);
LBM_API int lbm_jitter_lut(uint8_t* out);

/* ---- batched ensemble --------------------------------------------------- */
/* Hundreds of independent physics-mode domains of uneven size advanced
 * together: one launch per step over a tile work-list (captured in a CUDA
 * graph), or one persistent cooperative launch per lbm_batch_step call.  The
 * reference runs one domain at a time (src/main.cpp:1554-1591); a batch is
 * equivalent to lbm_step on each domain alone, bit for bit. */
typedef struct lbm_batch lbm_batch;

typedef struct lbm_batch_schedule {
    uint32_t struct_size;
    int32_t  rows_per_block;      /* 1, 2, 4, 8: a block is 32 x rows threads */
    int32_t  z_per_thread;        /* 1..16 nodes along z per thread           */
    int32_t  persistent;          /* 1 = one cooperative launch per call      */
    int64_t  spin_limit_cycles;   /* bound of a grid-barrier wait (persistent)*/
    int32_t  test_missing_blocks; /* testing only: barrier waits for this many
                                     blocks that never arrive -> TIMEOUT      */
} lbm_batch_schedule;

typedef struct lbm_batch_info {
    uint32_t struct_size;
    int32_t  domains;
    uint64_t total_nodes;
    uint32_t tiles;
    int32_t  grid;                /* persistent grid size (0 in graph mode)   */
    uint64_t iteration;
    uint64_t device_bytes;
    double   bytes_per_node;
} lbm_batch_info;

LBM_API int lbm_batch_schedule_default(lbm_batch_schedule* s);
/* All descriptors: physics mode, one precision and collision for all, no
 * Smagorinsky term, no body force.  Domains start all-fluid. */
LBM_API int lbm_batch_create(const lbm_desc* descs, int n, lbm_batch** out);
LBM_API int lbm_batch_destroy(lbm_batch* b);
LBM_API int lbm_batch_set_stream(lbm_batch* b, void* stream);
LBM_API int lbm_batch_set_flags(lbm_batch* b, int domain, const uint8_t* mask, size_t n);
/* domain = -1 initialises every domain. */
LBM_API int lbm_batch_init_equilibrium(lbm_batch* b, int domain, float rho0, const float u0[3]);
LBM_API int lbm_batch_init_from_moments(lbm_batch* b, int domain, const float* rho,
                                        const void* u, int u_fmt);
LBM_API int lbm_batch_step(lbm_batch* b, int nsteps);
/* LBM_ERR_NONFINITE as lbm_sync; LBM_ERR_TIMEOUT if a persistent launch's
 * grid barrier gave up (the domains then need a new init). */
LBM_API int lbm_batch_sync(lbm_batch* b);
LBM_API int lbm_batch_read_moments(lbm_batch* b, int domain, float* rho, void* u, int u_fmt);
LBM_API int lbm_batch_read_populations(lbm_batch* b, int domain, float* f, size_t n);
LBM_API int lbm_batch_set_schedule(lbm_batch* b, const lbm_batch_schedule* s);
LBM_API int lbm_batch_get_schedule(lbm_batch* b, lbm_batch_schedule* s);
/* Times every schedule (rows 2/4/8 x z 1/2/4 x graph/persistent) for
 * trial_steps steps, keeps the fastest and restores the populations.  Results
 * are cached per (precision, collision, size class) for the process and, if
 * $LBM_AUTOTUNE_CACHE names a file, across processes. */
LBM_API int lbm_batch_autotune(lbm_batch* b, int trial_steps, lbm_batch_schedule* best);
LBM_API int lbm_batch_get_info(lbm_batch* b, lbm_batch_info* info);
LBM_API const char* lbm_batch_last_error(lbm_batch* b);

/* ---- host-side helpers (no GPU needed) --------------------------------- */

/* D3Q19 tables in the reference's direction order
 * (shaders/lattice_constants.glsl:23-75): c[19][3], w[19], opp[19]. */
LBM_API int lbm_lattice_tables(int32_t* c, float* w, int32_t* opp);

/* NACA 4-digit airfoil voxeliser, extruded in z.  Restates
 * naca::voxelize_into (src/main.cpp:254-312) with the preset geometry of
 * apply_preset (src/main.cpp:1180-1190): chord = chord_frac*Nx, leading edge
 * at (center_x_frac*Nx - chord/2, Ny/2). */
LBM_API int lbm_voxelize_naca(const char* designation, int32_t nx, int32_t ny,
                      int32_t nz, float chord_frac, float center_x_frac,
                      float angle_of_attack_deg, uint8_t* mask, size_t n);

/* The same mask as lbm_voxelize_naca, produced on the device: the perimeter
 * is built on the host as lbm_voxelize_naca builds it, and the winding test of
 * every (x, y) column runs in a kernel on `stream` (a cudaStream_t; NULL = the
 * legacy default stream), writing all n = Nx*Ny*Nz bytes of the device buffer
 * d_mask.  Asynchronous; bit-identical to the host voxeliser.  Replaces
 * naca::voxelize_into (src/main.cpp:254-312) where the mask goes to the GPU. */
LBM_API int lbm_voxelize_naca_device(const char* designation, int32_t nx, int32_t ny,
                      int32_t nz, float chord_frac, float center_x_frac,
                      float angle_of_attack_deg, uint8_t* d_mask, size_t n,
                      void* stream);

/* binary16 -> binary32, as half_to_float (src/main.cpp:320-337). */
LBM_API int lbm_half_to_float(const uint16_t* h, float* f, size_t n);

/* Library build string (compiler, arch, ABI version). */
LBM_API const char* lbm_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
