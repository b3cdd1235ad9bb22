/*
 * slosh_b200.h — C ABI of the B200-native slosh MPM substep.
 *
 * The library replaces the device side of slosh's `MpmPipeline::launch_step`
 * (src/pipeline.rs:562-770 in dimforge/slosh): the sparse hashed grid build,
 * the APIC/MLS P2G scatter, the grid velocity update with collider boundary
 * conditions, the G2P gather fused with the particle update and constitutive
 * models, and the rigid-body integration pass.  All entry points are plain C:
 * pointers, sizes and status codes, no C++ or torch types.
 *
 * Conventions
 *  - Every function returns SLOSH_OK (0) or a negative SLOSH_E_* status.  The
 *    text of the last error of a context is available from slosh_last_error.
 *  - A context owns all of its device memory.  A context must not be used
 *    from two host threads at once (it mirrors `&mut MpmData`).
 *  - `stream` arguments are `cudaStream_t` values passed as `void*`; NULL
 *    means the context's own stream.
 *  - Matrices in the particle records are column-major 3x3 (glam `Mat3`), the
 *    layout slosh uploads and reads back.  In 2D only the top-left 2x2 block
 *    (elements 0, 1, 3, 4) is used.
 */
#ifndef SLOSH_B200_H
#define SLOSH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SLOSH_OK 0
#define SLOSH_E_INVALID (-1)   /* bad argument or record                  */
#define SLOSH_E_CUDA (-2)      /* a CUDA call failed                      */
#define SLOSH_E_OVERFLOW (-3)  /* block hash map / block list overflowed  */
#define SLOSH_E_CAPACITY (-4)  /* particle, body or material capacity     */
#define SLOSH_E_NOMEM (-5)     /* device allocation failed                */
#define SLOSH_E_STATE (-6)     /* call out of order (e.g. no particles)   */
#define SLOSH_E_MATERIAL (-7)  /* too many distinct materials             */
#define SLOSH_E_TIMEOUT (-8)   /* a bounded device-side wait gave up      */

/* ---- particle models: GpuParticleModel discriminants ------------------- */
/* src/solver/particle_model.rs:89-98; shaders/slosh/models/default.slang:73-80 */
#define SLOSH_MODEL_ELASTIC_LINEAR 0u      /* fixed-corotated (ElasticCoefficients) */
#define SLOSH_MODEL_ELASTIC_NEO_HOOKEAN 1u
#define SLOSH_MODEL_SAND_LINEAR 2u         /* Drucker-Prager + fixed-corotated  */
#define SLOSH_MODEL_SAND_NEO_HOOKEAN 3u
/* Extension through slosh's IParticleModel seam (ModelFlags::FLUID,
 * shaders/slosh/models/interfaces.slang:22-25): weakly compressible Tait
 * fluid.  data[0] = rest density, data[1] = bulk modulus K, data[2] = gamma.
 * Kirchhoff stress tau = -J p I with p = (K/gamma) (J^-gamma - 1) and
 * J = F[0][0] (the FLUID update keeps F = F00 I). */
#define SLOSH_MODEL_FLUID_TAIT 4u

/* 52-byte model record, byte-compatible with slosh's GpuParticleModel
 * (src/solver/particle_model.rs:102).  Payload words:
 *   ELASTIC_*: lambda, mu, cfl_coeff, 9 x 0
 *   SAND_*:    plastic det, plastic hardening q, log_vol_gain,
 *              h0, h1, h2, h3, plastic lambda, plastic mu,
 *              elastic lambda, elastic mu, cfl_coeff
 *   FLUID_TAIT: rest density, bulk modulus, gamma, 9 x 0 */
typedef struct slosh_model {
    uint32_t tag;
    float data[12];
} slosh_model;

/* One particle, the flattened form of slosh's `Particle<ParticleModel>`
 * (src/solver/particle.rs:23-55, :226-233).  192 bytes. */
typedef struct slosh_particle {
    float position[3];
    float velocity[3];
    float def_grad[9]; /* column-major */
    float affine[9];   /* column-major APIC affine matrix C */
    float force_dt[3];
    float vel_grad_det;
    float init_volume;
    float init_radius;
    float mass;
    float damping;
    float phase;
    uint32_t enabled;
    uint32_t fixed;
    slosh_model model;
} slosh_particle;

/* Collider shape types: shaders/slosh/rbd/shapes/shape.slang:19-25. */
#define SLOSH_SHAPE_BALL 0u
#define SLOSH_SHAPE_CUBOID 1u
#define SLOSH_SHAPE_CAPSULE 2u   /* 2D and 3D */
#define SLOSH_SHAPE_CONE 3u      /* 3D, axis along local y */
#define SLOSH_SHAPE_CYLINDER 4u  /* 3D, axis along local y */
#define SLOSH_SHAPE_TRIMESH 6u   /* 3D triangle mesh, made by slosh_add_trimesh */

/* Boundary conditions: src/solver/boundary_condition.rs:14-19. */
#define SLOSH_BC_STICK 0u
#define SLOSH_BC_SLIP 1u
#define SLOSH_BC_SEPARATE 2u
#define SLOSH_BC_FRICTION_Z_UP 3u
#define SLOSH_BC_NON_REFLECTING 4u
#define SLOSH_BC_DISABLED 5u

/* Body coupling (BodyCoupling, src/rbd/dynamics/body.rs:124-138).
 * ONE_WAY: the reference's behaviour on the GPU.  The body moves by its own
 *   velocity (plus gravity when it has inverse mass); the particles never
 *   push it, and the grid reuses cached collisions (colliders assumed still).
 * TWO_WAY: the grid pushes back.  Each grid node projected by the body's
 *   boundary condition is projected in the body's frame (the node velocity
 *   relative to the body velocity at the node), and the momentum the node
 *   loses is added to the body as an impulse at the node: linear and angular
 *   sums in 64-bit fixed point (2^-40 N s), so the total does not depend on
 *   the order of the additions.  The rigid update applies the impulse with
 *   the body's inverse mass and world inverse inertia and caps the velocities
 *   as rigid_impulses.slang:72-121 does.  While any body is TWO_WAY the grid
 *   runs collision detection on every node instead of the cache.  slosh
 *   declares the impulse buffer (rigid_impulses.slang:8-52) but no kernel of
 *   it fills the buffer, so this mode has no reference output to match; the
 *   oracle restates it for the parity tests. */
#define SLOSH_COUPLING_ONE_WAY 0u
#define SLOSH_COUPLING_TWO_WAY 1u

/* One rigid body with its collider shape and boundary condition: an entry of
 * slosh's GpuBodySet (src/rbd/dynamics/body.rs:74-90) plus its
 * GpuBoundaryCondition (src/solver/boundary_condition.rs:8-12).  192 bytes.
 * Shape layout as shaders/slosh/rbd/shapes/shape.slang:44-62:
 *   ball:     shape_a = (radius, -, -, type)
 *   cuboid:   shape_a = (hx, hy, hz, type)
 *   capsule:  shape_a = (ax, ay, az, type), shape_b = (bx, by, bz, radius):
 *             the segment a-b inflated by the radius
 *   cone, cylinder: shape_a = (half_height, radius, -, type); a cone's apex
 *             is at +half_height, its base disc at -half_height
 *   trimesh:  shape_a = (vertex offset, index offset, BVH nodes, type),
 *             shape_b = (triangles, vertices, mesh ordinal, -), all uint32
 *             bits, as slosh_add_trimesh writes them
 * where `type` is the shape type stored as uint32 bits.  The pose is a
 * similarity: rotation (3D unit quaternion i,j,k,w; 2D cos,sin), translation
 * xyz and uniform scale in translation[3].  Bodies coupled one-way (the
 * MpmData::new default, src/pipeline.rs:328) carry zero inverse mass. */
typedef struct slosh_body {
    float shape_a[4];
    float shape_b[4];
    float rotation[4];
    float translation[4];
    float linvel[4];
    float angvel[4];
    float inv_mass[4];
    float local_com[4];
    float inv_inertia[12]; /* world-space inverse inertia at this pose, 3 padded
                              columns (2D: the scalar in [0]) */
    uint32_t bc_type;
    float bc_friction;
    uint32_t coupling;     /* SLOSH_COUPLING_* */
    uint32_t pad;
} slosh_body;

/* Context creation parameters: the arguments of MpmData::new that size the
 * device state (src/pipeline.rs:311-320). */
typedef struct slosh_config {
    uint32_t dim;           /* 2 or 3 */
    float cell_width;       /* grid spacing h */
    uint32_t grid_capacity; /* max active blocks; the block hash map holds
                               2 x next_pow2(grid_capacity) slots */
    uint32_t max_particles;
    int32_t device;         /* CUDA device ordinal */
    uint32_t flags;         /* reserved, 0 */
} slosh_config;

/* SimulationParams (src/solver/params.rs:13-21). */
typedef struct slosh_params {
    float gravity[3];
    float dt;
} slosh_params;

typedef struct slosh_ctx slosh_ctx;

/* Creates the device state of one scene.  Replaces MpmData::new and
 * MpmPipeline::new_with_kernels (src/pipeline.rs:311, :462). */
int slosh_ctx_create(const slosh_config *cfg, slosh_ctx **out);

/* Frees every device buffer of the context. */
void slosh_ctx_destroy(slosh_ctx *ctx);

/* Sets gravity and dt.  Replaces GpuSimulationParams::new
 * (src/solver/params.rs:40-49). */
int slosh_set_params(slosh_ctx *ctx, const slosh_params *params);

/* Uploads `n` particles from HOST memory (pinned memory gives full PCIe
 * speed) and converts them to the device layout.  Replaces
 * GpuParticles::from_particles (src/solver/particle.rs:474-500).  Particle
 * models are deduplicated into a per-context material table on the device. */
int slosh_upload_particles(slosh_ctx *ctx, const slosh_particle *particles,
                           uint32_t n, void *stream);

/* Appends `n` particles from HOST memory behind the current ones; they take
 * the insertion-order indices [old count, old count + n).  Replaces
 * GpuParticles::append (src/solver/particle.rs:536-572). */
int slosh_append_particles(slosh_ctx *ctx, const slosh_particle *particles,
                           uint32_t n, void *stream);

/* Removes the particles with insertion-order indices [start, start + count)
 * (clamped to the current count); later particles move down to close the
 * gap.  `*removed` receives the number removed.  Replaces
 * GpuParticles::shift_remove (src/solver/particle.rs:505-534). */
int slosh_remove_particles(slosh_ctx *ctx, uint32_t start, uint32_t count,
                           uint32_t *removed, void *stream);

/* Reads the particles back into the record layout above (in upload order).
 * Replaces the staging readbacks of src_testbed/step.rs:260-334.
 * `vel_grad_det` is transient inside the fused G2P/update and reads as 0. */
int slosh_download_particles(slosh_ctx *ctx, slosh_particle *out, uint32_t n,
                             void *stream);

/* Reads positions back as vec4 (x, y, z, 0), the layout of slosh's position
 * buffer (src/solver/particle.rs:384-389). */
int slosh_download_positions(slosh_ctx *ctx, float *out_xyzw, uint32_t n,
                             void *stream);

/* Sets the rigid bodies and their colliders (<= 16).  Replaces
 * GpuBodySet::from_rapier + GpuMaterials::new (src/rbd/dynamics/body.rs:183;
 * src/solver/boundary_condition.rs:76-85). */
int slosh_set_bodies(slosh_ctx *ctx, const slosh_body *bodies, uint32_t n);

/* Reads the bodies back (poses and velocities after integration). */
int slosh_get_bodies(slosh_ctx *ctx, slosh_body *out, uint32_t n);

/* Adds a triangle-mesh collider shape (3D).  Replaces GpuShape::from_parry
 * for a TriMesh with convert_trimesh_to_gpu (src/rbd/shapes.rs:231-239;
 * src/trimesh.rs:23-103): builds the mesh's BVH and its vertex and edge
 * pseudo-normals, appends them to the context's mesh buffers and writes the
 * trimesh shape into body->shape_a / shape_b; the pose, velocities, mass and
 * boundary condition of `body` are the caller's.  `vertices` holds x, y, z a
 * vertex; `indices` three vertex indices a triangle, counter-clockwise seen
 * from outside.  Heightfields are passed as their triangle meshes, as slosh
 * converts them (src/rbd/shapes.rs:241-269).  The grid update projects a node
 * on the mesh only within 1.5 cells of its surface (collide.slang:124-134). */
int slosh_add_trimesh(slosh_ctx *ctx, const float *vertices, uint32_t n_vertices, const uint32_t *indices,
                      uint32_t n_triangles, slosh_body *body);

/* Enqueues `n_substeps` substeps on `stream` without any host round trip.
 * Replaces MpmPipeline::launch_step (src/pipeline.rs:562-770) called
 * n_substeps times into one encoder.  Asynchronous: errors raised on the
 * device are reported by slosh_sync.
 * Grid reuse: slosh rebuilds the sparse grid every substep
 * (src/grid/grid.rs:78-238).  Here a substep keeps the previous substep's
 * blocks, ranks and hash map when no particle left the set of blocks that
 * hold particles, and only re-counts the cells particles entered or left;
 * the decision is taken on the device.  The layout is the one a full build
 * gives, bit for bit.  Scenes of at least 262,144 particles keep their grid
 * this way; smaller ones are launch-bound, and the full build inside the
 * substep graph is faster for them.  The environment variable
 * SLOSH_GRID_REUSE at context creation overrides that: 0 makes every
 * substep run the full build, 1 keeps grids at any size. */
int slosh_step(slosh_ctx *ctx, uint32_t n_substeps, void *stream);

/* ---- stage hooks ------------------------------------------------------------
 * slosh's MpmPipelineHooks (src/pipeline.rs:146-238): callbacks at fixed
 * points of launch_step (src/pipeline.rs:562-770).  A hook runs on the host
 * thread inside slosh_step, once per substep, at the point the substep's
 * kernels have been enqueued up to; it may enqueue its own device work on
 * `stream` (a cudaStream_t), which then runs in order with the substep.  It
 * returns 0, or a negative status that stops slosh_step with that status;
 * the run hooks may return 1 instead, meaning "I replaced this stage", as
 * slosh's run_p2g / run_g2p return Ok(true).  While any hook is set, the
 * substeps are launched kernel by kernel instead of as CUDA graphs.
 *  AFTER_PARTICLE_SORT  after the grid build (the sort of particles by block)
 *  RUN_P2G              replaces P2G: the hook writes the P2G result of every
 *                       node of the active blocks, (momentum, mass) in the
 *                       view's `nodes`; the grid update then reads them
 *  AFTER_P2G            after P2G; the view's `nodes` hold (momentum, mass)
 *  AFTER_GRID_UPDATE    after the grid update; `nodes` hold (velocity, mass)
 *  RUN_G2P              replaces the G2P gather fused with the particle
 *                       update (slosh's g2p and particles_update passes): the
 *                       hook writes every particle's next state into the
 *                       view's out_* planes at its canonical position
 *  AFTER_G2P            after the fused G2P / particle update
 *  AFTER_PARTICLES_UPDATE  after AFTER_G2P, before the rigid-body update
 * The G2P gather and the particle update are one kernel here, so AFTER_G2P
 * and AFTER_PARTICLES_UPDATE both follow it. */
#define SLOSH_HOOK_AFTER_PARTICLE_SORT 0u
#define SLOSH_HOOK_RUN_P2G 1u
#define SLOSH_HOOK_AFTER_P2G 2u
#define SLOSH_HOOK_AFTER_GRID_UPDATE 3u
#define SLOSH_HOOK_RUN_G2P 4u
#define SLOSH_HOOK_AFTER_G2P 5u
#define SLOSH_HOOK_AFTER_PARTICLES_UPDATE 6u
#define SLOSH_HOOK_COUNT 7u

typedef int (*slosh_hook_fn)(slosh_ctx *ctx, uint32_t point, void *stream, void *user);

/* Sets (fn != NULL) or clears the hook of `point`.  `user` is passed back
 * to the hook (slosh's hooks_state). */
int slosh_set_hook(slosh_ctx *ctx, uint32_t point, slosh_hook_fn fn, void *user);

/* Enqueues on `stream` the built-in stage that run hook `point` replaces
 * (SLOSH_HOOK_RUN_P2G: P2G with its node sums written to the view's
 * `nodes`; SLOSH_HOOK_RUN_G2P: the fused G2P / particle update), so a
 * replacing hook can wrap the built-in stage with work of its own.  Only
 * valid inside that hook; the results are those of the built-in substep,
 * bit for bit. */
int slosh_enqueue_builtin(slosh_ctx *ctx, uint32_t point, void *stream);

/* Device buffers of the substep a hook runs in (valid inside a hook).
 * Particle storage is in the canonical order of this substep's grid: block
 * b's particles are perm[block_first[b] .. + block_count[b]), storage
 * indices of the input planes.  Planes (capacity entries each): x_mass
 * float4 (x, y, z, mass); vel float4 (vx, vy, vz, C22); affine and def_grad
 * two float4 planes each, row-major matrix elements 0-7 (2D: one plane,
 * elements 0-3); flags uint4 (flags, original index, V0 bits, F22 bits);
 * plastic float4 (plastic det, hardening q, log_vol_gain, damping).
 * The out_* planes are the next substep's storage, written by the fused
 * G2P / particle update at the canonical index.  nodes: 64 float4 a block,
 * node id = block * 64 + local index (grid.slang:409-417). */
typedef struct slosh_device_view {
    uint32_t dim, n_particles, capacity, grid_capacity;
    float cell_width, dt;
    uint32_t pad[2];
    const uint32_t *n_blocks;  /* device word: active blocks of the substep */
    const uint32_t *block_keys, *block_first, *block_count, *perm;
    void *x_mass, *vel, *affine, *def_grad, *flags, *plastic;
    void *out_x_mass, *out_vel, *out_affine, *out_def_grad, *out_flags, *out_plastic;
    void *nodes;
} slosh_device_view;

int slosh_device_view_get(slosh_ctx *ctx, slosh_device_view *out);

/* Waits for the context's work and returns the device error status
 * (SLOSH_E_OVERFLOW when the block hash map or block list overflowed). */
int slosh_sync(slosh_ctx *ctx, void *stream);

/* Number of device kernels a substep launches that runs the full grid
 * build (for launch accounting).  With grid reuse and conditional graphs a
 * substep that keeps the previous grid launches 7 fewer: the reuse's
 * permutation update and touched-cell gather instead of the 9 build
 * kernels (slosh_get_stats counts both kinds of substep). */
uint32_t slosh_kernels_per_substep(const slosh_ctx *ctx);

/* Runs `n_substeps` substeps with direct launches (not the CUDA graph) and a
 * pair of CUDA events around every kernel, and writes the summed device time
 * of each kernel in milliseconds to kernel_ms[0 .. *n_kernels).  Kernel names
 * come from slosh_kernel_name.  Stands in for slosh's per-pass
 * GpuTimestamps (src/pipeline.rs:588-757); advances the simulation like
 * slosh_step and synchronises after every substep. */
int slosh_profile_substeps(slosh_ctx *ctx, uint32_t n_substeps, void *stream,
                           float *kernel_ms, uint32_t cap, uint32_t *n_kernels);

/* Name of profiled kernel `index`. */
int slosh_kernel_name(uint32_t index, char *buf, size_t len);

/* Counters of the last completed substep (synchronises the context). */
typedef struct slosh_stats {
    uint32_t n_particles;
    uint32_t n_blocks;         /* active blocks of the last substep */
    uint32_t n_primary_blocks; /* blocks holding at least one particle */
    uint32_t n_materials;      /* distinct particle models */
    uint32_t n_svd_fp64;       /* SVDs recomputed in FP64 since upload */
    uint32_t n_grid_rebuilds;  /* substeps that ran the full grid build   */
    uint32_t n_grid_reuses;    /* substeps that kept the previous grid    */
    uint32_t conditional_graphs; /* 1: the substep graphs launch only the
                                    selected grid-build branch            */
} slosh_stats;

int slosh_get_stats(slosh_ctx *ctx, slosh_stats *out);

/* Grid-build result of the current positions, computed without advancing
 * the simulation (bit-exactness checks).  Blocks are in canonical order
 * (ascending packed key).  Two views are returned:
 *  - the hot path's own arrays: per block the first primary entry and the
 *    canonical permutation of primaries, ordered by (slab bucket, id);
 *  - slosh's complete layout (shaders/slosh/grid/sort.slang:248-357):
 *    per-block counts of all NB buckets, first_particle over primaries and
 *    extras, and the sorted ids with extras, each bucket ordered by id.
 * Any output pointer may be NULL.  Sizes are reported in the struct; arrays
 * must hold cap_blocks blocks (x NB or x (NASSOC-1) where noted), n
 * particles and cap_sorted entries. */
typedef struct slosh_grid_dump {
    uint32_t n_blocks;       /* out */
    uint32_t n_sorted;       /* out: entries of the full layout */
    uint32_t nb_buckets;     /* out: NB (10 in 3D, 18 in 2D) */
    uint32_t n_neighbors;    /* out: NASSOC - 1 (7 in 3D, 3 in 2D) */
    uint32_t *keys;          /* [cap_blocks] packed keys, ascending */
    uint32_t *first_particle;            /* [cap_blocks] full layout */
    uint32_t *num_particles;             /* [cap_blocks] primaries */
    uint32_t *num_particles_with_extras; /* [cap_blocks] */
    uint32_t *bucket_counts; /* [cap_blocks * NB] */
    uint32_t *sorted_ids;    /* [cap_sorted] full layout */
    uint32_t *primary_first; /* [cap_blocks] hot path */
    uint32_t *primary_perm;  /* [n particles] hot path */
    uint32_t *neighbors;     /* [cap_blocks * (NASSOC-1)] neighbour ranks */
} slosh_grid_dump;

int slosh_grid_debug(slosh_ctx *ctx, slosh_grid_dump *dump,
                     uint32_t cap_blocks, uint32_t cap_sorted);

/* Runs one substep's grid build followed by P2G (stage 1) or by P2G and the
 * grid update (stage 2) without advancing the particles, and copies the
 * nodes out: 64 nodes per block in canonical block order, 4 floats each
 * (momentum or velocity, mass).  Node id = block * 64 + local index as in
 * shaders/slosh/grid/grid.slang:409-417. */
int slosh_debug_nodes(slosh_ctx *ctx, int stage, float *nodes,
                      uint32_t cap_blocks, uint32_t *n_blocks);

/* Exclusive prefix sum of `n` u32 values (host arrays) with slosh's
 * semantics (src/grid/prefix_sum.rs:97-110: the result is as if a 0 had been
 * prepended; the total is dropped).  Uses the context's scan workspace;
 * n <= grid_capacity. */
int slosh_prefix_sum(slosh_ctx *ctx, const uint32_t *in, uint32_t *out,
                     uint32_t n);

/* Allocation-free variant of slosh_prefix_sum for callers that cannot
 * allocate device memory where they need the scan (hosts that own every
 * allocation up front, real-time loops, code inside another framework's
 * memory pool).  This entry point has no counterpart in the reference.
 *  - d_in, d_out: DEVICE arrays of n u32 on the current device, not aliased;
 *    same result as slosh_prefix_sum (exclusive scan, total dropped).
 *  - n <= 67,108,864 (16384 tiles of 4096); larger n returns
 *    SLOSH_E_CAPACITY without launching anything.
 *  - Scratch: a 64 KiB file-scope __device__ array that every GPU loading
 *    the library holds until exit.  It allocates nothing: no cudaMalloc,
 *    cudaFree or allocating library call.  Every call looks up the array's
 *    device address (cudaGetSymbolAddress) in the current context, so a
 *    device reset or a context switch between calls is safe; make the first
 *    call on a device before any stream capture.
 *  - Returns SLOSH_E_CUDA without launching while an earlier CUDA error is
 *    pending on the calling thread, and leaves that error for its owner.
 *  - Every call shares the scratch array: calls that overlap on the GPU
 *    (other streams, other host threads) race and must be serialised by the
 *    caller.  Nothing in the scratch needs to start at zero.
 *  - Asynchronous on `stream` (a cudaStream_t, NULL = legacy default). */
int slosh_prefix_sum_noalloc(const uint32_t *d_in, uint32_t *d_out, uint32_t n,
                             void *stream);

/* Largest stable timestep of the current particles, in seconds, for
 * adaptive substepping: per enabled particle the model's sound-speed bound
 * CFL * h / max(|v|, c) and the velocity bound h / |v|, quantised to whole
 * picoseconds (u32, saturating at ~4.29e-3 s), minimum over particles.
 * Replaces WgTimestepBounds::compute_bounds (src/solver/timestep_bound.rs:58-81;
 * shader shaders/slosh/solver/timestep_bound.slang:37-91).  Synchronous. */
int slosh_timestep_bound(slosh_ctx *ctx, float *dt_out, void *stream);

/* Copies the last error message of the context into `buf`. */
int slosh_last_error(const slosh_ctx *ctx, char *buf, size_t len);

/* ---- Multi-scene batches -------------------------------------------------
 * Many independent scenes, each with its own particles, cell width, dt,
 * gravity and colliders, advance together: a substep launches every kernel
 * once over the blocks and particles of all live scenes, as one CUDA graph.
 * Stepping a batch by k substeps is equivalent to calling
 * MpmPipeline::launch_step (src/pipeline.rs:562-770) k times on each
 * scene's own MpmData (src/pipeline.rs:311); the reference has no batched
 * step.  Each scene is sorted and reduced exactly as it would be alone (its
 * blocks are ranked scene-major, ascending key within the scene, and P2G
 * reduces in a fixed order), so a scene's results do not depend on the other
 * scenes in the batch, bit for bit.  External forces (force_dt) are not
 * supported in batches.  Scenes may be added and removed between steps
 * (continuous batching); a removed scene's particles leave storage at the
 * next substep and its slot is reusable after that substep. */
typedef struct slosh_batch slosh_batch;

typedef struct slosh_batch_config {
    int32_t dim;             /* 2 or 3, for every scene                     */
    uint32_t max_particles;  /* particle pool over all scenes              */
    uint32_t grid_capacity;  /* active blocks over all scenes (pow2 above) */
    uint32_t max_scenes;     /* scene slots, <= 16384                      */
    uint32_t max_bodies;     /* collider table over all scenes             */
    int32_t device;
    uint32_t flags;          /* reserved, 0                                */
} slosh_batch_config;

typedef struct slosh_scene_desc {
    float cell_width;        /* MpmData::new's cell_width                  */
    slosh_params params;     /* gravity, dt (SimulationParams)             */
} slosh_scene_desc;

/* Launch shape and tile parameters of the batched substep (no effect on
 * results). */
typedef struct slosh_tuning {
    uint32_t p2g_ctas_per_sm;  /* P2G grid = SMs x this CTAs of 4 warps (5 fit an SM) */
    uint32_t g2p_threads;      /* G2P CTA size (particles a CTA holds): 64, 128 or 256 */
    uint32_t g2p_ctas_per_sm;  /* G2P grid = SMs x this                     */
    uint32_t p2g_stages;       /* particles of a cell P2G stages ahead
                                  through cp.async: 2, 3 or 4 (0: 3)        */
    uint32_t fused;            /* 1: the whole substep as one persistent
                                  cooperative kernel (CTAs of 128 threads,
                                  all resident, grid barriers between the
                                  phases; the fields above are then unused);
                                  0: 13 kernels in one CUDA graph            */
} slosh_tuning;

typedef struct slosh_batch_stats {
    uint32_t live_scenes;
    uint32_t n_particles;      /* in storage                                */
    uint32_t n_blocks;         /* active blocks of the last substep         */
    uint32_t n_materials;
    uint32_t n_svd_fp64;
    uint32_t n_bodies;         /* collider table entries in use             */
    uint32_t fused_graph;      /* 1: the fused kernel runs inside the substep
                                  graph; 0: launched directly (the runtime
                                  refused the capture) or not in use         */
    uint32_t g2p_launches;     /* G2P launches of a graph-form substep: one
                                  per class of scene present (sand, linear
                                  elastic, fluid, other), at least one       */
    slosh_tuning tuning;
} slosh_batch_stats;

int slosh_batch_create(const slosh_batch_config *cfg, slosh_batch **out);
void slosh_batch_destroy(slosh_batch *b);

/* Adds a scene of n particles (records as for slosh_upload_particles) and
 * its colliders (as for slosh_set_bodies; <= 16).  Returns its slot.
 * SLOSH_E_CAPACITY when the pool, the slots or the body table are full. */
int slosh_batch_add_scene(slosh_batch *b, const slosh_scene_desc *desc, const slosh_particle *particles,
                          uint32_t n, const slosh_body *bodies, uint32_t n_bodies, uint32_t *slot,
                          void *stream);

/* Drops a scene (its results should have been downloaded). */
int slosh_batch_remove_scene(slosh_batch *b, uint32_t slot);

/* Advances every live scene by n_substeps (graph launches on `stream`; with
 * the fused tuning one cooperative kernel a substep, captured in the graph
 * where the runtime supports it).  SLOSH_E_TIMEOUT (at the next sync) when
 * a grid barrier of the fused kernel gave up waiting; the batch's state is
 * then undefined. */
int slosh_batch_step(slosh_batch *b, uint32_t n_substeps, void *stream);

/* Particles / positions (x, y, z, 0) of one scene, in its upload order. */
int slosh_batch_download_particles(slosh_batch *b, uint32_t slot, slosh_particle *out, uint32_t n,
                                   void *stream);
int slosh_batch_download_positions(slosh_batch *b, uint32_t slot, float *out_xyzw, uint32_t n, void *stream);
int slosh_batch_get_bodies(slosh_batch *b, uint32_t slot, slosh_body *out, uint32_t n);

/* slosh_timestep_bound for one scene of the batch. */
int slosh_batch_timestep_bound(slosh_batch *b, uint32_t slot, float *dt_out, void *stream);

/* Waits for the batch's work; reports device-side errors. */
int slosh_batch_sync(slosh_batch *b, void *stream);
int slosh_batch_get_stats(slosh_batch *b, slosh_batch_stats *out);

/* Autotuner: times seven launch shapes (P2G CTAs per SM; G2P CTA size and
 * CTAs per SM), then P2G's staging depth 2 and 4 with the best shape, then
 * the fused persistent kernel, each on `substeps` real substeps of the
 * current scenes (the simulation advances; every candidate gives identical
 * results), keeps the fastest (the fused kernel only when it is 5 % faster
 * than the best graph shape), and caches it per (dim, material mix,
 * particle-count bucket) for later batches in the process.  A cached entry
 * is reused without timing. */
int slosh_batch_autotune(slosh_batch *b, uint32_t substeps, void *stream);
int slosh_batch_set_tuning(slosh_batch *b, const slosh_tuning *t);
int slosh_batch_last_error(const slosh_batch *b, char *buf, size_t len);

/* ---- Serving loop -----------------------------------------------------------
 * A request is one scene to advance by a number of substeps.  A worker
 * thread owns a batch: it admits queued requests in arrival order while their
 * device footprint fits the HBM budget (particle pool, block capacity, scene
 * slots), advances all in-flight scenes together (continuous batching:
 * scenes join and leave between batched steps), and on completion writes the
 * scene's final positions to the request's output buffer and frees its slot.
 * No reference counterpart: slosh's frame loops (src_testbed/step.rs:208-224)
 * step one scene at a time. */
typedef struct slosh_server slosh_server;

typedef struct slosh_server_config {
    int32_t dim;
    int32_t device;
    uint64_t hbm_budget_bytes;  /* the batch's pool is carved from this      */
    uint32_t max_scenes;        /* in-flight scenes                            */
    uint32_t max_bodies;
    uint32_t tick_substeps;     /* substeps per batched step, at most          */
    uint32_t max_in_flight;     /* 0: no limit; 1: one request at a time       */
    uint32_t autotune;          /* 1: tune the launch shape under load, again
                                   whenever the in-flight mix changes bucket */
    uint32_t pad;
} slosh_server_config;

typedef struct slosh_request {
    slosh_scene_desc desc;
    uint32_t n;                      /* particles                                  */
    uint32_t n_bodies;
    uint32_t substeps;
    uint32_t pad;
    const slosh_particle *particles; /* caller-owned until completion            */
    const slosh_body *bodies;        /* caller-owned until completion            */
    float *out_positions;            /* n x 4 floats, written at completion      */
} slosh_request;

typedef struct slosh_completion {
    uint64_t id;
    int32_t status;  /* SLOSH_OK or the error that ended the request         */
    uint32_t n;
    uint32_t substeps;
    uint32_t pad;
    double submit_s, admit_s, done_s;  /* server clock, seconds                */
} slosh_completion;

typedef struct slosh_server_stats {
    uint64_t submitted, admitted, completed;
    uint64_t particle_substeps;  /* work done                                   */
    uint64_t in_flight_bytes;    /* footprint of the admitted scenes            */
    uint64_t pool_bytes;         /* device memory the batch holds               */
    double busy_s;               /* time with at least one scene in flight      */
    double now_s;
    uint32_t in_flight, queued;
    uint32_t max_in_flight_seen, pad;
    slosh_tuning tuning;         /* the batch's launch shape (after autotuning) */
} slosh_server_stats;

int slosh_server_create(const slosh_server_config *cfg, slosh_server **out);
/* Stops the worker; queued and in-flight requests are dropped. */
void slosh_server_destroy(slosh_server *s);
/* Queues a request (thread-safe, non-blocking); SLOSH_E_CAPACITY when it
 * can never fit the budget's pool. */
int slosh_server_submit(slosh_server *s, const slosh_request *req, uint64_t *id);
/* Takes up to `cap` completions (non-blocking). */
int slosh_server_poll(slosh_server *s, slosh_completion *out, uint32_t cap, uint32_t *n_out);
/* Waits until nothing is queued or in flight; SLOSH_E_STATE on timeout. */
int slosh_server_wait_idle(slosh_server *s, double timeout_s);
int slosh_server_get_stats(slosh_server *s, slosh_server_stats *out);
int slosh_server_last_error(const slosh_server *s, char *buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* SLOSH_B200_H */
