/*
 * bh.h -- C ABI of the B200 Barnes-Hut engine (libbh_b200.so).
 *
 * This is the drop-in boundary for the per-step compute pipeline of the
 * reference simulator (ElliottF05/webgpu-fluid-sim, class Simulation in
 * src/simulation.ts:39-433).  Every entry point below names the reference
 * member it replaces.  A host binding (Node-API addon, ctypes, cffi) wraps
 * these one to one.
 *
 * Conventions
 *  - Every function returns an int status: BH_OK (0) or a BH_ERR_* code.
 *    bh_last_error(sim) returns the message of the last failure on that
 *    handle (bh_global_last_error() for failures without a handle).
 *  - The handle owns every device buffer.  bh_set_num_bodies/bh_set_scenario
 *    reallocate them, exactly like simulation.ts:367-369, so device pointers
 *    returned by bh_get_buffers stay valid only until the next set call or
 *    bh_destroy (simulation.ts:427-429, interaction.ts:28-36).
 *  - One CUDA stream per handle.  Work is stream-ordered and asynchronous
 *    (like queue.submit); bh_sync waits for it.  A handle is not thread-safe;
 *    different handles may be used from different threads.
 *  - Host pointers are plain float arrays: mass[n], pos[2n] (x,y interleaved,
 *    vec2<f32> as in simulation.ts:82-84), vel[2n].
 */
#ifndef BH_B200_H
#define BH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BH_OK 0
#define BH_ERR_INVALID_ARGUMENT 1
#define BH_ERR_CUDA 2
#define BH_ERR_OUT_OF_MEMORY 3
#define BH_ERR_UNKNOWN_SCENARIO 4 /* simulation.ts:363-365 throws "Unknown scenario" */
#define BH_ERR_DEVICE_CHECK 5     /* a device-side check tripped (bounded spin, stack) */
#define BH_ERR_NO_DEVICE 6
#define BH_ERR_NOT_SUPPORTED 7

/* ---- configuration ----------------------------------------------------- */
#define BH_SOFTENING_REFERENCE 0 /* eps = epsMult*sqrt(G*max(m1,m2)*dt), barnes_hut.wgsl:90-91 */
#define BH_SOFTENING_PLUMMER 1   /* constant Plummer eps (extension) */

#define BH_DOMAIN_FIXED2000 0 /* square [-1000,1000)^2, lbvh.wgsl:49-57 */
#define BH_DOMAIN_BBOX 1      /* tight bounding box of the bodies (extension) */

#define BH_INTEGRATOR_SYMPLECTIC_EULER 0 /* kick then drift, barnes_hut.wgsl:110,119-120 */
#define BH_INTEGRATOR_LEAPFROG_KDK 1     /* kick-drift-kick with cached force (extension) */

/* Mirrors Config of src/config.ts:1-7 plus the engine's extensions. */
typedef struct bh_config {
    float grav_constant;      /* gravConstant (config.ts:10) */
    float bh_theta;           /* bhTheta (config.ts:11) */
    int32_t substeps;         /* substeps (config.ts:12): steps per bh_step frame */
    float delta_time;         /* deltaTime (config.ts:13) */
    float epsilon_multiplier; /* epsilonMultiplier (config.ts:14) */
    int32_t softening;        /* BH_SOFTENING_* */
    float plummer_eps;        /* used with BH_SOFTENING_PLUMMER */
    int32_t morton_bits;      /* 32 (reference, 16 bits/axis) or 64 (32 bits/axis) */
    int32_t morton_domain;    /* BH_DOMAIN_* for 32-bit keys; 64-bit keys use a power-of-two box */
    int32_t integrator;       /* BH_INTEGRATOR_* */
    int32_t leaf_size;        /* 1 = reference walk; >1: subtrees of <= leaf_size bodies are summed directly */
    int32_t walk_block;       /* threads per walk block (0 = autotuned default) */
    int32_t device;           /* CUDA device ordinal */
    int32_t use_graphs;       /* 1 = replay each step from a captured CUDA graph */
    int32_t fp64_levels;      /* 1 = FP64 mass/COM aggregation for nodes of >= 1024 bodies */
    int32_t walk_mode;        /* BH_WALK_EXACT (reference per-body walk) or BH_WALK_GROUP */
    int32_t multipole_order;  /* group walk: 1 = monopole, 2 = monopole + quadrupole */
    int32_t bodies_per_lane;  /* group walk: 1, 2 or 4 (group = 32 x this many bodies); 0 = 2 */
    float far_alpha;          /* group walk, Plummer softening: an accepted node whose distance R
                                 from the group's box centre exceeds r_g / far_alpha (r_g = the
                                 box's half-diagonal) acts through one local expansion per group
                                 instead of on each body (0 = off; at most 0.5) */
    int32_t reserved[3];
} bh_config;

#define BH_WALK_EXACT 0 /* lane-exact replica of barnes_hut.wgsl:48-111 (monopole, per-body theta test) */
#define BH_WALK_GROUP 1 /* extension: per-warp group test (group box vs node box) + multipoles */

/* getDefaultConfig() (config.ts:9-22) plus extension defaults that keep the
 * reference behaviour (reference softening, fixed domain, 32-bit keys,
 * symplectic Euler, leaf_size 1). */
int bh_default_config(bh_config* out);

/* ---- lifetime ----------------------------------------------------------- */
typedef struct bh_sim bh_sim;

/* new Simulation(config, device) (simulation.ts:55-66): 50000 bodies,
 * scenario "default", buffers allocated but not yet filled. */
int bh_create(const bh_config* config, bh_sim** out);
int bh_destroy(bh_sim* sim);

/* setNumBodies(n) (simulation.ts:227-231): reallocates and regenerates the
 * current scenario. */
int bh_set_num_bodies(bh_sim* sim, uint32_t n);

/* setScenario(name) (simulation.ts:233-374).  Names: "default",
 * "two-clusters", "planetary-disk" (the reference's three), and the seeded
 * benchmark generators "uniform-disk-kepler", "colliding-disks",
 * "gaussian-mixture", "plummer-projection".  The reference draws from
 * Math.random(); here every draw comes from PCG32 seeded by `seed`.  Unknown
 * names return BH_ERR_UNKNOWN_SCENARIO ("Unknown scenario: <name>"). */
int bh_set_scenario(bh_sim* sim, const char* name, uint64_t seed);

/* updateMetadataBuffer() (simulation.ts:212-225).  The engine's fill is
 * race-free, so the random leaf offset of lbvh.wgsl:171 has no effect; this
 * call only re-validates the configuration.  Kept for API parity. */
int bh_update_metadata(bh_sim* sim);

/* Host state in/out (queue.writeBuffer at simulation.ts:376-384, and the
 * checkpoint path).  n must equal the body count.  Any pointer may be NULL
 * to skip that array.  bh_upload is asynchronous for page-locked host
 * memory, which must stay valid until the copies are done (the next
 * bh_sync or bh_download).  The copies run on a second copy stream of the
 * handle, positions first, then masses, then velocities, each into its own
 * device staging buffer as soon as the previous upload of that array has
 * been moved out of it, so they may overlap steps still running; the
 * handle's stream moves each array into place before its next reader.  The
 * next step's stages before those readers (the hierarchy build for the
 * masses, the walk for the velocities) do not wait for them; every other
 * call orders the handle's stream after them.  bh_download synchronises
 * before returning. */
int bh_upload(bh_sim* sim, const float* mass, const float* pos, const float* vel, uint32_t n);
int bh_download(bh_sim* sim, float* mass, float* pos, float* vel, uint32_t n);

/* Same as bh_download, without waiting (extension; no reference counterpart
 * beyond the readback of simulation.ts:376-384).  The arrays are copied on
 * the handle's stream into a device snapshot, and from there to the host on
 * a third stream of the handle, so the steps enqueued next run while the
 * host copy is under way.  The host arrays (page-locked for an asynchronous
 * copy) are written by the next bh_sync or bh_download, which wait for the
 * copy and report device errors; a later bh_download_async reuses the
 * snapshot once this copy has left it. */
int bh_download_async(bh_sim* sim, float* mass, float* pos, float* vel, uint32_t n);

/* getCommands() + queue.submit (simulation.ts:386-425, main.ts:38-41):
 * enqueue `frames` frames of config.substeps steps each.  Asynchronous. */
int bh_step(bh_sim* sim, uint32_t frames);
int bh_sync(bh_sim* sim);

/* Accelerations at the current positions without integrating: builds the
 * tree and runs the walk; acc[2n] (device buffer, original body order) is
 * copied to acc_host when it is not NULL. */
int bh_compute_accelerations(bh_sim* sim, float* acc_host);

/* ---- buffers (getBuffers(), simulation.ts:8-18,427-429) ----------------- */
/* Device pointers borrowed from the handle.  Layouts:
 *   mass[n], pos[2n], vel[2n], radius_multiplier[n], acc[2n]  (original body order)
 *   morton_codes[n]: uint32 (32-bit keys) or uint64 (64-bit keys), sorted
 *   body_indices[n]: sorted permutation (sorted slot -> body)
 *   node4[2n-1]: float4 {com.x, com.y, mass, length}; internal nodes
 *                [0, n-2], leaves [n-1, 2n-2] (lbvh.wgsl:94)
 *   node_children[2(n-1)]: {left, right} per internal node
 *   node_parent[2n-1]: parent index, 0xFFFFFFFF at the root
 *   node_aabb[4(n-1)]: {min.x, min.y, max.x, max.y} per internal node
 *                      (a leaf's box is its body position)
 * With walk_mode BH_WALK_GROUP the step keeps the internal nodes in packed
 * 64-byte records and writes the internal entries of node4, node_children
 * and node_aabb only on request: each bh_get_buffers call (stream-ordered on
 * the handle's stream) and each bh_read_buffer of those names refreshes them
 * for the current tree.  Leaves, node_parent and the body arrays are
 * current after every step in both modes. */
typedef struct bh_buffers {
    float* mass;
    float* pos;
    float* vel;
    float* radius_multiplier;
    float* acc;
    void* morton_codes;
    uint32_t* body_indices;
    float* node4;
    uint32_t* node_children;
    uint32_t* node_parent;
    float* node_aabb;
    uint32_t num_bodies;
    int32_t morton_bits;
    void* stream; /* cudaStream_t of the handle */
} bh_buffers;

int bh_get_buffers(bh_sim* sim, bh_buffers* out);
int bh_get_num_bodies(bh_sim* sim, uint32_t* out); /* getNumBodies() (simulation.ts:430-432) */

/* Copy `bytes` from the start of a named device buffer to host memory
 * (synchronous).  Names: "mass", "pos", "vel", "acc", "radius_multiplier",
 * "morton_codes", "body_indices", "node4", "node_children", "node_parent",
 * "node_aabb". */
int bh_read_buffer(bh_sim* sim, const char* name, void* host, size_t bytes);

/* ---- scenarios generated on the GPU (extension) -------------------------- */
/* Same names, distributions and formulas as bh_set_scenario, generated on
 * the GPU: body i draws from its own PCG32 stream (sequence selector
 * splitmix64(i), state seeded by `seed`), in FP64, stored as FP32, so no host
 * arrays and no upload are involved (16.8M bodies in a few milliseconds).
 * The sample differs from bh_set_scenario's for the same seed (that one
 * draws all bodies from one sequential stream).  Reallocates the buffers
 * like bh_set_scenario; later bh_set_num_bodies calls regenerate on the GPU
 * until bh_set_scenario is called again.  Gaussian-mixture masses are
 * normalised by an FP64 total whose last bits follow the GPU's SM count. */
int bh_set_scenario_device(bh_sim* sim, const char* name, uint64_t seed);

/* The same generators on caller-owned device arrays (mass[n], pos[2n],
 * vel[2n], radius_multiplier[n] or NULL), enqueued on `stream` (a
 * cudaStream_t) of the current device. */
int bh_generate_scenario_device(const char* name, uint32_t n, uint64_t seed, float grav_constant,
                                float* mass, float* pos, float* vel, float* radius_multiplier,
                                void* stream);

/* ---- host-side scenario generation (no device work) --------------------- */
/* Fills mass[n], pos[2n], vel[2n] and (optionally) radius_multiplier[n] with
 * the named scenario, exactly as bh_set_scenario does before its upload. */
int bh_generate_scenario(const char* name, uint32_t n, uint64_t seed, float grav_constant,
                         float* mass, float* pos, float* vel, float* radius_multiplier);

/* ---- profiling ---------------------------------------------------------- */
#define BH_STAGE_MORTON 0  /* bbox + Morton encode + digit histograms */
#define BH_STAGE_SORT 1    /* radix sort passes */
#define BH_STAGE_TREE 2    /* hierarchy build + mass/COM fill */
#define BH_STAGE_WALK 3    /* walk + integrate */
#define BH_STAGE_OTHER 4   /* kick-drift (leapfrog), memsets */
#define BH_NUM_STAGES 5

/* Start recording CUDA events around every stage of the next `max_steps`
 * steps (on the handle's stream).  bh_profile_end synchronises and returns
 * the summed milliseconds per stage and the number of steps recorded. */
int bh_profile_begin(bh_sim* sim, uint32_t max_steps);
int bh_profile_end(bh_sim* sim, double* stage_ms, uint32_t* steps_recorded);

/* ---- autotuner (extension; no reference counterpart) -------------------- */
typedef struct bh_tune_result {
    int32_t bodies_per_lane; /* chosen walk group shape: 32 x this many bodies per warp */
    int32_t leaf_size;       /* chosen bucket size */
    float walk_ms;           /* its average walk time */
    int32_t candidates;      /* candidates timed */
    int32_t walk_block;      /* chosen threads per walk block */
} bh_tune_result;

/* Time the group walk (on force evaluations at the current positions, which
 * do not advance the state) for bodies_per_lane in {1, 2, 4} x leaf_size in
 * {2, 4, 8} with 128-thread blocks, then the best of those with 64- and
 * 256-thread blocks (walk_block; 128-body groups run blocks of at most 128
 * threads), `trials` launches each after one warm-up, and keep the fastest
 * in the handle's configuration (10 or 11 candidates).  Group walk only. */
int bh_autotune(bh_sim* sim, uint32_t trials, bh_tune_result* out);

/* The handle's current configuration (after bh_autotune, for instance). */
int bh_get_config(bh_sim* sim, bh_config* out);

/* Kernels one step launches (for launch accounting). */
int bh_kernels_per_step(bh_sim* sim, uint32_t* out);

/* Build the tree at the current positions and run an instrumented force walk
 * that counts node visits (exact walk: per body; group walk: per group) and
 * the interactions evaluated over all bodies: with a node's multipole
 * (monopole, or monopole + quadrupole) and with single bodies, and the
 * (node, group) pairs that went through the far-field local expansion (for
 * rooflines; any pointer may be NULL).  Leaves acc[] holding the forces;
 * does not integrate. */
int bh_walk_stats(bh_sim* sim, uint64_t* node_visits, uint64_t* multipole_interactions,
                  uint64_t* body_interactions, uint64_t* far_nodes);

/* ---- differentiation (extension; no reference counterpart) ---------------- */
/* Vector-Jacobian product of the force at the current positions: given
 * abar[2n] (host), returns xbar[2n] = (da/dx)^T abar and mbar[n] =
 * (da/dm)^T abar (host; either may be NULL).  The interaction lists are those
 * of the forward group walk (topology held fixed), node moments are
 * differentiated down to their member bodies.  Needs walk_mode
 * BH_WALK_GROUP and Plummer softening (else BH_ERR_NOT_SUPPORTED). */
int bh_force_vjp(bh_sim* sim, const float* abar, float* xbar, float* mbar);

/* Differentiable rollout: advances `steps` kick-drift-kick steps from the
 * current state, evaluates L = (1/n) sum_i |x_T,i - target_i|^2 and its
 * gradient with respect to the initial positions, velocities and masses by
 * a reverse sweep: positions and velocities are checkpointed every
 * `checkpoint_every` steps, each segment is replayed (trees rebuilt) and the
 * force VJP is applied once per force point.  The handle is left at step T.
 * Host arrays: target_pos[2n]; outputs grad_pos[2n], grad_vel[2n],
 * grad_mass[n] (any may be NULL).  Needs the leapfrog integrator, the group
 * walk and Plummer softening. */
int bh_rollout_grad(bh_sim* sim, uint32_t steps, uint32_t checkpoint_every,
                    const float* target_pos, float* loss, float* grad_pos, float* grad_vel,
                    float* grad_mass);

/* ---- one system on several GPUs (extension; the reference has one device) */
/* Every rank holds the whole state and builds the same tree (the pipeline is
 * deterministic).  bh_set_walk_slots(lo, hi) makes each step integrate only
 * the groups whose first sorted slot lies in [lo, hi) -- the ranks take
 * consecutive ranges of [0, n) -- while force evaluations stay complete.
 * After a step, bh_shard_pack writes what this rank updated -- (pos, vel)
 * for symplectic Euler, (vel, acc) for leapfrog -- in sorted-slot order into
 * a device chunk of 16 + 16 * capacity bytes (header {first slot, count, 0,
 * 0}, then one float4 per body; capacity >= ceil(n / ranks) + 32 *
 * bodies_per_lane covers any range); the caller all-gathers the chunks
 * (NCCL) and bh_shard_unpack applies all of them, after which every rank
 * holds the state one GPU would have computed.  Both are enqueued on the
 * handle's stream.  Group walk only; not for ensembles (shard those by
 * systems). */
int bh_set_walk_slots(bh_sim* sim, uint32_t slot_lo, uint32_t slot_hi);
int bh_shard_pack(bh_sim* sim, void* chunk, uint32_t capacity);
int bh_shard_unpack(bh_sim* sim, const void* chunks, uint32_t num_chunks, uint32_t capacity);

/* ---- batched ensembles (extension; no reference counterpart) ------------- */
/* An ensemble handle advances many independent systems with one launch per
 * stage: the bodies of all systems are concatenated (system k owns bodies
 * [off_k, off_k+1)), each system gets its own bounding box and 32-bit Morton
 * domain, the sort keys are (system << 32) | code so one sort and one
 * hierarchy build serve every system (the tree's top levels split by
 * system), and each walk group only interacts with its own system.  All
 * other calls (bh_step, bh_upload, bh_download, bh_get_buffers, ...) work on
 * the concatenation.  Needs walk_mode BH_WALK_GROUP and morton_bits 32; every
 * system has at least 256 bodies. */
int bh_ensemble_create(const bh_config* config, const uint32_t* bodies_per_system,
                       uint32_t num_systems, bh_sim** out);

/* Fill every system: names[k] is system k's scenario (seed derived from
 * `seed` and k); names == NULL picks a Plummer-sphere projection (scale
 * radius 0.1) or a uniform disk with probability 1/2 each. */
int bh_ensemble_set_scenarios(bh_sim* sim, const char* const* names, uint64_t seed);

/* Log-uniform system sizes in [min_bodies, max_bodies] from PCG32(seed). */
int bh_ensemble_sizes(uint32_t num_systems, uint64_t seed, uint32_t min_bodies,
                      uint32_t max_bodies, uint32_t* out);

int bh_get_num_systems(bh_sim* sim, uint32_t* out);       /* 0 for a single system */
int bh_get_system_offsets(bh_sim* sim, uint32_t* offsets); /* num_systems + 1 entries */

/* ---- allocation-free hierarchy build ------------------------------------ */
/* No counterpart in the reference.  For callers that cannot let this library
 * allocate device memory (a host that plans the whole GPU heap and hands out
 * every buffer, a frame loop that cannot take the device-wide sync of
 * cudaMalloc/cudaFree, code that must not allocate once running): builds the
 * hierarchy and fills node mass/COM/AABB -- the same kernel and results as the
 * tree stage of bh_step -- from caller-owned device buffers, with the
 * kernel's scratch in a static device array inside the library.
 *   in : sorted_codes[n] (uint32, or uint64 when morton_bits == 64),
 *        sorted_ids[n], mass[n], pos[2n] (original body order)
 *   out: node4[4(2n-1)], node_children[2(n-1)], node_parent[2n-1],
 *        node_aabb[4(n-1)]  (layouts as in bh_buffers)
 * Limit: n <= 262144 (larger n returns BH_ERR_INVALID_ARGUMENT).  Enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream); calls no cudaMalloc
 * or cudaFree.  All calls share the static scratch: calls that overlap on the
 * GPU race, so serialise them.  Every call looks the scratch up with
 * cudaGetSymbolAddress in the current context.  Under CUDA's lazy module
 * loading the first call on a device may load this library's module, which
 * reserves the static array (about 11.5 MB) and may synchronise: a caller
 * that must not allocate while running makes one warm-up call at start-up,
 * before any stream capture.  Errors are reported through
 * bh_global_last_error(). */
int bh_build_hierarchy_static(const void* sorted_codes, int32_t morton_bits,
                              const uint32_t* sorted_ids, const float* mass, const float* pos,
                              uint32_t n, float* node4, uint32_t* node_children,
                              uint32_t* node_parent, float* node_aabb, int32_t fp64_levels,
                              void* stream);

/* ---- FP64 diagnostics (extension; the reference only logs FPS, main.ts:44-49) */
/* Conserved quantities of the current state, summed in FP64 over all bodies:
 * total mass, centre of mass, linear momentum, angular momentum about the
 * origin (z), kinetic energy and -- when with_potential != 0 -- the
 * potential energy W = -G sum_{i<j} m_i m_j / sqrt(r_ij^2 + eps_ij^2) with
 * the softening of the handle's force law (Plummer eps, or the reference's
 * eps_ij^2 = epsMult^2 G dt max(m_i, m_j), barnes_hut.wgsl:90-92).  W is an
 * O(N^2) direct sum (pair terms in FP32, sums in FP64; ~0.1 s at 800k bodies
 * on a B200); potential_energy is NaN and pairs 0 when it is skipped.
 * Synchronises the handle's stream. */
typedef struct bh_diagnostics {
    double total_mass;
    double com[2];
    double momentum[2];
    double angular_momentum;
    double kinetic_energy;
    double potential_energy;
    uint64_t pairs;
} bh_diagnostics;

int bh_diagnostics_compute(bh_sim* sim, int with_potential, bh_diagnostics* out);

/* FP64 direct-sum accelerations of sampled bodies (extension; the reference
 * has no force check).  For each body index sample[k] (original order, host
 * array, count <= 2^20), acc_out[2k], acc_out[2k+1] (host) receive
 *   G sum_{j != i} m_j (x_j - x_i) / (|x_j - x_i|^2 + eps_ij^2)^(3/2)
 * summed in FP64 over every body at the handle's current positions, with the
 * softening of the handle's force law.  The error of a force walk is measured
 * against these.  O(count * n) work; synchronises the handle's stream. */
int bh_direct_forces_fp64(bh_sim* sim, const uint32_t* sample, uint32_t count, double* acc_out);

/* ---- density render (the reference's Renderer, src/renderer.ts:1-329) --- */
/* A headless replacement of the two render passes of Renderer.getCommands()
 * (renderer.ts:293-329): the density pass splats every body as the soft
 * disc of density.wgsl:39-97 (radius 2 * radiusMultiplier pixels, weight
 * base * exp(-10 r^2) * zoom_scale, additive), and the tone-map pass maps
 * density to colour as tone_map.wgsl:57-84 (exposure 8, Reinhard, gamma
 * 1/2.2, the four-stop colormap of tone_map.wgsl:24-46).  Instead of a canvas
 * the renderer owns two device buffers in display orientation (row 0 at the
 * top, canvas pixel (px, py) <-> world canvasPxToWorld(px + 0.5, py + 0.5)):
 *   density[height * width]  float32, accumulated in FP32 (the reference
 *                            blends into an r16float texture; the tone map
 *                            here reads each density rounded to FP16 as the
 *                            reference samples it)
 *   image[height * width * 4] uint8 RGBA (alpha 255), unorm rounding to nearest.
 * A pixel takes a body's contribution when its centre lies within the body's
 * disc (|uv| <= 1, the fragment's discard test); the reference rasterises
 * the quad around the disc first, which only differs on the disc's boundary.
 * All work is enqueued on the simulation handle's stream; the renderer
 * borrows the handle's position and radius buffers at each frame, so
 * setNumBodies / setScenario need no rebind (rebindSimBuffers,
 * renderer.ts:206-216, and setNumBodies, :219-222, have nothing to do). */
typedef struct bh_renderer bh_renderer;

/* new Renderer(...) (renderer.ts:43-61) for a width x height canvas: camera
 * centre (0, 0), half size (10 * width / height, 10) as after the
 * constructor's resizeCanvasToDisplaySize(). */
int bh_renderer_create(bh_sim* sim, uint32_t width, uint32_t height, bh_renderer** out);
int bh_renderer_destroy(bh_renderer* r);

/* resizeCanvasToDisplaySize() (renderer.ts:225-252) for a new canvas size:
 * new buffers, half size x = half size y * width / height. */
int bh_renderer_resize(bh_renderer* r, uint32_t width, uint32_t height);

/* panCamera (renderer.ts:271-277) and zoomCamera (:279-290), in canvas
 * pixels; set/get the camera {centre x, centre y, half size x, half size y}. */
int bh_renderer_pan(bh_renderer* r, float delta_px, float delta_py);
int bh_renderer_zoom(bh_renderer* r, float zoom_factor, float center_px, float center_py);
int bh_renderer_set_camera(bh_renderer* r, const float camera[4]);
int bh_renderer_get_camera(bh_renderer* r, float camera[4]);

/* getCommands(numBodies) + submit (renderer.ts:293-329, main.ts:38-41):
 * clear, density splat of the handle's current bodies, tone map.
 * Asynchronous on the simulation's stream. */
int bh_renderer_frame(bh_renderer* r);

/* Device buffers (valid until resize / destroy) and synchronous copies to
 * host memory: density[height * width] floats, image[height * width * 4]. */
int bh_renderer_get_targets(bh_renderer* r, float** density, uint8_t** image, uint32_t* width,
                            uint32_t* height);
int bh_renderer_read_density(bh_renderer* r, float* host);
int bh_renderer_read_image(bh_renderer* r, uint8_t* host);
const char* bh_renderer_last_error(bh_renderer* r);

/* ---- test hooks of the device-side checks (extension) -------------------- */
/* No counterpart in the reference, whose walk silently drops stack pushes
 * (barnes_hut.wgsl:100-105) and whose sort has no bounded wait.  The engine's
 * kernels check themselves instead of hanging or writing out of bounds: the
 * sort's decoupled look-back gives up after a bounded number of spins, and
 * the walks refuse a push that would overflow their stack.  A tripped check
 * sets the handle's device error word; the next synchronising call (bh_sync,
 * bh_download, bh_compute_accelerations, ...) returns BH_ERR_DEVICE_CHECK
 * with a message naming the check and clears the word.  After a failed sort
 * the step's hierarchy build and walk skip their work, so a failed step
 * leaves the bodies as they were before it (leapfrog: after its opening
 * kick-drift).
 * This call lowers those limits so a test can make them run out without
 * faulting or hanging the GPU:
 *   lookback_spin_cap  spins before the look-back gives up (0 = default,
 *                      about 4M spins, several seconds)
 *   walk_stack_cap     stack entries a walk warp may use (0 = full; >= 2)
 *   flags              BH_DEBUG_LOOKBACK_UNPUBLISHED: the second tile of the
 *                      first sort pass waits on a predecessor status that
 *                      never reads as published (needs n > 6144 bodies);
 *                      BH_DEBUG_SPLIT_BUILD: the split hierarchy build (local
 *                      phase + frontier climb) at every body count
 * Zeros restore normal operation.  Takes effect from the next call. */
#define BH_DEBUG_LOOKBACK_UNPUBLISHED 1u
#define BH_DEBUG_SPLIT_BUILD 2u
int bh_debug_set_limits(bh_sim* sim, uint32_t flags, uint32_t lookback_spin_cap,
                        uint32_t walk_stack_cap);

/* ---- errors ------------------------------------------------------------- */
const char* bh_last_error(bh_sim* sim);
const char* bh_global_last_error(void);
const char* bh_version(void);

#ifdef __cplusplus
}
#endif
#endif
