/*
 * bh_oracle.h -- CPU restatement of the reference Barnes-Hut step pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * and the timed CPU baseline; the engine never links, loads or calls it.
 *
 * It restates, invocation by invocation, the WGSL compute shaders of the
 * reference (ElliottF05/webgpu-fluid-sim):
 *   src/shaders/compute/lbvh.wgsl:42-69     Morton encode (fixed 2000-unit square)
 *   src/shaders/compute/lbvh.wgsl:72-83     delta(i,j) with index tie-break
 *   src/shaders/compute/lbvh.wgsl:85-165    Karras (2012) fig. 4 hierarchy build
 *   src/shaders/compute/lbvh.wgsl:168-232   bottom-up mass / COM / AABB fill
 *   src/shaders/compute/barnes_hut.wgsl:48-111  per-body DFS walk + velocity kick
 *   src/shaders/compute/barnes_hut.wgsl:113-120 position drift
 *   src/simulation.ts:386-425               stage order of one step
 * The sort stage is the third-party npm package webgpu-radix-sort@1.0.7
 * (package-lock.json:880-885; called at simulation.ts:132-140,400), which is
 * not vendored.  Its contract here is the stable LSD radix sort of
 * (key, id) pairs, i.e. the unique stable order by key.
 *
 * Parity status: the reference ships no tests, golden vectors or fixtures, and
 * its WGSL needs a WebGPU device, which this machine does not have.  The
 * restatement is pinned by hand-computed known-answer tests and, in the build
 * container, against a mechanical C++ translation of the reference's own WGSL
 * (oracle/wgsl_to_cpp.py -> oracle/_ref/).
 *
 * Extensions with no reference counterpart (selected by orc_params fields):
 * 64-bit Morton keys over a power-of-two domain, tight-bounding-box 32-bit
 * keys, Plummer softening, kick-drift-kick leapfrog, leaf buckets in the walk,
 * and an FP64 direct sum.
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SOFT_REFERENCE = 0, ORC_SOFT_PLUMMER = 1 };
enum { ORC_DOMAIN_FIXED2000 = 0, ORC_DOMAIN_BBOX = 1 };
enum { ORC_INT_SYMPLECTIC_EULER = 0, ORC_INT_LEAPFROG_KDK = 1 };

typedef struct orc_params {
    float grav_constant;      /* config.ts gravConstant */
    float delta_time;         /* config.ts deltaTime */
    float epsilon_multiplier; /* config.ts epsilonMultiplier (reference softening) */
    float bh_theta;           /* config.ts bhTheta */
    int softening;            /* ORC_SOFT_* */
    float plummer_eps;        /* softening length for ORC_SOFT_PLUMMER */
    int morton_bits;          /* 32 or 64 */
    int morton_domain;        /* ORC_DOMAIN_* (64-bit keys always use the power-of-two domain) */
    int integrator;           /* ORC_INT_* */
    int leaf_size;            /* 1 = reference walk; >1 = direct sum over subtrees of <= leaf_size bodies */
    int threads;              /* OpenMP threads for the parallel baseline (0 = all) */
    int walk_mode;            /* 0 = reference per-body walk, 1 = group walk (extension) */
    int multipole;            /* group walk: 1 monopole, 2 monopole + quadrupole */
    int bodies_per_lane;      /* group walk: group = 32 * bodies_per_lane consecutive sorted slots */
    float far_alpha;          /* group walk, Plummer: far nodes through a local expansion (0 = off) */
} orc_params;

/* Domain used by the Morton encode: scale/offset for 32-bit keys, or the
 * power-of-two exponent for 64-bit keys. */
typedef struct orc_domain {
    float lo_x, lo_y;   /* lower corner (32-bit keys) */
    float extent;       /* side of the square (32-bit keys) */
    int pow2_exp;       /* 64-bit keys: domain is [-2^(e-1), 2^(e-1))^2 */
} orc_domain;

void orc_domain_compute(const orc_params* p, uint32_t n, const float* pos, orc_domain* out);

/* lbvh.wgsl:42-69 (and the extensions).  codes are always stored as uint64. */
void orc_morton(const orc_params* p, const orc_domain* dom, uint32_t n, const float* pos,
                uint64_t* codes, uint32_t* ids);

/* Stable sort of (codes, ids) by code (the radix-sort contract). */
void orc_sort(uint32_t n, uint64_t* codes, uint32_t* ids);

/* lbvh.wgsl:72-165: left/right child and parent indices (2n-1 nodes). */
void orc_build(uint32_t n, int morton_bits, const uint64_t* sorted_codes,
               uint32_t* left, uint32_t* right, uint32_t* parent);

/* lbvh.wgsl:168-232, executed invocation by invocation in dispatch order
 * (race-free).  com: 2*(2n-1), mass_node: 2n-1, aabb: 4*(2n-1), length: 2n-1. */
void orc_fill(uint32_t n, uint32_t offset, const uint32_t* ids, const float* mass,
              const float* pos, const uint32_t* left, const uint32_t* right,
              const uint32_t* parent, float* com, float* mass_node, float* aabb, float* length);

/* barnes_hut.wgsl:48-111 without the kick: acc[2*body] for every body. */
void orc_walk(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
              const float* pos, const float* com, const float* mass_node, const float* length,
              const uint32_t* left, const uint32_t* right, float* acc);

/* Extension: second moments about each node's COM, quad[3*(2n-1)] = {Sxx, Sxy, Syy}
 * (leaves 0), combined left child first: S = sum_c S_c + m_c d_c d_c^T. */
void orc_quadrupoles(uint32_t n, const uint32_t* left, const uint32_t* right, const float* com,
                     const float* mass_node, float* quad);

/* Extension: group walk.  Groups are the maximal subtrees of at most
 * G = 32*bodies_per_lane bodies (contiguous sorted slots); a group opens a
 * node unless L^2 < theta^2 d^2 (L = longest side of the node's
 * box, d = distance between the group's box and the node's box); accepted
 * nodes act through monopole (+ quadrupole), leaves and opened nodes of
 * <= leaf_size bodies body by body.  acc[2*body]. */
void orc_walk_group(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
                    const float* pos, const float* com, const float* mass_node, const float* aabb,
                    const float* quad, const uint32_t* left, const uint32_t* right, float* acc);

/* Node visit / interaction counters of the same walk (for rooflines). */
void orc_walk_counts(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
                     const float* pos, const float* com, const float* mass_node,
                     const float* length, const uint32_t* left, const uint32_t* right,
                     uint64_t* visits, uint64_t* interactions);

/* FP64 direct sum for the listed bodies: acc_out[2*k] for body sample[k]. */
void orc_direct_sum_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                         uint32_t nsample, const uint32_t* sample, double* acc_out);

/* Extension: FP64 direct-sum rollout of `steps` kick-drift-kick steps
 * (Plummer softening) and its exact adjoint.  Returns
 * L = (1/n) sum_i |x_T,i - target_i|^2 and writes dL/dx0 (gx[2n]),
 * dL/dv0 (gv[2n]) and dL/dm (gm[n]). */
double orc_rollout_grad_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                             const float* vel, const float* target, uint32_t steps, double* gx,
                             double* gv, double* gm);

/* Extension: FP64 direct-sum force VJP, xbar[2n] = (da/dx)^T abar and
 * mbar[n] = (da/dm)^T abar (Plummer softening). */
void orc_force_vjp_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                        const float* abar, double* xbar, double* mbar);

/* Full state of a run: the buffers of simulation.ts:82-91 plus scratch. */
typedef struct orc_state orc_state;

orc_state* orc_create(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                      const float* vel);
void orc_destroy(orc_state* s);
/* One step (simulation.ts:394-420), the reference stage order. */
void orc_step(orc_state* s, uint32_t nsteps);
/* Accelerations at the current positions (tree + walk, no integration). */
void orc_accelerations(orc_state* s, float* acc);
void orc_get_state(const orc_state* s, float* pos, float* vel);
/* Intermediate buffers of the last tree built (sorted codes, ids, tree). */
void orc_get_tree(const orc_state* s, uint64_t* codes, uint32_t* ids, uint32_t* left,
                  uint32_t* right, uint32_t* parent, float* com, float* mass_node, float* aabb,
                  float* length);
uint32_t orc_num_bodies(const orc_state* s);

/* Density render (next to the path: the reference's Renderer, renderer.ts).
 * cam = {centre x, centre y, half size x, half size y}; buffers in display
 * orientation (row 0 at the top, world y growing downwards as in
 * renderer.ts:262-269 canvasPxToWorld).
 * orc_render_density: density.wgsl:39-97 -- every body adds
 *   base * exp(-10 r^2) * zoom_scale to each pixel centre within r = |uv| <= 1
 *   of its disc of 2 * radius_multiplier pixels; summed in FP64 in body order.
 * orc_tone_map: tone_map.wgsl:57-84 -- density rounded to FP16, exposure 8,
 *   Reinhard, gamma 1/2.2, colormap (tone_map.wgsl:24-46), RGBA8. */
void orc_render_density(const float cam[4], uint32_t width, uint32_t height, uint32_t n,
                        const float* pos, const float* radius_multiplier, double* density);
void orc_tone_map(uint32_t pixels, const float* density, uint8_t* rgba);
/* colormap(t) of tone_map.wgsl:24-46 (rgb). */
void orc_colormap(float t, float rgb[3]);
/* The per-pixel parts of the two passes: density.wgsl:73-97 for a pixel at
 * quad coordinates (ux, uy) (discarded outside the disc), and
 * tone_map.wgsl:63-84 for one r16float texel value (rgb before the unorm
 * conversion). */
float orc_splat_weight(float ux, float uy, float radius_multiplier, float zoom_scale,
                       int* discarded);
void orc_tone_map_rgb(float texel, float rgb[3]);

/* FP64 diagnostics: out = {M, COM x, COM y, P x, P y, Lz, K, W}; W is the
 * direct pair sum -G sum_{i<j} m_i m_j / sqrt(r^2 + eps_ij^2) with the
 * softening of p (Plummer, or barnes_hut.wgsl:90-92's mass-dependent eps). */
void orc_diagnostics_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                          const float* vel, double out[8]);

/* Scenarios with one PCG32 stream per body (the engine's GPU generators):
 * body i draws from PCG32(seed, sequence splitmix64(i)); formulas of the
 * engine's host generators (simulation.ts:233-374 and the benchmark
 * scenarios).  Returns -1 for an unknown name.  radius may be NULL. */
int orc_generate_per_body(const char* name, uint32_t n, uint64_t seed, double G, float* mass,
                          float* pos, float* vel, float* radius);

/* OpenMP thread count the parallel paths use. */
int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
