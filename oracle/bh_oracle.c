/*
 * bh_oracle.c -- CPU restatement of the reference Barnes-Hut step pipeline.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  The CUDA
 * engine never links or calls this file.  Each function names the reference
 * file:line it restates.  Compile with -ffp-contract=off so that every f32
 * operation rounds exactly as written, like the WGSL source.
 *
 * Parallelism: every stage is a parallel-for over the shader's invocations
 * (OpenMP).  The results do not depend on the thread count: the sort is a
 * stable LSD radix sort, the build is per-node independent, the fill combines
 * the two finished children whichever arrives second (acq_rel arrival
 * counters), and the walk is per-body independent.
 */
#include "bh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define STACK_SIZE 256 /* barnes_hut.wgsl:67 */

static int nthreads(const orc_params* p) {
#ifdef _OPENMP
    return (p && p->threads > 0) ? p->threads : omp_get_max_threads();
#else
    (void)p;
    return 1;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

/* ------------------------------------------------------------------------ */
/* Morton encode                                                             */
/* ------------------------------------------------------------------------ */

static inline uint32_t spread16(uint32_t v) { /* bit b -> bit 2b (lbvh.wgsl:59-65) */
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

static inline uint64_t spread32(uint64_t v) {
    v &= 0xFFFFFFFFull;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}

/* WGSL u32(f32) for a finite value in [0, 2^32): truncation. */
static inline uint32_t quant16(float u) {
    /* lbvh.wgsl:54-57: clamp to [0,1], u32(u*65535+0.5), min with 65535 */
    if (!(u > 0.0f)) u = 0.0f; /* clamp low (NaN maps to 0) */
    if (u > 1.0f) u = 1.0f;
    float t = u * 65535.0f;
    t = t + 0.5f;
    uint32_t q = (uint32_t)t;
    return q > 65535u ? 65535u : q;
}

void orc_domain_compute(const orc_params* p, uint32_t n, const float* pos, orc_domain* out) {
    out->lo_x = -1000.0f; /* lbvh.wgsl:49-50: fixed square of side 2000 centred at 0 */
    out->lo_y = -1000.0f;
    out->extent = 2000.0f;
    out->pow2_exp = 1;
    float lx = INFINITY, ly = INFINITY, hx = -INFINITY, hy = -INFINITY;
    for (uint32_t i = 0; i < n; ++i) {
        float x = pos[2 * i], y = pos[2 * i + 1];
        lx = fminf(lx, x); hx = fmaxf(hx, x);
        ly = fminf(ly, y); hy = fmaxf(hy, y);
    }
    if (n == 0) { lx = ly = hx = hy = 0.0f; }
    if (p->morton_bits == 64) {
        float m = fmaxf(fmaxf(fabsf(lx), fabsf(hx)), fmaxf(fabsf(ly), fabsf(hy)));
        int e;
        if (m < 0x1p-60f) e = -60;
        else { int ex; frexpf(m, &ex); e = ex + 1; } /* m < 2^ex  ->  m < 2^(e-1) */
        out->pow2_exp = e;
        return;
    }
    if (p->morton_domain == ORC_DOMAIN_BBOX) {
        float ext = fmaxf(hx - lx, hy - ly);
        if (!(ext > 0.0f)) ext = 1.0f;
        out->lo_x = lx;
        out->lo_y = ly;
        out->extent = ext;
    }
}

void orc_morton(const orc_params* p, const orc_domain* dom, uint32_t n, const float* pos,
                uint64_t* codes, uint32_t* ids) {
    int nt = nthreads(p);
    if (p->morton_bits == 64) {
        /* Extension: 32 bits per axis over [-2^(e-1), 2^(e-1)): q = floor(x*2^(32-e)) + 2^31,
         * exact because scaling by a power of two is exact. */
        float s = ldexpf(1.0f, 32 - dom->pow2_exp);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            float xs = pos[2 * i] * s, ys = pos[2 * i + 1] * s;
            int64_t qx = (int64_t)floorf(xs) + 2147483648LL;
            int64_t qy = (int64_t)floorf(ys) + 2147483648LL;
            if (qx < 0) qx = 0;
            if (qx > 4294967295LL) qx = 4294967295LL;
            if (qy < 0) qy = 0;
            if (qy > 4294967295LL) qy = 4294967295LL;
            codes[i] = spread32((uint64_t)qx) | (spread32((uint64_t)qy) << 1);
            ids[i] = (uint32_t)i;
        }
        return;
    }
    /* lbvh.wgsl:49-68 with (lo, extent) = (-1000, 2000) in the reference domain. */
    const float lo_x = dom->lo_x, lo_y = dom->lo_y, ext = dom->extent;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float ux = (pos[2 * i] - lo_x) / ext;
        float uy = (pos[2 * i + 1] - lo_y) / ext;
        uint32_t x = quant16(ux), y = quant16(uy);
        codes[i] = (uint64_t)(spread16(x) | (spread16(y) << 1));
        ids[i] = (uint32_t)i; /* lbvh.wgsl:68 */
    }
}

/* ------------------------------------------------------------------------ */
/* Stable LSD radix sort (the contract of webgpu-radix-sort)                 */
/* ------------------------------------------------------------------------ */

static void radix_sort_impl(uint32_t n, uint64_t* codes, uint32_t* ids, int bits, int nt) {
    if (n < 2) return;
    uint64_t* kt = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint32_t* vt = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint64_t *ks = codes, *kd = kt;
    uint32_t *vs = ids, *vd = vt;
    size_t* hist = (size_t*)malloc(sizeof(size_t) * 256 * (size_t)nt);
    int passes = bits / 8;
    for (int pass = 0; pass < passes; ++pass) {
        int shift = 8 * pass;
        memset(hist, 0, sizeof(size_t) * 256 * (size_t)nt);
#pragma omp parallel num_threads(nt)
        {
            int t = 0, T = 1;
#ifdef _OPENMP
            t = omp_get_thread_num();
            T = omp_get_num_threads();
#endif
            size_t lo = (size_t)n * t / T, hi = (size_t)n * (t + 1) / T;
            size_t* h = hist + 256 * (size_t)t;
            for (size_t i = lo; i < hi; ++i) h[(ks[i] >> shift) & 0xFF]++;
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int tt = 0; tt < T; ++tt) {
                        size_t c = hist[256 * (size_t)tt + d];
                        hist[256 * (size_t)tt + d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                size_t dst = h[(ks[i] >> shift) & 0xFF]++;
                kd[dst] = ks[i];
                vd[dst] = vs[i];
            }
        }
        uint64_t* tk = ks; ks = kd; kd = tk;
        uint32_t* tv = vs; vs = vd; vd = tv;
    }
    if (ks != codes) {
        memcpy(codes, ks, sizeof(uint64_t) * n);
        memcpy(ids, vs, sizeof(uint32_t) * n);
    }
    free(hist);
    free(kt);
    free(vt);
}

void orc_sort(uint32_t n, uint64_t* codes, uint32_t* ids) {
    uint64_t any = 0;
    for (uint32_t i = 0; i < n; ++i) any |= codes[i];
    radix_sort_impl(n, codes, ids, (any >> 32) ? 64 : 32, orc_max_threads());
}

/* ------------------------------------------------------------------------ */
/* Karras build: lbvh.wgsl:72-165                                            */
/* ------------------------------------------------------------------------ */

static inline int delta_fn(const uint64_t* k, int64_t n, int bits, int64_t i, int64_t j) {
    /* lbvh.wgsl:72-83 (tie-break offset = key width; 64 for 64-bit keys) */
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[i], b = k[j];
    if (a == b) return bits + clz32((uint32_t)i ^ (uint32_t)j);
    return bits == 64 ? clz64(a ^ b) : clz32((uint32_t)(a ^ b));
}

void orc_build(uint32_t n, int morton_bits, const uint64_t* k, uint32_t* left, uint32_t* right,
               uint32_t* parent) {
    if (n == 0) return;
    const int64_t N = n;
    const int bits = morton_bits;
    /* n == 1: build_lbvh_main has no internal node to run (lbvh.wgsl:95-97),
     * so the only node keeps the zero-initialised parent of its buffer. */
    if (n == 1) parent[0] = 0u;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N - 1; ++i) {
        int d = delta_fn(k, N, bits, i, i + 1) > delta_fn(k, N, bits, i, i - 1) ? 1 : -1;
        int dmin = delta_fn(k, N, bits, i, i - d);
        int64_t lmax = 2;
        while (delta_fn(k, N, bits, i, i + d * lmax) > dmin) lmax *= 2;
        int64_t l = 0;
        for (int64_t t = lmax / 2; t >= 1; t /= 2)
            if (delta_fn(k, N, bits, i, i + d * (l + t)) > dmin) l += t;
        int64_t j = i + d * l;
        int dnode = delta_fn(k, N, bits, i, j);
        int64_t s = 0, t = (l + 1) / 2;
        for (;;) {
            if (delta_fn(k, N, bits, i, i + d * (s + t)) > dnode) s += t;
            if (t == 1) break;
            t = (t + 1) / 2;
        }
        int64_t gamma = i + d * s + (d < 0 ? d : 0);
        int64_t mn = i < j ? i : j, mx = i < j ? j : i;
        uint32_t lc = (mn == gamma) ? (uint32_t)(N - 1 + gamma) : (uint32_t)gamma;
        uint32_t rc = (mx == gamma + 1) ? (uint32_t)(N - 1 + gamma + 1) : (uint32_t)(gamma + 1);
        left[i] = lc;
        right[i] = rc;
        parent[lc] = (uint32_t)i;
        parent[rc] = (uint32_t)i;
    }
    if (n > 1) parent[0] = 0xFFFFFFFFu;
}

/* ------------------------------------------------------------------------ */
/* Bottom-up fill: lbvh.wgsl:168-232                                         */
/* ------------------------------------------------------------------------ */

void orc_fill(uint32_t n, uint32_t offset, const uint32_t* ids, const float* mass,
              const float* pos, const uint32_t* left, const uint32_t* right,
              const uint32_t* parent, float* com, float* mass_node, float* aabb, float* length) {
    if (n == 0) return;
    uint32_t* status = (uint32_t*)calloc(n, sizeof(uint32_t));
    const uint32_t nm1 = n - 1;
    /* Exactly n invocations (the reference's padding invocations re-run real
     * leaves; see lbvh.wgsl:171-176).  Arrival counters are acq_rel. */
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < (int64_t)n; ++g) {
        uint32_t i = (uint32_t)(((uint64_t)g + offset) % n);
        uint32_t cur = nm1 + i;
        uint32_t b = ids[i];
        float m = mass[b], px = pos[2 * b], py = pos[2 * b + 1];
        mass_node[cur] = m;
        com[2 * cur] = px; com[2 * cur + 1] = py;
        aabb[4 * cur] = px; aabb[4 * cur + 1] = py;
        aabb[4 * cur + 2] = px; aabb[4 * cur + 3] = py;
        length[cur] = 0.0f;
        while (cur != 0u) {
            uint32_t pidx = parent[cur];
            if (pidx == cur) break;
            uint32_t prev = __atomic_fetch_add(&status[pidx], 1u, __ATOMIC_ACQ_REL);
            if (prev == 0u) break;
            uint32_t l = left[pidx], r = right[pidx];
            float lminx = aabb[4 * l], lminy = aabb[4 * l + 1], lmaxx = aabb[4 * l + 2], lmaxy = aabb[4 * l + 3];
            float rminx = aabb[4 * r], rminy = aabb[4 * r + 1], rmaxx = aabb[4 * r + 2], rmaxy = aabb[4 * r + 3];
            float minx = fminf(lminx, rminx), miny = fminf(lminy, rminy);
            float maxx = fmaxf(lmaxx, rmaxx), maxy = fmaxf(lmaxy, rmaxy);
            aabb[4 * pidx] = minx; aabb[4 * pidx + 1] = miny;
            aabb[4 * pidx + 2] = maxx; aabb[4 * pidx + 3] = maxy;
            float ml = mass_node[l], mr = mass_node[r];
            float tm = ml + mr;
            mass_node[pidx] = tm;
            if (tm > 0.0f) {
                com[2 * pidx] = (com[2 * l] * ml + com[2 * r] * mr) / tm;
                com[2 * pidx + 1] = (com[2 * l + 1] * ml + com[2 * r + 1] * mr) / tm;
            } else {
                com[2 * pidx] = 0.0f;
                com[2 * pidx + 1] = 0.0f;
            }
            float sx = maxx - minx, sy = maxy - miny;
            length[pidx] = fmaxf(sx, sy);
            cur = pidx;
        }
    }
    free(status);
}

/* ------------------------------------------------------------------------ */
/* Walk: barnes_hut.wgsl:48-111                                              */
/* ------------------------------------------------------------------------ */

/* Sorted-slot range [first, last] of every node (used for leaf buckets). */
static void node_ranges(uint32_t n, const uint32_t* left, const uint32_t* right, uint32_t* first,
                        uint32_t* last) {
    const uint32_t nm1 = n - 1;
    for (uint32_t i = 0; i < n; ++i) first[nm1 + i] = last[nm1 + i] = i;
    if (n < 2) return;
    /* iterative post-order from the root */
    uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)n);
    uint8_t* seen = (uint8_t*)calloc(n, 1);
    int64_t sp = 0;
    st[sp++] = 0;
    while (sp > 0) {
        uint32_t v = st[sp - 1];
        if (v >= nm1) { sp--; continue; }
        if (!seen[v]) {
            seen[v] = 1;
            st[sp++] = left[v];
            st[sp++] = right[v];
        } else {
            sp--;
            first[v] = first[left[v]];
            last[v] = last[right[v]];
        }
    }
    free(st);
    free(seen);
}

static inline float soft2(const orc_params* p, float m1, float m2) {
    if (p->softening == ORC_SOFT_PLUMMER) return p->plummer_eps * p->plummer_eps;
    float meff = m1 > m2 ? m1 : m2;                                  /* barnes_hut.wgsl:90 */
    float eps = p->epsilon_multiplier * sqrtf(p->grav_constant * meff * p->delta_time); /* :91 */
    return eps * eps;
}

static void walk_impl(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
                      const float* pos, const float* com, const float* mass_node,
                      const float* length, const uint32_t* left, const uint32_t* right,
                      float* acc, uint64_t* visits_out, uint64_t* inter_out) {
    if (n == 0) return;
    const uint32_t nm1 = n - 1;
    const float g = p->grav_constant, theta = p->bh_theta;
    const int L = p->leaf_size > 1 ? p->leaf_size : 1;
    uint32_t *first = NULL, *last = NULL;
    if (L > 1) {
        first = (uint32_t*)malloc(sizeof(uint32_t) * (2 * (size_t)n - 1));
        last = (uint32_t*)malloc(sizeof(uint32_t) * (2 * (size_t)n - 1));
        node_ranges(n, left, right, first, last);
    }
    uint64_t tv = 0, ti = 0;
#pragma omp parallel for num_threads(nthreads(p)) schedule(dynamic, 256) reduction(+ : tv, ti)
    for (int64_t tid = 0; tid < (int64_t)n; ++tid) {
        uint32_t body = ids[tid];                        /* barnes_hut.wgsl:56 */
        float p1x = pos[2 * body], p1y = pos[2 * body + 1], m1 = mass[body];
        float ax = 0.0f, ay = 0.0f;
        uint32_t stack[STACK_SIZE];
        int sp = 0;
        stack[0] = 0u;
        while (sp >= 0) {                                /* barnes_hut.wgsl:72 */
            uint32_t node = stack[sp];
            sp -= 1;
            tv++;
            float p2x = com[2 * node], p2y = com[2 * node + 1], m2 = mass_node[node];
            float rx = p2x - p1x, ry = p2y - p1y;
            float d2 = rx * rx + ry * ry;
            int leaf = node >= nm1;
            if (leaf && ids[node - nm1] == body) continue; /* barnes_hut.wgsl:83-88 */
            float inv = 1.0f / sqrtf(d2 + soft2(p, m1, m2));
            if (leaf || length[node] * inv < theta) {       /* barnes_hut.wgsl:94 */
                float inv3 = inv * inv * inv;
                float gm = g * m2;
                ax += gm * rx * inv3;
                ay += gm * ry * inv3;
                ti++;
            } else if (L > 1 && last[node] - first[node] + 1 <= (uint32_t)L) {
                /* Extension: direct sum over the bucket's bodies in slot order. */
                for (uint32_t s = first[node]; s <= last[node]; ++s) {
                    if (s == (uint32_t)tid) continue;
                    uint32_t bj = ids[s];
                    float qx = pos[2 * bj] - p1x, qy = pos[2 * bj + 1] - p1y;
                    float mj = mass[bj];
                    float e2 = qx * qx + qy * qy;
                    float iv = 1.0f / sqrtf(e2 + soft2(p, m1, mj));
                    float iv3 = iv * iv * iv;
                    float gmj = g * mj;
                    ax += gmj * qx * iv3;
                    ay += gmj * qy * iv3;
                    ti++;
                }
            } else if (sp + 2 < STACK_SIZE) {               /* barnes_hut.wgsl:100-105 */
                sp += 1;
                stack[sp] = left[node];
                sp += 1;
                stack[sp] = right[node];
            }
        }
        if (acc) {
            acc[2 * body] = ax;
            acc[2 * body + 1] = ay;
        }
    }
    if (visits_out) *visits_out = tv;
    if (inter_out) *inter_out = ti;
    free(first);
    free(last);
}

void orc_walk(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
              const float* pos, const float* com, const float* mass_node, const float* length,
              const uint32_t* left, const uint32_t* right, float* acc) {
    walk_impl(p, n, ids, mass, pos, com, mass_node, length, left, right, acc, NULL, NULL);
}

void orc_walk_counts(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
                     const float* pos, const float* com, const float* mass_node,
                     const float* length, const uint32_t* left, const uint32_t* right,
                     uint64_t* visits, uint64_t* interactions) {
    walk_impl(p, n, ids, mass, pos, com, mass_node, length, left, right, NULL, visits,
              interactions);
}

/* ------------------------------------------------------------------------ */
/* Extension: quadrupole moments and the group walk                          */
/* ------------------------------------------------------------------------ */

void orc_quadrupoles(uint32_t n, const uint32_t* left, const uint32_t* right, const float* com,
                     const float* mass_node, float* quad) {
    const size_t nn = n ? 2 * (size_t)n - 1 : 0;
    memset(quad, 0, sizeof(float) * 3 * nn);
    if (n < 2) return;
    const uint32_t nm1 = n - 1;
    uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)n);
    uint8_t* seen = (uint8_t*)calloc(n, 1);
    int64_t sp = 0;
    st[sp++] = 0;
    while (sp > 0) {
        uint32_t v = st[sp - 1];
        if (v >= nm1) { sp--; continue; }
        if (!seen[v]) {
            seen[v] = 1;
            st[sp++] = left[v];
            st[sp++] = right[v];
            continue;
        }
        sp--;
        const uint32_t l = left[v], r = right[v];
        const float cx = com[2 * v], cy = com[2 * v + 1];
        const float ml = mass_node[l], mr = mass_node[r];
        const float dlx = com[2 * l] - cx, dly = com[2 * l + 1] - cy;
        const float drx = com[2 * r] - cx, dry = com[2 * r + 1] - cy;
        quad[3 * v] = (quad[3 * l] + ml * (dlx * dlx)) + (quad[3 * r] + mr * (drx * drx));
        quad[3 * v + 1] = (quad[3 * l + 1] + ml * (dlx * dly)) + (quad[3 * r + 1] + mr * (drx * dry));
        quad[3 * v + 2] = (quad[3 * l + 2] + ml * (dly * dly)) + (quad[3 * r + 2] + mr * (dry * dry));
    }
    free(st);
    free(seen);
}

/* Far field of the group walk (no reference counterpart): a node's
 * potential Phi = -[M g + 1/2 (Sxx g_xx + 2 Sxy g_xy + Syy g_yy)] with the
 * softened kernel g(R) = (|R|^2 + eps^2)^-1/2 is expanded about the group's
 * box centre.  d^(a,b) g = s^(a+b+1) P_ab(rho), s = (|R|^2 + eps^2)^-1/2,
 * rho = s R, with P_ab = sum_i sum_j c(a,i) c(b,j) rho_x^(a-2i) rho_y^(b-2j)
 * w(a+b-i-j), c(a,i) = a!/(i! (a-2i)! 2^i), w(m) = (-1)^m (2m-1)!!.  The
 * coefficients scaled by the length lambda (the box's half-diagonal),
 * C_ab = lambda^(a+b) d^(a,b) Phi for 1 <= a+b <= 4, are summed over the far
 * nodes; a body at x_g + lambda d feels
 *   a_x = -(1/lambda) sum_{a+b<=3} C_(a+1)b d_x^a d_y^b/(a! b!),  a_y likewise. */
#define ORC_FAR_COEFFS 14

static int far_index(int a, int b) { return (a + b - 1) * (a + b + 2) / 2 + b; }

static float fact_f(int k) {
    float v = 1.0f;
    for (int i = 2; i <= k; ++i) v *= (float)i;
    return v;
}

static float far_poly_c(int a, int b, const float* px, const float* py) {
    float acc = 0.0f;
    for (int i = 0; 2 * i <= a; ++i) {
        const float ca = fact_f(a) / (fact_f(i) * fact_f(a - 2 * i) * (float)(1 << i));
        for (int j = 0; 2 * j <= b; ++j) {
            const float cb = fact_f(b) / (fact_f(j) * fact_f(b - 2 * j) * (float)(1 << j));
            const int m = a + b - i - j;
            float w = 1.0f;
            for (int k = 1; k <= m; ++k) w *= -(float)(2 * k - 1);
            acc += ca * cb * w * (px[a - 2 * i] * py[b - 2 * j]);
        }
    }
    return acc;
}

/* Add the scaled coefficients of one node (COM offset R = x_g - c) to C. */
static void far_add_node(float* C, float rx, float ry, float m, float sxx, float sxy, float syy,
                         float lambda, float eps2) {
    const float u = (rx * rx + ry * ry) + eps2;
    const float s = (float)(1.0 / sqrt((double)u));
    float px[7], py[7];
    px[0] = 1.0f;
    py[0] = 1.0f;
    px[1] = rx * s;
    py[1] = ry * s;
    for (int k = 2; k < 7; ++k) {
        px[k] = px[k - 1] * px[1];
        py[k] = py[k - 1] * py[1];
    }
    const float t = lambda * s, s2 = s * s;
    const float qxx = s2 * sxx, qxy = s2 * sxy, qyy = s2 * syy;
    for (int o = 1; o <= 4; ++o) {
        float st = s;
        for (int k = 0; k < o; ++k) st *= t;
        for (int b = 0; b <= o; ++b) {
            const int a = o - b;
            const float quad = qxx * far_poly_c(a + 2, b, px, py) +
                               2.0f * qxy * far_poly_c(a + 1, b + 1, px, py) +
                               qyy * far_poly_c(a, b + 2, px, py);
            const float v = m * far_poly_c(a, b, px, py) + 0.5f * quad;
            C[far_index(a, b)] -= st * v;
        }
    }
}

/* The expansion's force at d (without the factor -1/lambda). */
static void far_force(const float* C, float dx, float dy, float* fx, float* fy) {
    float x = 0.0f, y = 0.0f;
    for (int a = 0; a <= 3; ++a)
        for (int b = 0; a + b <= 3; ++b) {
            float mono = 1.0f;
            for (int k = 0; k < a; ++k) mono *= dx;
            for (int k = 0; k < b; ++k) mono *= dy;
            mono /= fact_f(a) * fact_f(b);
            x += C[far_index(a + 1, b)] * mono;
            y += C[far_index(a, b + 1)] * mono;
        }
    *fx = x;
    *fy = y;
}

void orc_walk_group(const orc_params* p, uint32_t n, const uint32_t* ids, const float* mass,
                    const float* pos, const float* com, const float* mass_node, const float* aabb,
                    const float* quad, const uint32_t* left, const uint32_t* right, float* acc) {
    if (n == 0) return;
    const uint32_t nm1 = n - 1;
    const uint32_t G = 32u * (uint32_t)(p->bodies_per_lane > 0 ? p->bodies_per_lane : 2);
    const uint32_t L = (uint32_t)(p->leaf_size > 1 ? p->leaf_size : 1);
    const float th2 = p->bh_theta * p->bh_theta;
    const int plummer = p->softening == ORC_SOFT_PLUMMER;
    const float eps2 = p->plummer_eps * p->plummer_eps;
    const float ecoef = p->epsilon_multiplier * p->epsilon_multiplier * p->grav_constant * p->delta_time;
    uint32_t* first = (uint32_t*)malloc(sizeof(uint32_t) * (2 * (size_t)n - 1));
    uint32_t* last = (uint32_t*)malloc(sizeof(uint32_t) * (2 * (size_t)n - 1));
    node_ranges(n, left, right, first, last);
    /* Groups: the maximal subtrees of <= G bodies (contiguous slots of one cell). */
    uint32_t* gfirst = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* gcount = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t ngroups = 0;
    {
        uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)n);
        int64_t sp = 0;
        st[sp++] = n > 1 ? 0u : nm1;
        while (sp > 0) {
            const uint32_t v = st[--sp];
            const uint32_t c = last[v] - first[v] + 1;
            if (c <= G) {
                gfirst[ngroups] = first[v];
                gcount[ngroups++] = c;
            } else {
                st[sp++] = right[v];
                st[sp++] = left[v];
            }
        }
        free(st);
    }
#pragma omp parallel num_threads(nthreads(p))
    {
        /* Per-thread lists; a list never holds more than 2n-1 entries, so
         * capacity 2n can always hold a push. */
        size_t cap = 4096 < 2 * (size_t)n ? 4096 : 2 * (size_t)n;
        uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        uint32_t* nodes = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        uint32_t* rfirst = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        uint32_t* rcount = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        uint32_t* fars = (uint32_t*)malloc(sizeof(uint32_t) * cap);
#define ORC_GROW(need)                                                         \
        if ((size_t)(need) > cap) {                                            \
            cap = 2 * cap > (size_t)(need) ? 2 * cap : (size_t)(need);         \
            stack = (uint32_t*)realloc(stack, sizeof(uint32_t) * cap);         \
            nodes = (uint32_t*)realloc(nodes, sizeof(uint32_t) * cap);         \
            rfirst = (uint32_t*)realloc(rfirst, sizeof(uint32_t) * cap);       \
            rcount = (uint32_t*)realloc(rcount, sizeof(uint32_t) * cap);       \
            fars = (uint32_t*)realloc(fars, sizeof(uint32_t) * cap);           \
        }
#pragma omp for schedule(dynamic, 1)
        for (int64_t g = 0; g < (int64_t)ngroups; ++g) {
            const uint32_t base = gfirst[g];
            const uint32_t end = base + gcount[g];
            float lox = INFINITY, loy = INFINITY, hix = -INFINITY, hiy = -INFINITY;
            for (uint32_t s = base; s < end; ++s) {
                const uint32_t b = ids[s];
                lox = fminf(lox, pos[2 * b]); hix = fmaxf(hix, pos[2 * b]);
                loy = fminf(loy, pos[2 * b + 1]); hiy = fmaxf(hiy, pos[2 * b + 1]);
            }
            /* far field: box centre and squared half-diagonal */
            const float gcx = 0.5f * (lox + hix), gcy = 0.5f * (loy + hiy);
            const float ghx = hix - lox, ghy = hiy - loy;
            const float rg2 = 0.25f * (ghx * ghx + ghy * ghy);
            const float fa2 = p->far_alpha * p->far_alpha;
            const int far_on = plummer && p->multipole >= 2 && fa2 > 0.0f && rg2 > 0.0f;
            size_t nn_ = 0, nr = 0, nf = 0;
            int64_t sp = 0;
            if (n > 1) stack[sp++] = 0;
            while (sp > 0) {
                ORC_GROW((size_t)sp + 2);
                ORC_GROW(nn_ + 1);
                ORC_GROW(nr + 1);
                ORC_GROW(nf + 1);
                const uint32_t v = stack[--sp];
                if (v >= nm1) { rfirst[nr] = v - nm1; rcount[nr++] = 1; continue; }
                const float* bx = &aabb[4 * (size_t)v];
                const float cx = com[2 * (size_t)v], cy = com[2 * (size_t)v + 1];
                /* accept: size L < theta x distance from the group's box to the
                 * node's COM, and the two boxes apart */
                const float dx = fmaxf(0.0f, fmaxf(cx - hix, lox - cx));
                const float dy = fmaxf(0.0f, fmaxf(cy - hiy, loy - cy));
                const float d2 = dx * dx + dy * dy;
                const float Ls = fmaxf(bx[2] - bx[0], bx[3] - bx[1]);
                const float sx = fmaxf(bx[0] - hix, lox - bx[2]);
                const float sy = fmaxf(bx[1] - hiy, loy - bx[3]);
                if (Ls * Ls < th2 * d2 && (sx > 0.0f || sy > 0.0f)) {
                    const float ox = cx - gcx, oy = cy - gcy;
                    if (far_on && rg2 < fa2 * (ox * ox + oy * oy)) fars[nf++] = v;
                    else nodes[nn_++] = v;
                } else if (last[v] - first[v] + 1 <= L) {
                    rfirst[nr] = first[v];
                    rcount[nr++] = last[v] - first[v] + 1;
                } else {
                    stack[sp++] = right[v];
                    stack[sp++] = left[v];
                }
            }
            float C[ORC_FAR_COEFFS] = {0};
            const float lam = far_on ? sqrtf(rg2) : 1.0f;
            for (size_t j = 0; j < nf; ++j) {
                const uint32_t v = fars[j];
                far_add_node(C, gcx - com[2 * (size_t)v], gcy - com[2 * (size_t)v + 1],
                             mass_node[v], quad[3 * (size_t)v], quad[3 * (size_t)v + 1],
                             quad[3 * (size_t)v + 2], lam, eps2);
            }
            for (uint32_t s = base; s < end; ++s) {
                const uint32_t b = ids[s];
                const float x = pos[2 * b], y = pos[2 * b + 1], m1 = mass[b];
                float ax = 0.0f, ay = 0.0f;
                if (nf > 0) {
                    const float il = 1.0f / lam;
                    float fx, fy;
                    far_force(C, (x - gcx) * il, (y - gcy) * il, &fx, &fy);
                    ax = -(fx * il);
                    ay = -(fy * il);
                }
                for (size_t j = 0; j < nn_; ++j) {
                    const uint32_t v = nodes[j];
                    const float m2 = mass_node[v];
                    const float rx = com[2 * (size_t)v] - x, ry = com[2 * (size_t)v + 1] - y;
                    const float e2 = plummer ? eps2 : ecoef * fmaxf(m1, m2);
                    const float r2 = rx * rx + ry * ry + e2;
                    const float inv = 1.0f / sqrtf(r2);
                    const float inv2 = inv * inv, inv3 = inv * inv2;
                    if (p->multipole >= 2) {
                        const float sxx = quad[3 * (size_t)v], sxy = quad[3 * (size_t)v + 1],
                                    syy = quad[3 * (size_t)v + 2];
                        const float tr = sxx + syy;
                        const float qxx = 3.0f * sxx - tr, qxy = 3.0f * sxy, qyy = 3.0f * syy - tr;
                        const float qrx = qxx * rx + qxy * ry, qry = qxy * rx + qyy * ry;
                        const float rqr = rx * qrx + ry * qry;
                        const float inv5 = inv3 * inv2;
                        const float f = 2.5f * rqr * (inv5 * inv2) + m2 * inv3;
                        ax += f * rx - qrx * inv5;
                        ay += f * ry - qry * inv5;
                    } else {
                        const float f = m2 * inv3;
                        ax += f * rx;
                        ay += f * ry;
                    }
                }
                for (size_t j = 0; j < nr; ++j) {
                    for (uint32_t t = rfirst[j]; t < rfirst[j] + rcount[j]; ++t) {
                        if (t == s) continue;
                        const uint32_t bj = ids[t];
                        const float rx = pos[2 * bj] - x, ry = pos[2 * bj + 1] - y;
                        const float m2 = mass[bj];
                        const float e2 = plummer ? eps2 : ecoef * fmaxf(m1, m2);
                        const float inv = 1.0f / sqrtf(rx * rx + ry * ry + e2);
                        const float f = m2 * (inv * inv * inv);
                        ax += f * rx;
                        ay += f * ry;
                    }
                }
                acc[2 * b] = p->grav_constant * ax;
                acc[2 * b + 1] = p->grav_constant * ay;
            }
        }
#undef ORC_GROW
        free(stack);
        free(nodes);
        free(rfirst);
        free(rcount);
        free(fars);
    }
    free(gfirst);
    free(gcount);
    free(first);
    free(last);
}

/* ------------------------------------------------------------------------ */
/* FP64 direct sum (accuracy oracle; no reference counterpart)               */
/* ------------------------------------------------------------------------ */

void orc_direct_sum_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                         uint32_t nsample, const uint32_t* sample, double* acc_out) {
    const double g = p->grav_constant;
#pragma omp parallel for num_threads(nthreads(p)) schedule(dynamic, 4)
    for (int64_t k = 0; k < (int64_t)nsample; ++k) {
        uint32_t i = sample[k];
        double xi = pos[2 * i], yi = pos[2 * i + 1], mi = mass[i];
        double ax = 0.0, ay = 0.0;
        for (uint32_t j = 0; j < n; ++j) {
            if (j == i) continue;
            double rx = (double)pos[2 * j] - xi, ry = (double)pos[2 * j + 1] - yi;
            double mj = mass[j], e2;
            if (p->softening == ORC_SOFT_PLUMMER) {
                e2 = (double)p->plummer_eps * (double)p->plummer_eps;
            } else {
                double meff = mi > mj ? mi : mj;
                double eps = (double)p->epsilon_multiplier * sqrt(g * meff * (double)p->delta_time);
                e2 = eps * eps;
            }
            double r2 = rx * rx + ry * ry + e2;
            double inv = 1.0 / sqrt(r2);
            double f = g * mj * inv * inv * inv;
            ax += f * rx;
            ay += f * ry;
        }
        acc_out[2 * k] = ax;
        acc_out[2 * k + 1] = ay;
    }
}

/* ------------------------------------------------------------------------ */
/* FP64 direct-sum rollout adjoint (no reference counterpart)                */
/* ------------------------------------------------------------------------ */

/* a_i = G sum_{j != i} m_j r_ij s_ij^3, r_ij = x_j - x_i, s = (r.r + eps^2)^-1/2 */
static void ds_accel(int nt, uint32_t n, double G, double e2, const double* m, const double* x,
                     double* a) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double ax = 0.0, ay = 0.0;
        for (uint32_t j = 0; j < n; ++j) {
            if ((int64_t)j == i) continue;
            double rx = x[2 * j] - x[2 * i], ry = x[2 * j + 1] - x[2 * i + 1];
            double s = 1.0 / sqrt(rx * rx + ry * ry + e2);
            double f = m[j] * s * s * s;
            ax += f * rx;
            ay += f * ry;
        }
        a[2 * i] = G * ax;
        a[2 * i + 1] = G * ay;
    }
}

/* (xbar, mbar) += (da/dx, da/dm)^T abar.  With rbar_ij = m_j (s^3 ab_i -
 * 3 s^5 (ab_i.r) r): xbar_i -= sum_j rbar_ij, xbar_j += sum_i rbar_ij,
 * mbar_j += sum_i s^3 (ab_i.r).  Two passes keep every write private. */
static void ds_vjp(int nt, uint32_t n, double G, double e2, const double* m, const double* x,
                   const double* ab, double* xbar, double* mbar) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double bx = 0.0, by = 0.0;
        const double ax = G * ab[2 * i], ay = G * ab[2 * i + 1];
        for (uint32_t j = 0; j < n; ++j) {
            if ((int64_t)j == i) continue;
            double rx = x[2 * j] - x[2 * i], ry = x[2 * j + 1] - x[2 * i + 1];
            double s = 1.0 / sqrt(rx * rx + ry * ry + e2), s3 = s * s * s, s5 = s3 * s * s;
            double ar = ax * rx + ay * ry;
            bx += m[j] * (s3 * ax - 3.0 * s5 * ar * rx);
            by += m[j] * (s3 * ay - 3.0 * s5 * ar * ry);
        }
        xbar[2 * i] -= bx;
        xbar[2 * i + 1] -= by;
    }
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t j = 0; j < (int64_t)n; ++j) {
        double bx = 0.0, by = 0.0, bm = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            if ((int64_t)i == j) continue;
            const double ax = G * ab[2 * i], ay = G * ab[2 * i + 1];
            double rx = x[2 * j] - x[2 * i], ry = x[2 * j + 1] - x[2 * i + 1];
            double s = 1.0 / sqrt(rx * rx + ry * ry + e2), s3 = s * s * s, s5 = s3 * s * s;
            double ar = ax * rx + ay * ry;
            bx += m[j] * (s3 * ax - 3.0 * s5 * ar * rx);
            by += m[j] * (s3 * ay - 3.0 * s5 * ar * ry);
            bm += s3 * ar;
        }
        xbar[2 * j] += bx;
        xbar[2 * j + 1] += by;
        mbar[j] += bm;
    }
}

void orc_force_vjp_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                        const float* abar, double* xbar, double* mbar) {
    const size_t n2 = 2 * (size_t)n;
    double* m = (double*)malloc(sizeof(double) * n);
    double* x = (double*)malloc(sizeof(double) * n2);
    double* ab = (double*)malloc(sizeof(double) * n2);
    for (uint32_t i = 0; i < n; ++i) m[i] = mass[i];
    for (size_t k = 0; k < n2; ++k) {
        x[k] = pos[k];
        ab[k] = abar[k];
        xbar[k] = 0.0;
    }
    for (uint32_t i = 0; i < n; ++i) mbar[i] = 0.0;
    ds_vjp(nthreads(p), n, p->grav_constant, (double)p->plummer_eps * (double)p->plummer_eps, m,
           x, ab, xbar, mbar);
    free(m); free(x); free(ab);
}

double orc_rollout_grad_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                             const float* vel, const float* target, uint32_t steps, double* gx,
                             double* gv, double* gm) {
    const int nt = nthreads(p);
    const double G = p->grav_constant, dt = p->delta_time, h = 0.5 * dt;
    const double e2 = (double)p->plummer_eps * (double)p->plummer_eps;
    const size_t n2 = 2 * (size_t)n;
    double* m = (double*)malloc(sizeof(double) * n);
    double* xs = (double*)malloc(sizeof(double) * n2 * (steps + 1)); /* x_0 .. x_T */
    double* v = (double*)malloc(sizeof(double) * n2);
    double* a = (double*)malloc(sizeof(double) * n2);
    double* ab = (double*)malloc(sizeof(double) * n2);
    double* ap = (double*)calloc(n2, sizeof(double));
    for (uint32_t i = 0; i < n; ++i) m[i] = mass[i];
    for (size_t k = 0; k < n2; ++k) {
        xs[k] = pos[k];
        v[k] = vel[k];
    }
    ds_accel(nt, n, G, e2, m, xs, a);
    for (uint32_t t = 0; t < steps; ++t) {
        const double* x0 = xs + n2 * t;
        double* x1 = xs + n2 * (t + 1);
        for (size_t k = 0; k < n2; ++k) {
            v[k] += h * a[k];
            x1[k] = x0[k] + dt * v[k];
        }
        ds_accel(nt, n, G, e2, m, x1, a);
        for (size_t k = 0; k < n2; ++k) v[k] += h * a[k];
    }
    const double* xT = xs + n2 * steps;
    double L = 0.0;
    for (size_t k = 0; k < n2; ++k) {
        double d = xT[k] - target[k];
        L += d * d / n;
        gx[k] = 2.0 * d / n;
        gv[k] = 0.0;
    }
    for (uint32_t i = 0; i < n; ++i) gm[i] = 0.0;
    for (int64_t t = (int64_t)steps - 1; t >= 0; --t) {
        for (size_t k = 0; k < n2; ++k) ab[k] = ap[k] + h * gv[k];
        ds_vjp(nt, n, G, e2, m, xs + n2 * (t + 1), ab, gx, gm);
        for (size_t k = 0; k < n2; ++k) {
            gv[k] += dt * gx[k];
            ap[k] = h * gv[k];
        }
    }
    ds_vjp(nt, n, G, e2, m, xs, ap, gx, gm);
    free(m); free(xs); free(v); free(a); free(ab); free(ap);
    return L;
}

/* ------------------------------------------------------------------------ */
/* Whole-step state (simulation.ts:82-91 buffers, :386-425 stage order)      */
/* ------------------------------------------------------------------------ */

struct orc_state {
    orc_params p;
    uint32_t n;
    float *mass, *pos, *vel, *acc;
    int acc_valid;
    uint64_t* codes;
    uint32_t *ids, *left, *right, *parent;
    float *com, *mass_node, *aabb, *length;
    float* quad; /* group walk: second moments */
};

orc_state* orc_create(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                      const float* vel) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    s->p = *p;
    s->n = n;
    size_t nn = n ? 2 * (size_t)n - 1 : 1;
    size_t nb = n ? n : 1;
    s->mass = (float*)malloc(sizeof(float) * nb);
    s->pos = (float*)malloc(sizeof(float) * 2 * nb);
    s->vel = (float*)malloc(sizeof(float) * 2 * nb);
    s->acc = (float*)calloc(2 * nb, sizeof(float));
    s->codes = (uint64_t*)malloc(sizeof(uint64_t) * nb);
    s->ids = (uint32_t*)malloc(sizeof(uint32_t) * nb);
    s->left = (uint32_t*)calloc(nn, sizeof(uint32_t));
    s->right = (uint32_t*)calloc(nn, sizeof(uint32_t));
    s->parent = (uint32_t*)calloc(nn, sizeof(uint32_t));
    s->com = (float*)calloc(2 * nn, sizeof(float));
    s->mass_node = (float*)calloc(nn, sizeof(float));
    s->aabb = (float*)calloc(4 * nn, sizeof(float));
    s->length = (float*)calloc(nn, sizeof(float));
    s->quad = (float*)calloc(3 * nn, sizeof(float));
    if (n) {
        memcpy(s->mass, mass, sizeof(float) * n);
        memcpy(s->pos, pos, sizeof(float) * 2 * n);
        memcpy(s->vel, vel, sizeof(float) * 2 * n);
    }
    return s;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    free(s->mass); free(s->pos); free(s->vel); free(s->acc);
    free(s->codes); free(s->ids); free(s->left); free(s->right); free(s->parent);
    free(s->com); free(s->mass_node); free(s->aabb); free(s->length); free(s->quad);
    free(s);
}

/* Morton -> sort -> build -> fill (simulation.ts:395-410). */
static void build_tree(orc_state* s) {
    orc_domain dom;
    orc_domain_compute(&s->p, s->n, s->pos, &dom);
    orc_morton(&s->p, &dom, s->n, s->pos, s->codes, s->ids);
    radix_sort_impl(s->n, s->codes, s->ids, s->p.morton_bits, nthreads(&s->p));
    orc_build(s->n, s->p.morton_bits, s->codes, s->left, s->right, s->parent);
    orc_fill(s->n, 0, s->ids, s->mass, s->pos, s->left, s->right, s->parent, s->com,
             s->mass_node, s->aabb, s->length);
}

static void forces(orc_state* s) {
    build_tree(s);
    if (s->p.walk_mode == 1) {
        orc_quadrupoles(s->n, s->left, s->right, s->com, s->mass_node, s->quad);
        orc_walk_group(&s->p, s->n, s->ids, s->mass, s->pos, s->com, s->mass_node, s->aabb,
                       s->quad, s->left, s->right, s->acc);
    } else {
        walk_impl(&s->p, s->n, s->ids, s->mass, s->pos, s->com, s->mass_node, s->length, s->left,
                  s->right, s->acc, NULL, NULL);
    }
    s->acc_valid = 1;
}

void orc_accelerations(orc_state* s, float* acc) {
    forces(s);
    if (acc) memcpy(acc, s->acc, sizeof(float) * 2 * s->n);
}

void orc_step(orc_state* s, uint32_t nsteps) {
    const uint32_t n = s->n;
    const float dt = s->p.delta_time;
    const int nt = nthreads(&s->p);
    if (n == 0) return;
    for (uint32_t step = 0; step < nsteps; ++step) {
        if (s->p.integrator == ORC_INT_LEAPFROG_KDK) {
            /* Extension: kick-drift-kick with the force of the previous step cached. */
            const float hdt = 0.5f * dt;
            if (!s->acc_valid) forces(s);
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int64_t b = 0; b < (int64_t)n; ++b) {
                float vx = s->vel[2 * b] + s->acc[2 * b] * hdt;
                float vy = s->vel[2 * b + 1] + s->acc[2 * b + 1] * hdt;
                s->vel[2 * b] = vx;
                s->vel[2 * b + 1] = vy;
                s->pos[2 * b] = s->pos[2 * b] + vx * dt;
                s->pos[2 * b + 1] = s->pos[2 * b + 1] + vy * dt;
            }
            forces(s);
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int64_t b = 0; b < (int64_t)n; ++b) {
                s->vel[2 * b] = s->vel[2 * b] + s->acc[2 * b] * hdt;
                s->vel[2 * b + 1] = s->vel[2 * b + 1] + s->acc[2 * b + 1] * hdt;
            }
        } else {
            /* Reference: kick (barnes_hut.wgsl:110) then drift (:119-120). */
            forces(s);
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int64_t b = 0; b < (int64_t)n; ++b) {
                float vx = s->vel[2 * b] + s->acc[2 * b] * dt;
                float vy = s->vel[2 * b + 1] + s->acc[2 * b + 1] * dt;
                s->vel[2 * b] = vx;
                s->vel[2 * b + 1] = vy;
                s->pos[2 * b] = s->pos[2 * b] + vx * dt;
                s->pos[2 * b + 1] = s->pos[2 * b + 1] + vy * dt;
            }
            s->acc_valid = 0;
        }
    }
}

void orc_get_state(const orc_state* s, float* pos, float* vel) {
    if (pos) memcpy(pos, s->pos, sizeof(float) * 2 * s->n);
    if (vel) memcpy(vel, s->vel, sizeof(float) * 2 * s->n);
}

void orc_get_tree(const orc_state* s, uint64_t* codes, uint32_t* ids, uint32_t* left,
                  uint32_t* right, uint32_t* parent, float* com, float* mass_node, float* aabb,
                  float* length) {
    size_t n = s->n, nn = n ? 2 * n - 1 : 0;
    if (codes) memcpy(codes, s->codes, sizeof(uint64_t) * n);
    if (ids) memcpy(ids, s->ids, sizeof(uint32_t) * n);
    if (left) memcpy(left, s->left, sizeof(uint32_t) * nn);
    if (right) memcpy(right, s->right, sizeof(uint32_t) * nn);
    if (parent) memcpy(parent, s->parent, sizeof(uint32_t) * nn);
    if (com) memcpy(com, s->com, sizeof(float) * 2 * nn);
    if (mass_node) memcpy(mass_node, s->mass_node, sizeof(float) * nn);
    if (aabb) memcpy(aabb, s->aabb, sizeof(float) * 4 * nn);
    if (length) memcpy(length, s->length, sizeof(float) * nn);
}

uint32_t orc_num_bodies(const orc_state* s) { return s->n; }


/* ---- density render (renderer.ts:293-329) -------------------------------- */

/* density.wgsl:39-97.  Pixel-space form of the vertex + fragment stages:
 * centre_ndc = (p - cam_centre) / cam_half (density.wgsl:60-62), radius
 * 2 * rm pixels (:64-66), uv = (pixel centre - centre) / radius, discard
 * |uv| > 1 (:76-78), w = exp(-k r r) with k = 10 (:81-82), zoom_scale =
 * 1 / (1 + 0.05 max(half)) (:86-88), base 0.1 when rm > 1 else 0.02
 * (:90-93); evaluated as (base zoom_scale) exp(-10 |uv|^2) with uv scaled
 * by 1 / radius, as the CUDA kernel does. */
float orc_splat_weight(float ux, float uy, float radius_multiplier, float zoom_scale,
                       int* discarded) {
    const float r2 = ux * ux + uy * uy;
    *discarded = r2 > 1.0f;
    if (*discarded) return 0.0f;
    const float bw = (radius_multiplier > 1.0f ? 0.1f : 0.02f) * zoom_scale;
    return bw * expf(-10.0f * r2);
}

void orc_render_density(const float cam[4], uint32_t width, uint32_t height, uint32_t n,
                        const float* pos, const float* radius_multiplier, double* density) {
    const float W = (float)width, H = (float)height;
    const float zoom = cam[2] > cam[3] ? cam[2] : cam[3];
    const float zoom_scale = 1.0f / (1.0f + 0.05f * zoom);
    memset(density, 0, sizeof(double) * (size_t)width * height);
    for (uint32_t b = 0; b < n; ++b) {
        const float x = pos[2 * b], y = pos[2 * b + 1], rm = radius_multiplier[b];
        const float cnx = (x - cam[0]) / cam[2];
        const float cny = (y - cam[1]) / cam[3];
        const float R = 2.0f * rm;
        const float cpx = ((cnx + 1.0f) * 0.5f) * W;
        const float cpy = ((cny + 1.0f) * 0.5f) * H;
        if (!isfinite(cpx) || !isfinite(cpy) || !(R > 0.0f) || !isfinite(R)) continue;
        float i0 = ceilf(cpx - R - 0.5f), i1 = floorf(cpx + R - 0.5f);
        float j0 = ceilf(cpy - R - 0.5f), j1 = floorf(cpy + R - 0.5f);
        if (i0 < 0.0f) i0 = 0.0f;
        if (j0 < 0.0f) j0 = 0.0f;
        if (i1 > W - 1.0f) i1 = W - 1.0f;
        if (j1 > H - 1.0f) j1 = H - 1.0f;
        if (!(i0 <= i1) || !(j0 <= j1)) continue;
        const float inv_r = 1.0f / R;
        for (uint32_t j = (uint32_t)j0; j <= (uint32_t)j1; ++j) {
            for (uint32_t i = (uint32_t)i0; i <= (uint32_t)i1; ++i) {
                const float ux = (((float)i + 0.5f) - cpx) * inv_r;
                const float uy = (((float)j + 0.5f) - cpy) * inv_r;
                int discarded;
                const float w = orc_splat_weight(ux, uy, rm, zoom_scale, &discarded);
                if (!discarded) density[(size_t)j * width + i] += (double)w;
            }
        }
    }
}

static float orc_mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }

/* tone_map.wgsl:24-46 */
void orc_colormap(float t, float rgb[3]) {
    static const float c[4][3] = {{0.0f, 0.0f, 0.0f}, {0.10f, 0.20f, 0.90f},
                                  {0.20f, 0.90f, 0.90f}, {1.0f, 1.0f, 1.0f}};
    const float x = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
    int seg;
    float a;
    if (x < 0.33f) {
        seg = 0;
        a = x / 0.33f;
    } else if (x < 0.66f) {
        seg = 1;
        a = (x - 0.33f) / 0.33f;
    } else {
        seg = 2;
        a = (x - 0.66f) / 0.34f;
    }
    for (int k = 0; k < 3; ++k) rgb[k] = orc_mix(c[seg][k], c[seg + 1][k], a);
}

static uint8_t orc_unorm8(float c) {
    const float v = (c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c)) * 255.0f;
    return (uint8_t)lrintf(v);
}

void orc_tone_map_rgb(float texel, float rgb[3]) {
    const float gamma = (float)(1.0 / 2.2);
    const float x = 8.0f * texel;
    const float mapped = x / (1.0f + x);
    const float m = mapped < 0.0f ? 0.0f : (mapped > 1.0f ? 1.0f : mapped);
    orc_colormap(powf(m, gamma), rgb);
}

/* tone_map.wgsl:63-84 (the r16float texel is the density rounded to FP16) */
void orc_tone_map(uint32_t pixels, const float* density, uint8_t* rgba) {
    for (uint32_t p = 0; p < pixels; ++p) {
        float rgb[3];
        orc_tone_map_rgb((float)(_Float16)density[p], rgb);
        rgba[4 * (size_t)p] = orc_unorm8(rgb[0]);
        rgba[4 * (size_t)p + 1] = orc_unorm8(rgb[1]);
        rgba[4 * (size_t)p + 2] = orc_unorm8(rgb[2]);
        rgba[4 * (size_t)p + 3] = 255;
    }
}


/* ---- FP64 diagnostics ----------------------------------------------------- */

void orc_diagnostics_fp64(const orc_params* p, uint32_t n, const float* mass, const float* pos,
                          const float* vel, double out[8]) {
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = 0; i < n; ++i) {
        const double m = mass[i], x = pos[2 * i], y = pos[2 * i + 1];
        const double vx = vel[2 * i], vy = vel[2 * i + 1];
        a[0] += m;
        a[1] += m * x;
        a[2] += m * y;
        a[3] += m * vx;
        a[4] += m * vy;
        a[5] += m * (x * vy - y * vx);
        a[6] += 0.5 * m * (vx * vx + vy * vy);
    }
    const double G = p->grav_constant;
    /* the engine forms this coefficient in f32 (epsMult^2 G dt) */
    const double coef = (double)(p->epsilon_multiplier * p->epsilon_multiplier * p->grav_constant *
                                 p->delta_time);
    const double e2p = (double)p->plummer_eps * p->plummer_eps;
    double W = 0.0;
#pragma omp parallel for reduction(+ : W) schedule(dynamic, 64)
    for (uint32_t i = 0; i < n; ++i) {
        const double mi = mass[i], xi = pos[2 * i], yi = pos[2 * i + 1];
        double s = 0.0;
        for (uint32_t j = i + 1; j < n; ++j) {
            const double mj = mass[j];
            const double dx = pos[2 * j] - xi, dy = pos[2 * j + 1] - yi;
            const double e2 = p->softening == 1 ? e2p : coef * (mi > mj ? mi : mj);
            const double r2 = dx * dx + dy * dy + e2;
            if (r2 > 0.0) s += mj / sqrt(r2);
        }
        W += mi * s;
    }
    out[0] = a[0];
    out[1] = a[0] > 0.0 ? a[1] / a[0] : 0.0;
    out[2] = a[0] > 0.0 ? a[2] / a[0] : 0.0;
    out[3] = a[3];
    out[4] = a[4];
    out[5] = a[5];
    out[6] = a[6];
    out[7] = -G * W;
}


/* ---- scenarios with one PCG32 stream per body ------------------------------ */

#define ORC_PI 3.14159265358979323846 /* M_PI of <math.h> (not declared under -std=c11) */

typedef struct orc_pcg {
    uint64_t state, inc;
} orc_pcg;

static uint32_t orc_pcg_next(orc_pcg* r) {
    const uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

/* PCG32 (O'Neill 2014): increment 2 seq + 1, state advanced, seeded, advanced */
static orc_pcg orc_pcg_make(uint64_t seed, uint64_t seq) {
    orc_pcg r = {0, (seq << 1u) | 1u};
    orc_pcg_next(&r);
    r.state += seed;
    orc_pcg_next(&r);
    return r;
}

static double orc_pcg_uniform(orc_pcg* r) {
    const uint64_t a = orc_pcg_next(r) >> 5, b = orc_pcg_next(r) >> 6;
    return (double)(a * 67108864ULL + b) * (1.0 / 9007199254740992.0);
}

static double orc_pcg_normal(orc_pcg* r) {
    double u1 = orc_pcg_uniform(r);
    const double u2 = orc_pcg_uniform(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(2.0 * ORC_PI * u2);
}

static uint64_t orc_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

static void orc_put(float* mass, float* pos, float* vel, uint32_t i, double m, double x, double y,
                    double vx, double vy) {
    mass[i] = (float)m;
    pos[2 * i] = (float)x;
    pos[2 * i + 1] = (float)y;
    vel[2 * i] = (float)vx;
    vel[2 * i + 1] = (float)vy;
}

#define ORC_MIX_K 64

static void orc_mixture_point(uint64_t seed, const double* cx, const double* cy, const double* sig,
                              uint32_t j, float* x, float* y) {
    for (;;) {
        orc_pcg r = orc_pcg_make(seed, orc_splitmix64(j));
        (void)orc_pcg_normal(&r); /* the body's mass draw */
        if (j > 0 && orc_pcg_uniform(&r) < 0.01) {
            j = (uint32_t)(orc_pcg_uniform(&r) * (double)j);
            continue;
        }
        int k = (int)(orc_pcg_uniform(&r) * ORC_MIX_K);
        if (k >= ORC_MIX_K) k = ORC_MIX_K - 1;
        const double px = cx[k] + sig[k] * orc_pcg_normal(&r);
        const double py = cy[k] + sig[k] * orc_pcg_normal(&r);
        *x = (float)px;
        *y = (float)py;
        return;
    }
}

int orc_generate_per_body(const char* name, uint32_t n, uint64_t seed, double G, float* mass,
                          float* pos, float* vel, float* radius) {
    int sc;
    if (!name) return -1;
    if (!strcmp(name, "default")) sc = 0;
    else if (!strcmp(name, "two-clusters")) sc = 1;
    else if (!strcmp(name, "planetary-disk")) sc = 2;
    else if (!strcmp(name, "uniform-disk-kepler")) sc = 3;
    else if (!strcmp(name, "colliding-disks")) sc = 4;
    else if (!strcmp(name, "gaussian-mixture")) sc = 5;
    else if (!strcmp(name, "plummer-projection")) sc = 6;
    else return -1;
    double cx[ORC_MIX_K], cy[ORC_MIX_K], sig[ORC_MIX_K];
    if (sc == 5) {
        orc_pcg r = orc_pcg_make(seed, 0x5851f42d4c957f2dULL);
        for (int k = 0; k < ORC_MIX_K; ++k) {
            cx[k] = -4.0 + 8.0 * orc_pcg_uniform(&r);
            cy[k] = -4.0 + 8.0 * orc_pcg_uniform(&r);
            sig[k] = exp(log(1e-3) + (log(0.5) - log(1e-3)) * orc_pcg_uniform(&r));
        }
    }
    double total = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        if (radius) radius[i] = 1.0f;
        orc_pcg r = orc_pcg_make(seed, orc_splitmix64(i));
        if (sc == 0) { /* simulation.ts:243-266 */
            const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
            const double rr = 5.0 * sqrt(orc_pcg_uniform(&r));
            const double x = rr * cos(angle), y = rr * sin(angle);
            const double dist = sqrt(x * x + y * y);
            const double speed = 0.1 * sqrt(G * (double)n / dist);
            orc_put(mass, pos, vel, i, 1.0, x, y, -speed * (y / dist), speed * (x / dist));
        } else if (sc == 1) { /* simulation.ts:267-306 */
            const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
            const double rr = 3.0 * sqrt(orc_pcg_uniform(&r));
            const double xb = rr * cos(angle), yb = rr * sin(angle);
            const int first = (double)i < (double)n / 2.0;
            const double dist = sqrt(xb * xb + yb * yb);
            const double speed = 0.12 * sqrt(G * ((double)n / 2.0) / dist);
            orc_put(mass, pos, vel, i, 1.0, first ? xb - 15.0 : xb + 15.0, yb,
                    first ? -speed * (yb / dist) : speed * (yb / dist),
                    first ? speed * (xb / dist) : -speed * (xb / dist));
        } else if (sc == 2) { /* simulation.ts:308-361 */
            const double central = 1000.0, planet = 10.0;
            if (i == 0) {
                orc_put(mass, pos, vel, i, central, 0.0, 0.0, 0.0, 0.0);
                if (radius) radius[i] = 12.0f;
            } else if (i == 1) {
                orc_put(mass, pos, vel, i, planet, 2.5, 0.0, 0.0, 0.8 * sqrt(G * central / 2.5));
                if (radius) radius[i] = 5.0f;
            } else if (i == 2) {
                orc_put(mass, pos, vel, i, planet, 12.0, 0.0, 0.0, sqrt(G * central / 12.5));
                if (radius) radius[i] = 5.0f;
            } else {
                const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
                const double rr = sqrt(orc_pcg_uniform(&r) * (15.0 * 15.0 - 0.1 * 0.1) + 0.1 * 0.1);
                const double x = rr * cos(angle), y = rr * sin(angle);
                const double dist = sqrt(x * x + y * y);
                const double speed = 1.01 * sqrt(G * central / (2.0 + dist));
                orc_put(mass, pos, vel, i, central / (100.0 * (double)n), x, y, -speed * (y / dist),
                        speed * (x / dist));
            }
        } else if (sc == 3) { /* uniform disk, Keplerian about M(<r) = r^2 */
            const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
            const double rr = sqrt(orc_pcg_uniform(&r));
            const double x = rr * cos(angle), y = rr * sin(angle);
            const double v = sqrt(G * rr * rr / (rr > 1e-12 ? rr : 1e-12));
            const double c = rr > 0 ? x / rr : 1.0, s = rr > 0 ? y / rr : 0.0;
            orc_put(mass, pos, vel, i, 1.0 / (double)n, x, y, -v * s, v * c);
        } else if (sc == 4) { /* two colliding exponential disks */
            const double h = 0.2, rmax = 10.0 * h, md = 1.0 / 2.2, mc = 0.1 * md;
            const uint32_t half = n / 2;
            const int gal = i < half ? 0 : 1;
            const uint32_t lo = gal == 0 ? 0 : half, hi = gal == 0 ? half : n, cnt = hi - lo;
            const double gx = gal == 0 ? 1.5 : -1.5;
            const double bvx = gal == 0 ? -0.3 : 0.3, bvy = gal == 0 ? 0.1 : -0.1;
            if (i == lo) {
                orc_put(mass, pos, vel, i, cnt > 1 ? mc : md + mc, gx, 0.0, bvx, bvy);
                continue;
            }
            double R = rmax;
            for (int t = 0; t < 64; ++t) {
                double u1 = orc_pcg_uniform(&r), u2 = orc_pcg_uniform(&r);
                if (u1 < 1e-300) u1 = 1e-300;
                if (u2 < 1e-300) u2 = 1e-300;
                R = -h * log(u1 * u2);
                if (R <= rmax) break;
            }
            if (R > rmax) R = rmax;
            const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
            const double x = R * cos(angle), y = R * sin(angle);
            const double menc = mc + md * (1.0 - (1.0 + R / h) * exp(-R / h));
            const double Rs = R > 1e-6 ? R : 1e-6;
            const double v = sqrt(G * menc / Rs);
            orc_put(mass, pos, vel, i, md / (double)(cnt - 1), gx + x, y, bvx - v * (y / Rs),
                    bvy + v * (x / Rs));
        } else if (sc == 5) { /* Gaussian mixture, 1% duplicates, log-normal masses */
            const double m = exp(orc_pcg_normal(&r));
            total += (double)(float)m;
            mass[i] = (float)m;
            orc_mixture_point(seed, cx, cy, sig, i, &pos[2 * i], &pos[2 * i + 1]);
            vel[2 * i] = 0.0f;
            vel[2 * i + 1] = 0.0f;
        } else { /* projected Plummer sphere, a = 0.1 */
            const double a = 0.1;
            const double u = orc_pcg_uniform(&r) * 0.999;
            const double R = a * sqrt(u / (1.0 - u));
            const double angle = orc_pcg_uniform(&r) * 2.0 * ORC_PI;
            const double x = R * cos(angle), y = R * sin(angle);
            const double menc = R * R / (R * R + a * a);
            const double Rs = R > 1e-9 ? R : 1e-9;
            const double v = sqrt(G * menc / Rs);
            orc_put(mass, pos, vel, i, 1.0 / (double)n, x, y, -v * (y / Rs), v * (x / Rs));
        }
    }
    if (sc == 5 && total > 0.0)
        for (uint32_t i = 0; i < n; ++i) mass[i] = (float)((double)mass[i] / total);
    return 0;
}
