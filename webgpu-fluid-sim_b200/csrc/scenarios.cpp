// scenarios.cpp -- seeded initial conditions.
//
// The reference generates its three scenarios on the CPU from Math.random()
// (src/simulation.ts:233-374).  Here every draw comes from PCG32 (O'Neill
// 2014, the pcg32 XSH-RR output function) seeded by the caller, so runs are
// reproducible.  Arithmetic is done in double, like JavaScript numbers, and
// stored as float, like the reference's Float32Array.
//
// Benchmark generators (no reference counterpart) follow the body-count,
// distribution and unit choices stated beside each.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

namespace bh {

struct Pcg32 {
    uint64_t state = 0, inc = 0;
    explicit Pcg32(uint64_t seed, uint64_t seq = 0x5851f42d4c957f2dULL) {
        inc = (seq << 1u) | 1u;
        next();
        state += seed;
        next();
    }
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    // Uniform double in [0, 1) with 53 random bits (the role of Math.random()).
    double uniform() {
        uint64_t a = next() >> 5, b = next() >> 6;
        return (double)(a * 67108864ULL + b) * (1.0 / 9007199254740992.0);
    }
    double normal() {  // Box-Muller
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
};

static void set_body(float* mass, float* pos, float* vel, uint32_t i, double m, double x,
                     double y, double vx, double vy) {
    mass[i] = (float)m;
    pos[2 * i] = (float)x;
    pos[2 * i + 1] = (float)y;
    vel[2 * i] = (float)vx;
    vel[2 * i + 1] = (float)vy;
}

// simulation.ts:243-266 "default": disk of radius 5, mass 1 per body,
// circular speed 0.1*sqrt(G*N/r).
static void gen_default(uint32_t n, Pcg32& rng, double G, float* mass, float* pos, float* vel) {
    const double radius = 5.0, speed_factor = 0.1;
    for (uint32_t i = 0; i < n; ++i) {
        double angle = rng.uniform() * 2.0 * M_PI;
        double r = radius * std::sqrt(rng.uniform());
        double x = r * std::cos(angle), y = r * std::sin(angle);
        double dist = std::sqrt(x * x + y * y);
        double speed = speed_factor * std::sqrt(G * (double)n / dist);
        set_body(mass, pos, vel, i, 1.0, x, y, -speed * (y / dist), speed * (x / dist));
    }
}

// simulation.ts:267-306 "two-clusters": two disks of radius 3 at x = -15 and
// x = +15 spinning in opposite directions.
static void gen_two_clusters(uint32_t n, Pcg32& rng, double G, float* mass, float* pos, float* vel) {
    const double offset = 15.0, radius = 3.0, speed_factor = 0.12;
    for (uint32_t i = 0; i < n; ++i) {
        double angle = rng.uniform() * 2.0 * M_PI;
        double r = radius * std::sqrt(rng.uniform());
        double xb = r * std::cos(angle), yb = r * std::sin(angle);
        bool first = (double)i < (double)n / 2.0;
        double x = first ? xb - offset : xb + offset, y = yb;
        double dist = std::sqrt(xb * xb + yb * yb);
        double speed = speed_factor * std::sqrt(G * ((double)n / 2.0) / dist);
        double vx = first ? -speed * (yb / dist) : speed * (yb / dist);
        double vy = first ? speed * (xb / dist) : -speed * (xb / dist);
        set_body(mass, pos, vel, i, 1.0, x, y, vx, vy);
    }
}

// simulation.ts:308-361 "planetary-disk": central mass 1000, two planets of
// mass 10, and n-3 bodies of mass 1000/(100 n) in an annulus [0.1, 15].
static void gen_planetary_disk(uint32_t n, Pcg32& rng, double G, float* mass, float* pos,
                               float* vel, float* radius_mul) {
    const double disk_max = 15.0, disk_min = 0.1, central = 1000.0, planet = 10.0;
    const double body_mass = central / (100.0 * (double)n);
    if (n > 0) {
        set_body(mass, pos, vel, 0, central, 0.0, 0.0, 0.0, 0.0);
        if (radius_mul) radius_mul[0] = 12.0f;
    }
    if (n > 1) {
        set_body(mass, pos, vel, 1, planet, 2.5, 0.0, 0.0, 0.8 * std::sqrt(G * central / 2.5));
        if (radius_mul) radius_mul[1] = 5.0f;
    }
    if (n > 2) {
        set_body(mass, pos, vel, 2, planet, 12.0, 0.0, 0.0, std::sqrt(G * central / 12.5));
        if (radius_mul) radius_mul[2] = 5.0f;
    }
    for (uint32_t i = 3; i < n; ++i) {
        double angle = rng.uniform() * 2.0 * M_PI;
        double r = std::sqrt(rng.uniform() * (disk_max * disk_max - disk_min * disk_min) +
                             disk_min * disk_min);
        double x = r * std::cos(angle), y = r * std::sin(angle);
        double dist = std::sqrt(x * x + y * y);
        double speed = 1.01 * std::sqrt(G * central / (2.0 + dist));
        set_body(mass, pos, vel, i, body_mass, x, y, -speed * (y / dist), speed * (x / dist));
    }
}

// Benchmark: uniform unit disk, m = 1/N, circular Keplerian speed about the
// enclosed mass M(<r) = r^2 (total mass 1): v = sqrt(G r).
static void gen_uniform_disk_kepler(uint32_t n, Pcg32& rng, double G, float* mass, float* pos,
                                    float* vel) {
    const double m = n ? 1.0 / (double)n : 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double angle = rng.uniform() * 2.0 * M_PI;
        double r = std::sqrt(rng.uniform());
        double x = r * std::cos(angle), y = r * std::sin(angle);
        double v = std::sqrt(G * r * r / (r > 1e-12 ? r : 1e-12));
        double c = r > 0 ? x / r : 1.0, s = r > 0 ? y / r : 0.0;
        set_body(mass, pos, vel, i, m, x, y, -v * s, v * c);
    }
}

// Benchmark: two colliding exponential disks (scale length h = 0.2), n/2
// bodies each.  Each galaxy's first body is a central point of 10% of its
// disk mass; total system mass 1.  Centres (+1.5, 0) and (-1.5, 0) with bulk
// velocities (-0.3, +0.1) and (+0.3, -0.1).  Circular speed about the
// enclosed mass of the exponential disk plus the central point.
static void gen_colliding_disks(uint32_t n, Pcg32& rng, double G, float* mass, float* pos,
                                float* vel) {
    const double h = 0.2, rmax = 10.0 * h;
    const double md = 1.0 / 2.2, mc = 0.1 * md;  // 2 * (md + mc) = 1
    uint32_t half = n / 2;
    for (int gal = 0; gal < 2; ++gal) {
        uint32_t lo = gal == 0 ? 0 : half, hi = gal == 0 ? half : n;
        uint32_t cnt = hi - lo;
        if (cnt == 0) continue;
        double cx = gal == 0 ? 1.5 : -1.5, cy = 0.0;
        double bvx = gal == 0 ? -0.3 : 0.3, bvy = gal == 0 ? 0.1 : -0.1;
        double mdisk = cnt > 1 ? md / (double)(cnt - 1) : 0.0;
        set_body(mass, pos, vel, lo, cnt > 1 ? mc : md + mc, cx, cy, bvx, bvy);
        for (uint32_t i = lo + 1; i < hi; ++i) {
            double R;
            do {  // Gamma(2, h) radius = exponential surface density
                double u1 = rng.uniform(), u2 = rng.uniform();
                if (u1 < 1e-300) u1 = 1e-300;
                if (u2 < 1e-300) u2 = 1e-300;
                R = -h * std::log(u1 * u2);
            } while (R > rmax);
            double angle = rng.uniform() * 2.0 * M_PI;
            double x = R * std::cos(angle), y = R * std::sin(angle);
            double menc = mc + md * (1.0 - (1.0 + R / h) * std::exp(-R / h));
            double Rs = R > 1e-6 ? R : 1e-6;
            double v = std::sqrt(G * menc / Rs);
            set_body(mass, pos, vel, i, mdisk, cx + x, cy + y, bvx - v * (y / Rs),
                     bvy + v * (x / Rs));
        }
    }
}

// Benchmark: 64 isotropic Gaussians, centres U[-4,4]^2, sigma log-uniform in
// [1e-3, 0.5], component chosen uniformly per body; masses log-normal(0, 1)
// normalised to total 1; 1% of bodies copy the exact coordinates of an
// earlier body; velocities zero (cold start).
static void gen_gaussian_mixture(uint32_t n, Pcg32& rng, float* mass, float* pos, float* vel) {
    const int K = 64;
    double cxs[K], cys[K], sig[K];
    for (int k = 0; k < K; ++k) {
        cxs[k] = -4.0 + 8.0 * rng.uniform();
        cys[k] = -4.0 + 8.0 * rng.uniform();
        sig[k] = std::exp(std::log(1e-3) + (std::log(0.5) - std::log(1e-3)) * rng.uniform());
    }
    double total = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double m = std::exp(rng.normal());
        total += m;
        mass[i] = (float)m;
        if (i > 0 && rng.uniform() < 0.01) {
            uint32_t j = (uint32_t)(rng.uniform() * (double)i);
            pos[2 * i] = pos[2 * j];
            pos[2 * i + 1] = pos[2 * j + 1];
        } else {
            int k = (int)(rng.uniform() * K);
            if (k >= K) k = K - 1;
            pos[2 * i] = (float)(cxs[k] + sig[k] * rng.normal());
            pos[2 * i + 1] = (float)(cys[k] + sig[k] * rng.normal());
        }
        vel[2 * i] = 0.0f;
        vel[2 * i + 1] = 0.0f;
    }
    if (total > 0)
        for (uint32_t i = 0; i < n; ++i) mass[i] = (float)((double)mass[i] / total);
}

// Benchmark: Plummer sphere of scale radius a = 0.1 projected on the plane
// (projected enclosed mass R^2/(R^2+a^2), truncated at 99.9%), m = 1/N,
// circular speed about the projected enclosed mass.
static void gen_plummer_projection(uint32_t n, Pcg32& rng, double G, float* mass, float* pos,
                                   float* vel) {
    const double a = 0.1, m = n ? 1.0 / (double)n : 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double u = rng.uniform() * 0.999;
        double R = a * std::sqrt(u / (1.0 - u));
        double angle = rng.uniform() * 2.0 * M_PI;
        double x = R * std::cos(angle), y = R * std::sin(angle);
        double menc = R * R / (R * R + a * a);
        double Rs = R > 1e-9 ? R : 1e-9;
        double v = std::sqrt(G * menc / Rs);
        set_body(mass, pos, vel, i, m, x, y, -v * (y / Rs), v * (x / Rs));
    }
}

// Draw `draw` of stream `stream` of a PCG32 seeded with `seed` (ensemble
// sizes and per-system scenario choices).
double pcg_uniform(uint64_t seed, uint64_t stream, uint32_t draw) {
    Pcg32 rng(seed, 0x5851f42d4c957f2dULL + 2 * stream);
    double u = rng.uniform();
    for (uint32_t k = 0; k < draw; ++k) u = rng.uniform();
    return u;
}

// Returns 0 on success, -1 for an unknown name.
int generate_scenario(const char* name, uint32_t n, uint64_t seed, float grav_constant,
                      float* mass, float* pos, float* vel, float* radius_mul) {
    if (!name) return -1;
    std::string s(name);
    Pcg32 rng(seed);
    const double G = grav_constant;
    if (radius_mul)
        for (uint32_t i = 0; i < n; ++i) radius_mul[i] = 1.0f;
    if (s == "default") gen_default(n, rng, G, mass, pos, vel);
    else if (s == "two-clusters") gen_two_clusters(n, rng, G, mass, pos, vel);
    else if (s == "planetary-disk") gen_planetary_disk(n, rng, G, mass, pos, vel, radius_mul);
    else if (s == "uniform-disk-kepler") gen_uniform_disk_kepler(n, rng, G, mass, pos, vel);
    else if (s == "colliding-disks") gen_colliding_disks(n, rng, G, mass, pos, vel);
    else if (s == "gaussian-mixture") gen_gaussian_mixture(n, rng, mass, pos, vel);
    else if (s == "plummer-projection") gen_plummer_projection(n, rng, G, mass, pos, vel);
    else return -1;
    return 0;
}

}  // namespace bh
