"""Config (src/config.ts:1-22) and the engine's extension parameters."""
from __future__ import annotations

import dataclasses

from . import _lib


@dataclasses.dataclass(frozen=True)
class Config:
    """Readonly physics parameters.

    The first five fields are the reference's ``Config`` type
    (config.ts:1-7) with the same defaults (config.ts:9-22).  The rest select
    engine extensions; their defaults keep the reference's behaviour.
    """

    gravConstant: float = 1.0
    bhTheta: float = 0.6
    substeps: int = 1
    deltaTime: float = 0.1 * 1.0 / (60.0 * 1)
    epsilonMultiplier: float = 1.0
    # extensions
    softening: str = "reference"        # "reference" | "plummer"
    plummerEps: float = 1e-3
    mortonBits: int = 32                # 32 | 64
    mortonDomain: str = "fixed2000"     # "fixed2000" | "bbox"
    integrator: str = "symplectic-euler"  # "symplectic-euler" | "leapfrog-kdk"
    leafSize: int = 1
    walkBlock: int = 0
    useGraphs: bool = True
    fp64Levels: bool = True
    walk: str = "exact"                 # "exact" (reference per-body walk) | "group"
    multipole: int = 2                  # group walk: 1 monopole, 2 + quadrupole
    bodiesPerLane: int = 2              # group walk: group = 32 x bodiesPerLane bodies
    farAlpha: float = 0.0               # group walk, Plummer: far nodes (r_g < farAlpha R)
                                        # act through one local expansion per group (0 = off)

    def to_c(self, device: int = 0) -> _lib.bh_config:
        c = _lib.bh_config()
        c.grav_constant = self.gravConstant
        c.bh_theta = self.bhTheta
        c.substeps = self.substeps
        c.delta_time = self.deltaTime
        c.epsilon_multiplier = self.epsilonMultiplier
        c.softening = {"reference": _lib.BH_SOFTENING_REFERENCE,
                       "plummer": _lib.BH_SOFTENING_PLUMMER}[self.softening]
        c.plummer_eps = self.plummerEps
        c.morton_bits = self.mortonBits
        c.morton_domain = {"fixed2000": _lib.BH_DOMAIN_FIXED2000,
                           "bbox": _lib.BH_DOMAIN_BBOX}[self.mortonDomain]
        c.integrator = {"symplectic-euler": _lib.BH_INTEGRATOR_SYMPLECTIC_EULER,
                        "leapfrog-kdk": _lib.BH_INTEGRATOR_LEAPFROG_KDK}[self.integrator]
        c.leaf_size = self.leafSize
        c.walk_block = self.walkBlock
        c.device = device
        c.use_graphs = 1 if self.useGraphs else 0
        c.fp64_levels = 1 if self.fp64Levels else 0
        c.walk_mode = {"exact": _lib.BH_WALK_EXACT, "group": _lib.BH_WALK_GROUP}[self.walk]
        c.multipole_order = self.multipole
        c.bodies_per_lane = self.bodiesPerLane
        c.far_alpha = self.farAlpha
        return c


def getDefaultConfig() -> Config:
    """config.ts:9-22: G=1, theta=0.6, substeps=1, dt=0.1/(60*substeps), epsMult=1."""
    substeps = 1
    return Config(gravConstant=1.0, bhTheta=0.6, substeps=substeps,
                  deltaTime=0.1 * 1.0 / (60.0 * substeps), epsilonMultiplier=1.0)


# The seeded benchmark workloads (Plummer softening, group walk with
# quadrupoles, leaf buckets of 8), by name.  The benchmark points also act
# on far nodes through one local expansion per group (farAlpha = 0.4: on
# B200 the 800k walk 0.56 -> 0.43 ms and the 16.8M walk 12.1 -> 8.3 ms with
# 128-body groups, the median FP64 force error 4.9e-4 and 6.2e-4); the
# parity workload keeps the plain group walk.
FAR_ALPHA = 0.4
WORKLOADS = {
    # N=16,384 uniform disk, theta 0.7, eps 1e-3, dt 1e-4, 32-bit keys over the bbox
    "uniform-disk-16k": dict(n=16384, scenario="uniform-disk-kepler", steps=100,
                             config=Config(bhTheta=0.7, deltaTime=1e-4, softening="plummer",
                                           plummerEps=1e-3, mortonDomain="bbox",
                                           integrator="leapfrog-kdk", walk="group",
                                           leafSize=8)),
    # N=800,000 two colliding exponential disks, theta 0.5, eps 1e-3, dt 5e-5.
    # No integrator is named for this point: the reference's own (symplectic
    # Euler, barnes_hut.wgsl:110,119-120), as its reference arm runs it.
    "colliding-disks-800k": dict(n=800_000, scenario="colliding-disks", steps=1000,
                                 config=Config(bhTheta=0.5, deltaTime=5e-5, softening="plummer",
                                               plummerEps=1e-3, mortonDomain="bbox",
                                               integrator="symplectic-euler", walk="group",
                                               leafSize=8, farAlpha=FAR_ALPHA)),
    # N=16,777,216 Gaussian mixture, 64-bit keys, theta 0.5, eps 1e-4, dt 1e-5
    # (no integrator named: the reference's)
    "gaussian-mixture-16m": dict(n=16_777_216, scenario="gaussian-mixture", steps=50,
                                 config=Config(bhTheta=0.5, deltaTime=1e-5, softening="plummer",
                                               plummerEps=1e-4, mortonBits=64,
                                               integrator="symplectic-euler", walk="group",
                                               leafSize=8, farAlpha=FAR_ALPHA)),
    # N=4,194,304 from the same Gaussian-mixture generator and settings: the
    # profiling case of the 16M point (inputs > L2, a few GB on the device)
    "gaussian-mixture-4m": dict(n=4_194_304, scenario="gaussian-mixture", steps=50,
                                config=Config(bhTheta=0.5, deltaTime=1e-5, softening="plummer",
                                              plummerEps=1e-4, mortonBits=64,
                                              integrator="symplectic-euler", walk="group",
                                              leafSize=8, farAlpha=FAR_ALPHA)),
}
