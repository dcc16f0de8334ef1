"""Run configurations: the reference's compile-time parameters and the
seeded synthetic cylinder cases.

reference_params() mirrors src/parameters.f90 (nim_formulation = 2);
reference_mesh() mirrors create_hollow(R_i,R_o,L,0,0,L/2,NMESH_i,NMESH_j,
NMESH_k) followed by deform_nodes (main.f90:36, general.f90:428-460).

The named cases (CASES) use the benchmark geometry: a cylinder of diameter 1
and height 1 holding a coaxial hexagonal prism of side 0.2, with two-sided
tanh radial stretching of factor 1.5 and seeded 1e-6 noise on the initial
temperature.  The reference has no such mode; it is the documented
extension of the same mesh generator (tanh instead of the power law,
blend radii scaled with the annulus).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import _abi

MATH_PI = 3.14159265359          # parameters.f90:31


def physics(Ra: float, Pr: float, g_beta: float = 1.0, th_tc: float = 1.0):
    """nu, alpha as parameters.f90:169-173 computes them."""
    nu = 1.0 / math.sqrt(Ra / (g_beta * th_tc * Pr))
    alpha = nu / Pr
    return nu, alpha


def reference_params(**over) -> _abi.Params:
    """parameters.f90 defaults: DT=0.01, Ra=1e5, Pr=0.7, w=0.4,
    tolerances 1e-6 (u,v,w,T) / 5e-3 (p), v_limit=1e-2, R_i=MATH_PI/3, R_o=2,
    hot inner wall (BC id 4, T=1, general.f90:85-100)."""
    p = _abi.Params()
    Ra, Pr = over.pop("Ra", 1.0e5), over.pop("Pr", 0.7)
    p.DT = 0.01
    p.nu, p.alpha = physics(Ra, Pr)
    p.rho = 1.0
    p.g_beta = 1.0
    p.w_u = p.w_v = p.w_w = p.w_p = p.w_p2 = p.w_T = 0.4
    p.tol_u = p.tol_v = p.tol_w = p.tol_T = 1e-6
    p.tol_p = 5e-3
    p.v_limit = 1e-2
    p.dudt_epsilon = 1e-5
    p.R_i = 1.0 * (MATH_PI / 3.0)
    p.R_o = 2.0
    for f in range(5):
        for b in range(_abi.NIM_NBC):
            p.bc_value[f][b] = 0.0
    p.bc_value[4][3] = 1.0       # T on BC id 4 (inner hexagon)
    p.max_iters = 100000
    p.check_steady = 1
    p.dpdx_tolerance = 0
    p.schedule = _abi.SCHEDULE_PARALLEL
    p.formulation = 2            # parameters.f90:194
    p.precision = _abi.PRECISION_FP64
    for k, v in over.items():
        setattr(p, k, v)
    return p


def reference_mesh(**over) -> _abi.MeshParams:
    m = _abi.MeshParams()
    m.n_r = 6
    m.n_theta = 6 * m.n_r
    m.n_z = 2 * m.n_r
    m.R_i = 1.0 * (MATH_PI / 3.0)
    m.R_o = 2.0
    m.L = 2.0
    m.cluster = _abi.CLUSTER_POWER
    m.cluster_factor = 1.5
    m.hexagon = 1
    m.blend_r1, m.blend_r2, m.blend_n = 1.25, 1.75, -1.0
    for k, v in over.items():
        setattr(m, k, v)
    return m


def scaled_blend(R_i: float, R_o: float):
    """The reference blends the hexagon into the circle between the absolute
    radii 1.25 and 1.75 of its R_i=MATH_PI/3 .. R_o=2 annulus (general.f90:
    433); keep the same fractions of the annulus for other radii."""
    ri0, ro0 = 1.0 * (MATH_PI / 3.0), 2.0
    f1 = (1.25 - ri0) / (ro0 - ri0)
    f2 = (1.75 - ri0) / (ro0 - ri0)
    return R_i + f1 * (R_o - R_i), R_i + f2 * (R_o - R_i)


@dataclass
class Case:
    """A named run: mesh, physics, time step and step count."""
    name: str
    n_theta: int
    n_r: int
    n_z: int
    Ra: float
    Pr: float
    dt: float
    steps: int
    R_i: float = 0.2
    R_o: float = 0.5
    L: float = 1.0
    stretch: float = 1.5
    noise: float = 1e-6
    seed: int = 12345
    extra: dict = field(default_factory=dict)

    @property
    def ncells(self) -> int:
        return self.n_theta * self.n_r * self.n_z

    def mesh_params(self) -> _abi.MeshParams:
        r1, r2 = scaled_blend(self.R_i, self.R_o)
        return reference_mesh(n_theta=self.n_theta, n_r=self.n_r, n_z=self.n_z,
                              R_i=self.R_i, R_o=self.R_o, L=self.L,
                              cluster=_abi.CLUSTER_TANH, cluster_factor=self.stretch,
                              hexagon=1, blend_r1=r1, blend_r2=r2, blend_n=-1.0)

    def params(self, **over) -> _abi.Params:
        p = reference_params(Ra=self.Ra, Pr=self.Pr)
        p.DT = self.dt
        p.R_i, p.R_o = self.R_i, self.R_o
        for k, v in {**self.extra, **over}.items():
            setattr(p, k, v)
        return p


# The seeded synthetic cylinder cases (diameter 1, height 1, hexagon side 0.2).
CASES = {
    "c1": Case("c1", 48, 48, 32, Ra=1e4, Pr=0.71, dt=1e-3, steps=200),
    "c2": Case("c2", 128, 128, 96, Ra=1e5, Pr=0.71, dt=5e-4, steps=2000),
    "c3": Case("c3", 256, 256, 192, Ra=1e6, Pr=0.71, dt=2.5e-4, steps=1000),
    "c5": Case("c5", 64, 64, 48, Ra=1e5, Pr=0.71, dt=1e-3, steps=500),
    # profiling size: per-kernel working set above the 126 MB L2, ~1.3 GB held
    "p1": Case("p1", 96, 96, 64, Ra=1e5, Pr=0.71, dt=5e-4, steps=10),
}


def small_case(n_theta=12, n_r=6, n_z=6, Ra=1e4, Pr=0.71, dt=1e-3, steps=5, **kw) -> Case:
    return Case("small", n_theta, n_r, n_z, Ra=Ra, Pr=Pr, dt=dt, steps=steps, **kw)


def batch_cases(n: int = 64, seed: int = 2024, a_min: int = 24, a_max: int = 64) -> list[Case]:
    """The seeded batch of independent enclosures: cylinder D=1, H=1 with a
    coaxial hexagonal prism of side U[0.1, 0.3]; a x a x round(0.75 a)
    cells with a uniform in [a_min, a_max]; Ra log-uniform in [1e3, 1e6];
    Pr from {0.71, 7.0}; dt = 1e-3; seeded 1e-6 T noise per instance."""
    import random
    rng = random.Random(seed)
    out = []
    for q in range(n):
        a = rng.randint(a_min, a_max)
        side = rng.uniform(0.1, 0.3)
        Ra = 10.0 ** rng.uniform(3.0, 6.0)
        Pr = rng.choice((0.71, 7.0))
        out.append(Case(f"batch{q}", a, a, max(3, round(0.75 * a)), Ra=Ra, Pr=Pr, dt=1e-3, steps=500,
                        R_i=side, R_o=0.5, L=1.0, seed=seed + q))
    return out