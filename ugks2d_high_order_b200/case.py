"""Couette case description: the subset of the reference's `&config_para` / `&boundary_para`
namelists (Config.ini, parsed by mod_ImportPara.f90:141-173) that the kinetic hot path reads.

Derived constants follow set_const_para (mod_ImportPara.f90:911-930):
gamma = (ck+4)/(ck+2); with CouetteMuRef > 0, mu_ref = CouetteMuRef and Kn = sqrt(pi)*mu_ref.
"""
from dataclasses import dataclass, field, replace
import math
import os

import numpy as np

_GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")


@dataclass
class CouetteCase:
    nx: int = 8                      # Nx_all
    ny: int = 64                     # Ny_all
    dx: float = 0.125                # uniform mesh of Mesh2d.dat: x in [0,1], y in [0,1]
    dy: float = 1.0 / 64.0
    ck: int = 1
    pr: float = 0.66666666666666666667
    omega: float = 0.5
    mu_ref: float = 0.05637282460904075   # CouetteMuRef
    cfl: float = 0.1
    tinf: float = 2.0                # initial T_native (theta = T/2 = 1)
    wall_ux: tuple = (-3.872983346207417, 3.872983346207417)   # WallUx(3:4): bottom, top
    wall_tnative: tuple = (2.0, 2.0)                           # Tw per wall
    method: str = "Explicit"        # Explicit | ImplicitSteady | HighOrderImplicit | S2CN2
    ncfl: float = 1000.0             # Implicit_nCFL
    nslab: int = 8                   # NP_Y of the reference's 1 x NP_Y MPI blocking (block-Jacobi seams)
    mass_rescale: bool = False       # ClosedCouetteMassRescale
    macro_sweeps: int = 2            # Implicit_MacroSweeps
    residual_tol: float = 1.0e-8     # Implicit_ResidualTol
    moment_tol: float = 1.0e-12      # Implicit_MomentTol
    min_alpha: float = 1.0e-6        # Implicit_MinAlpha
    max_iter: int = 3000             # MAX_ITER (the loop cap; 200000 in the explicit case)
    # the research S2CN2 wall variants (mod_ImportPara.f90:88-93), off in every delivered case
    flux_wall: int = 1               # FluxWall_type: 1 multiscale wall (s2w2), 0 free-streaming wall (s2w1)
    s2w1_time_centered: int = 0      # S2W1_time_centered: W1T midpoint wall (needs FluxWall_type 0)
    s2w1d_face_time: int = 0         # S2W1D_face_time_consistent: W1D face correction (needs W1T)
    s2w2r_shared_predictor: int = 0  # S2W2R_shared_predictor: W2R (FluxWall_type 1, ck 1, Pr 1)

    @property
    def gamma(self):
        return float(self.ck + 4) / float(self.ck + 2)

    @property
    def kn(self):
        return math.sqrt(math.pi) * self.mu_ref

    def with_(self, **kw):
        return replace(self, **kw)


def reference_case(method="Explicit"):
    """The reference's delivered Ma3 Couette case (cases/low_explicit|low_implicit|high_implicit, and
    consistency/high_explicit for the explicit high-order S2CN2 method: no mass rescale)."""
    c = CouetteCase(method=method)
    if method in ("ImplicitSteady", "HighOrderImplicit"):
        c.mass_rescale = True
    if method == "Explicit":
        c.max_iter = 200000
    return c


def refined_high_order_case():
    """The refined HighOrderImplicit variant: 16 x 128 cells on the unit square (uniform mesh) with a
    48 x 48 velocity set (generated half-range table, scale 2); otherwise the high_implicit case.
    The reference has no 48^2 table and no run at this size, so only the oracle checks it."""
    c = reference_case("HighOrderImplicit")
    return c.with_(nx=16, ny=128, dx=1.0 / 16.0, dy=1.0 / 128.0)


def baseline_explicit_case():
    """Throughput variant of the explicit case: CFL 0.5, omega 0.81 (same mesh, walls, Kn)."""
    return CouetteCase(cfl=0.5, omega=0.81)


def load_velocity_half32():
    """The reference's velocity_half32_scale2.dat table (u, v, w), k = i + (j-1)*Nu."""
    t = np.load(os.path.join(_GOLDEN, "velocity_half32_scale2.npy"))
    return t[:, 0].copy(), t[:, 1].copy(), t[:, 2].copy()


def velocity_table(n_per_axis, scale=2.0):
    """(u, v, w) of an n x n half-range table with the given scale: the reference's own file for
    32 x 32 at scale 2, otherwise generated (ugks2d_high_order_b200.velocity)."""
    if n_per_axis == 32 and scale == 2.0:
        return load_velocity_half32()
    from .velocity import structured_table
    return structured_table(n_per_axis, scale)


def batched_cases(n=256, seed=20261203, ny_choices=(32, 64, 128), nvel_choices=(24, 32, 48)):
    """The batched Couette distribution: Kn log-uniform in [0.01, 1] (mu_ref = Kn / sqrt(pi),
    mod_ImportPara.f90:926), wall Mach uniform in [0.5, 3] (WallUx = -/+ Ma sqrt(5/3 theta_w) per
    wall), wall temperature ratio uniform in [0.8, 1.2] (T_native,wall = 2 ratio, gas T_native 2),
    grids 8 x {32, 64, 128} on the unit square, velocity sets {24^2, 32^2, 48^2}, all uniform, from
    numpy's PCG64(seed).  Method S2CN2 at CFL 0.1.  Returns [(CouetteCase, n_per_axis)]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        kn = 10.0 ** rng.uniform(-2.0, 0.0)
        ma = rng.uniform(0.5, 3.0)
        ratio = rng.uniform(0.8, 1.2)
        ny = int(rng.choice(ny_choices))
        nva = int(rng.choice(nvel_choices))
        tw = 2.0 * ratio
        ux = ma * math.sqrt(5.0 / 3.0 * (0.5 * tw))
        c = CouetteCase(ny=ny, dy=1.0 / ny, mu_ref=kn / math.sqrt(math.pi), wall_ux=(-ux, ux),
                        wall_tnative=(tw, tw), method="S2CN2")
        out.append((c, nva))
    return out
