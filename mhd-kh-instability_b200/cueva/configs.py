"""The Kelvin-Helmholtz workloads, in the reference orientation.

The benchmark problem is posed with the shear flow along x (periodic) and
the shear normal along y (outflow).  The reference's KH set-up
(03_init_var_primitive.f95:2297-2336, boundary BOUND 6 of 04_boundary.f95:
2867-3033) has the flow along y (periodic) and the normal along x (copy
boundaries), and its reconstruction scratch needs jmax <= imax
(scalar.f95:371-372).  The workloads are therefore run after the proper
rotation (x, y, z) -> (y, x, -z), which maps vectors and pseudovectors
alike: reference x = problem y in [-1, 1] with imax = Ny cells, reference
y = problem x in [-0.5, 0.5] with jmax = Nx cells.  The uniform field
B = (0.1, 0, 0) becomes (0, 0.1, 0); E = -v x B is evaluated in the
rotated frame.
"""
import math
from dataclasses import dataclass, field


@dataclass
class KHConfig:
    name: str
    nx: int               # cells along the flow (periodic), = reference jmax
    ny: int               # cells across the shear layer (outflow), = reference imax
    order: int            # IMEX tableau id
    flux_solver: int      # 5 HLL, 7 HLLC
    rec_mp: int = 0       # 0 MP5, 1 MP7, 2 MP9
    c2p: int = 1          # 1 Cardano
    sigma: float = 1e3
    v0: float = 0.5
    a: float = 0.01
    steps: int = 200
    cfl: float = 0.25
    precision: int = 0
    intsum_reset: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def imax(self):
        return self.ny

    @property
    def jmax(self):
        return self.nx

    def solver_kwargs(self):
        return dict(imax=self.imax, jmax=self.jmax, order=self.order, flux_solver=self.flux_solver,
                    rec_mp=self.rec_mp, c2p=self.c2p, bc_x=0, bc_y=1, precision=self.precision, lx=2.0, ly=1.0,
                    lz=1.0, cfl=self.cfl, sigma=self.sigma, gamma=4.0 / 3.0, intsum_reset=self.intsum_reset)

    def kh_kwargs(self):
        return dict(v0=self.v0, a=self.a, amp=0.01, width=0.01, kpert=2 * math.pi, phase=0.0, bshear=0.1,
                    rho0=1.0, p0=1.0)


# small plain-FP64 workload: 128 x 256, sigma 1e3, MP5 + HLL, SSP2(2,2,2), 200 steps, Cardano
C1 = KHConfig("kh-128x256-mp5-hll-ssp222-sigma1e3", 128, 256, order=2, flux_solver=5, sigma=1e3, steps=200)
# benchmark workload: plain FP64 at 1024 x 2048, MP5 + HLLC, sigma 1e6, SSP3(4,3,3), 500 steps.
# The reference's SSP3(4,3,3) keeps accumulating the stage sums across stages
# (cleanvarint runs once per step) and breaks down within a few steps; the
# workload runs the tableau with the sums reset before every stage.
C2 = KHConfig("kh-1024x2048-mp5-hllc-ssp433-sigma1e6", 1024, 2048, order=4, flux_solver=7, sigma=1e6, steps=500,
              intsum_reset=1)
# large study workload: 2048 x 4096, V0 = 0.8, sigma 1e5 (MP7 / MP9 variants; mixed precision)
C3 = KHConfig("kh-2048x4096-mp5-hllc-ssp433-v08-sigma1e5", 2048, 4096, order=4, flux_solver=7, sigma=1e5,
              v0=0.8, steps=1000, intsum_reset=1)
# target workload: 2048 x 4096 MP5 + HLLC resistive KH, sigma 1e6
TARGET = KHConfig("kh-2048x4096-mp5-hllc-ssp433-sigma1e6", 2048, 4096, order=4, flux_solver=7, sigma=1e6,
                  steps=500, intsum_reset=1)

CONFIGS = {c.name: c for c in (C1, C2, C3, TARGET)}
