"""Channel configuration and the named workloads.

``ChannelConfig`` carries the inputs the reference reads from ``input.in`` for the hot
path (start.f90:62-227, read by name instead of by line position; the shipped input.in
and the reader disagree, start.f90:157-183 vs input.in:49-65) plus the cylinder lattice
of the roughness.  ``build_channel`` turns it into the arrays every implementation of the
step consumes: the y-grid, the IB point lists and the C-ABI config struct values.

Named workloads (seeded synthetic inputs; no dataset is involved):

=========  =======================================================  ==================
name       grid Ngal1 x ny x Ngal2, flow                            cylinders (h units)
=========  =======================================================  ==================
re180      64 x 97 x 64, Re_tau 180, 100 steps (CPU-runnable case)   H .10 D .05 s .20
re395      192 x 193 x 192, Re_tau 395, FP64                         H .08 D .04 s .16
re550      384 x 257 x 384, Re_tau 550, FP32-mixed vs FP64           H .06 D .03 s .12
re1000     768 x 385 x 768, Re_tau 1000                              H .04 D .02 s .08
=========  =======================================================  ==================

The box is Lx = 2*pi, Lz = pi (alp = 1, bet = 2).  The bulk Reynolds number follows
Dean's correlation Re_tau = 0.09 (2 Re_b)^0.88 and the constant pressure gradient is
mpgx = -(Re_tau/Re_b)^2 (flag_ctpress = 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional


def reb_from_retau(re_tau: float) -> float:
    """Bulk Reynolds number (half-height, bulk velocity) from Dean's correlation."""
    return 0.5 * (re_tau / 0.09) ** (1.0 / 0.88)


@dataclass
class ChannelConfig:
    ngal1: int
    ngal2: int
    ny: int
    re_tau: float
    re_b: Optional[float] = None
    mpgx: Optional[float] = None
    alp: float = 1.0
    bet: float = 2.0
    dyq: float = 10.0            # dymax/dymin of the crest-to-crest map (input.in dyq)
    ppp: int = 5                 # polynomial exponent (input.in pp)
    posth: float = 0.0           # cylinder height (canopy depth), h units
    cyl_diameter: float = 0.0
    cyl_spacing: float = 0.0
    stagger: float = 0.0         # fraction of a tile by which odd tile rows shift in z
    cfl: float = 0.5
    dt: Optional[float] = None   # None: CFL-limited dt of the initial field
    flag_ctpress: int = 1
    qxt: float = 0.0
    precision: str = "fp64"      # "fp64" or "mixed"
    seed: int = 1000
    perturbation: float = 0.1
    kmax: int = 8
    name: str = ""
    # three y-bands (start.f90:76-111): band_vface = N(3,1), the last v face of the bottom
    # band; the middle band runs at ngal1_mid x ngal2_mid (0: the wall bands' size)
    band_vface: int = 0
    ngal1_mid: int = 0
    ngal2_mid: int = 0

    def __post_init__(self):
        if self.re_b is None:
            self.re_b = reb_from_retau(self.re_tau)
        if self.mpgx is None:
            self.mpgx = -(self.re_tau / self.re_b) ** 2

    @property
    def n1(self) -> int:
        return 2 * (self.ngal1 // 3)

    @property
    def n2(self) -> int:
        return 2 * (self.ngal2 // 3)

    @property
    def nkx(self) -> int:
        return self.n1 // 2 + 1

    @property
    def ncol(self) -> int:
        return self.nkx * self.n2

    @property
    def lx(self) -> float:
        return 2.0 * math.pi / self.alp

    @property
    def lz(self) -> float:
        return 2.0 * math.pi / self.bet

    def with_(self, **kw) -> "ChannelConfig":
        return replace(self, **kw)


PRESETS = {
    "re180": ChannelConfig(ngal1=64, ngal2=64, ny=97, re_tau=180.0, posth=0.10,
                           cyl_diameter=0.05, cyl_spacing=0.20, name="re180"),
    "re395": ChannelConfig(ngal1=192, ngal2=192, ny=193, re_tau=395.0, posth=0.08,
                           cyl_diameter=0.04, cyl_spacing=0.16, name="re395"),
    "re550": ChannelConfig(ngal1=384, ngal2=384, ny=257, re_tau=550.0, posth=0.06,
                           cyl_diameter=0.03, cyl_spacing=0.12, name="re550",
                           precision="mixed"),
    "re1000": ChannelConfig(ngal1=768, ngal2=768, ny=385, re_tau=1000.0, posth=0.04,
                            cyl_diameter=0.02, cyl_spacing=0.08, name="re1000",
                            precision="mixed"),
}


def preset(name: str, **overrides) -> ChannelConfig:
    return replace(PRESETS[name], **overrides)


# Batched ensemble: 16 independent channels of uneven size (4 x 96x97x96 at Re_tau 180,
# 8 x 128x129x128 at Re_tau 260, 4 x 192x161x192 at Re_tau 395), cylinder height 0.08 h,
# diameter drawn uniformly from [0.03 h, 0.06 h] per member, spacing 4 diameters, own seeds.
ENSEMBLE_GROUPS = ((4, 96, 97, 180.0), (8, 128, 129, 260.0), (4, 192, 161, 395.0))


def ensemble_configs(seed: int = 2000, precision: str = "mixed", groups=ENSEMBLE_GROUPS):
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for count, ng, ny, rt in groups:
        for _ in range(count):
            dia = float(rng.uniform(0.03, 0.06))
            k = len(out)
            out.append(ChannelConfig(ngal1=ng, ngal2=ng, ny=ny, re_tau=rt, posth=0.08, cyl_diameter=dia,
                                     cyl_spacing=4.0 * dia, precision=precision, seed=seed + k,
                                     name=f"ens{k}-{ng}x{ny}x{ng}"))
    return out


def tiny(ngal1: int = 24, ngal2: int = 18, ny: int = 17, **kw) -> ChannelConfig:
    """A small channel for parity tests (seconds on the oracle)."""
    base = dict(ngal1=ngal1, ngal2=ngal2, ny=ny, re_tau=180.0, posth=0.12,
                cyl_diameter=0.5, cyl_spacing=2.0, dyq=3.0, name=f"tiny{ngal1}x{ny}x{ngal2}")
    base.update(kw)
    return ChannelConfig(**base)
