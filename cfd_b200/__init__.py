"""cfd_b200 - B200-native (sm_100a) hot path of the LittleHarsh channel DNS.

The per-timestep path of the reference (Fourier x/z, staggered finite differences in y,
Kim & Moin fractional step with RK3/Crank-Nicolson, immersed-boundary cylinders) runs as
hand-written CUDA kernels behind the C ABI in include/cfd_b200.h; this package holds the
kernels (csrc/), the host driver mirroring the reference's entry points (channel.py) and
the host set-up of grids, IB lists and seeded initial fields.
"""
from .config import ChannelConfig, PRESETS, preset, tiny  # noqa: F401
from .channel import Channel, ChannelSetup, build_channel  # noqa: F401
from .ensemble import Ensemble  # noqa: F401

__version__ = "0.1.0"
