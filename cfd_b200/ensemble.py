"""Batched ensemble of independent channels on one GPU (cfd_ensemble_* of the C ABI).

Every member is an ordinary :class:`cfd_b200.channel.Channel` (its own grid, IB lattice,
seed and precision); :class:`Ensemble` advances all of them with one CUDA-graph launch per
RK3 step, the members' steps running as parallel branches of that graph.
"""
from __future__ import annotations

import ctypes as C

from . import capi
from .channel import Channel, build_channel


class Ensemble:
    def __init__(self, members):
        self.members = list(members)
        self.lib = self.members[0].lib
        arr = (C.c_void_p * len(self.members))(*[m.ctx for m in self.members])
        h = C.c_void_p()
        st = self.lib.cfd_ensemble_create(arr, len(self.members), C.byref(h))
        self.h = h
        if st != capi.CFD_OK:
            msg = self.lib.cfd_ensemble_last_error(h) if h else b""
            self.close()
            raise capi.CfdError(f"ensemble_create: {capi.ERRORS.get(st, st)}: {msg.decode() if msg else ''}")

    @classmethod
    def from_configs(cls, cfgs, device: int = 0, tuning=None):
        """Members from ChannelConfigs (tuning as for Channel, e.g. "auto")."""
        chans = []
        for cfg in cfgs:
            ch = Channel(build_channel(cfg), device=device, precision=cfg.precision, tuning=tuning)
            ch.upload_state()
            chans.append(ch)
        return cls(chans)

    def _chk(self, st, what):
        if st != capi.CFD_OK:
            msg = self.lib.cfd_ensemble_last_error(self.h)
            raise capi.CfdError(f"{what}: {capi.ERRORS.get(st, st)}: {msg.decode() if msg else ''}")

    def step(self, nsteps: int = 1):
        self._chk(self.lib.cfd_ensemble_step(self.h, int(nsteps)), "ensemble_step")

    def stream(self) -> int:
        """cudaStream_t (as an integer) the ensemble's graph runs on."""
        s = C.c_void_p()
        self._chk(self.lib.cfd_ensemble_stream(self.h, C.byref(s)), "ensemble_stream")
        return s.value or 0

    def synchronize(self):
        self._chk(self.lib.cfd_ensemble_synchronize(self.h), "ensemble_synchronize")

    def close(self, members: bool = False):
        if getattr(self, "h", None):
            self.lib.cfd_ensemble_destroy(self.h)
            self.h = None
        if members:
            for m in self.members:
                m.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
