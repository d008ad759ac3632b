"""Generate the golden fixtures of tests/golden with the numpy restatement (numpy_ref.py).

Each fixture holds a complete, self-contained problem (grid arrays, IB lists, dt, seeded
initial state) and the states after one substep (krk = 1) and after two RK3 steps, as
computed by the independent numpy restatement.  Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from cfd_b200.channel import build_channel  # noqa: E402
from cfd_b200.config import tiny  # noqa: E402
from numpy_ref import NumpyChannel  # noqa: E402

CASES = {
    "tiny_ib_ctp1": tiny(ngal1=24, ngal2=18, ny=17),
    "tiny_ib_ctp0": tiny(ngal1=18, ngal2=24, ny=15, flag_ctpress=0, qxt=2.0, seed=7),
    "tiny_smooth": tiny(ngal1=12, ngal2=12, ny=13, posth=0.0, cyl_diameter=0.0, seed=3),
}


def pack(setup):
    g = setup.grid
    d = dict(ngal1=setup.cfg.ngal1, ngal2=setup.cfg.ngal2, ny=setup.cfg.ny, dny=g.dny,
             re_b=setup.cfg.re_b, alp=setup.cfg.alp, bet=setup.cfg.bet, mpgx=setup.cfg.mpgx,
             qxt=setup.cfg.qxt, ctp=setup.cfg.flag_ctpress, dt=setup.dt,
             yu=g.yu, yv=g.yv, dthdyu=g.dthdyu, dthdyv=g.dthdyv, dyu2i=g.dyu2i, dyv2i=g.dyv2i,
             ibu_idx=setup.ibu.idx, ibu_w=setup.ibu.w, ibu_rng=np.array(setup.ibu.jlo + setup.ibu.jhi),
             ibv_idx=setup.ibv.idx, ibv_w=setup.ibv.w, ibv_rng=np.array(setup.ibv.jlo + setup.ibv.jhi))
    for k, v in setup.state().items():
        d["in_" + k] = v
    return d


def main():
    for name, cfg in CASES.items():
        setup = build_channel(cfg)
        d = pack(setup)
        ref = NumpyChannel(setup)
        ref.upload_state(setup.state())
        ref.rk_substep(1)
        for k, v in ref.download_state().items():
            d["sub1_" + k] = v
        ref = NumpyChannel(setup)
        ref.upload_state(setup.state())
        ref.step(2)
        for k, v in ref.download_state().items():
            d["step2_" + k] = v
        d["step2_mpgx"] = ref.mpgx
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, **d)
        print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
