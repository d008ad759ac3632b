"""Load a golden fixture (make_golden.py) back into a ChannelSetup."""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("tiny_ib_ctp1", "tiny_ib_ctp0", "tiny_smooth")


def load(name):
    from cfd_b200.channel import ChannelSetup
    from cfd_b200.config import ChannelConfig
    from cfd_b200.geometry import IBList
    from cfd_b200.grid import YGrid
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    cfg = ChannelConfig(ngal1=int(z["ngal1"]), ngal2=int(z["ngal2"]), ny=int(z["ny"]), re_tau=180.0,
                        re_b=float(z["re_b"]), mpgx=float(z["mpgx"]), alp=float(z["alp"]),
                        bet=float(z["bet"]), flag_ctpress=int(z["ctp"]), qxt=float(z["qxt"]),
                        dt=float(z["dt"]), name=name)
    g = YGrid(ny=int(z["ny"]), dny=int(z["dny"]), yu=z["yu"], yv=z["yv"], dthdyu=z["dthdyu"],
              dthdyv=z["dthdyv"], dyu2i=z["dyu2i"], dyv2i=z["dyv2i"])
    ru, rv = z["ibu_rng"], z["ibv_rng"]
    ibu = IBList(z["ibu_idx"].astype(np.int32), z["ibu_w"], (int(ru[0]), int(ru[1])), (int(ru[2]), int(ru[3])))
    ibv = IBList(z["ibv_idx"].astype(np.int32), z["ibv_w"], (int(rv[0]), int(rv[1])), (int(rv[2]), int(rv[3])))
    setup = ChannelSetup(cfg=cfg, grid=g, ibu=ibu, ibv=ibv, dt=float(z["dt"]), u1=z["in_u1"],
                         u2=z["in_u2"], u3=z["in_u3"], p=z["in_p"])
    return setup, z
