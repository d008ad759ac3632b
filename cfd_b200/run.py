"""Run a channel for a number of RK3 steps on one GPU (the restored main loop of
littleharsh.f90:159-200) and print timing and diagnostics.

    python -m cfd_b200.run --config re550 --steps 10 --precision mixed
    python -m cfd_b200.run --config re550 --ny 33 --steps 1 --stages   # small profiling case

--ny/--ngal override the named workload's grid (same x/z transform lengths, fewer planes)
so that a profiler can capture single launches of the production kernels cheaply.
"""
from __future__ import annotations

import argparse
import json
import time

from .channel import Channel, build_channel
from .config import preset


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cfd_b200.run")
    ap.add_argument("--config", default="re550")
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--ngal", type=int, nargs=2, default=None, metavar=("NGAL1", "NGAL2"))
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"])
    ap.add_argument("--stages", action="store_true", help="launch through the stage entry points (no graph)")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    kw = {}
    if a.ny:
        kw["ny"] = a.ny
    if a.ngal:
        kw["ngal1"], kw["ngal2"] = a.ngal
    if a.precision:
        kw["precision"] = a.precision
    cfg = preset(a.config, **kw)
    t0 = time.perf_counter()
    setup = build_channel(cfg)
    t_setup = time.perf_counter() - t0
    ch = Channel(setup, device=a.device)
    ch.upload_state()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        if a.stages:
            for k in (1, 2, 3):
                ch.rhs0(k)
                ch.nonlinear(k)
                ch.solve_uvw(k)
                ch.meanflow(k)
                ch.solve_p(k)
                ch.vcorr(k)
            if cfg.flag_ctpress == 1:
                ch.meanflow(1)
        else:
            ch.step(1)
    ch.synchronize()
    el = time.perf_counter() - t0
    out = {"config": cfg.name, "grid": [cfg.ngal1, setup.grid.nyv, cfg.ngal2], "precision": cfg.precision,
           "steps": a.steps, "seconds": el, "setup_seconds": t_setup, "divergence": ch.divergence_max(),
           **ch.scalars()}
    print(json.dumps(out))
    ch.close()


if __name__ == "__main__":
    main()
