"""Autotuner of the launch shapes (cfd_tuning): for one grid, precision and GPU it builds a
context per candidate, times RK3 steps with CUDA events, and keeps the fastest.

Candidates: the x-line path (marching in y; register two-step; the same held to 64
registers; with 1.5 complex lines per row; on packed FP32 line pairs; or shared-memory
Stockham) searched jointly with the radix order of its two-step transform (N = N1*N2 or
N2*N1: which register DFT runs first), rows per CTA of the two-step x-line kernel, lines per CTA of the two-step
z kernels, the radix order of the z transforms, the y-planes per thread of the
right-hand-side kernel, and the threads per CTA of the column sweeps.
The search is coordinate-wise from the library default, one knob at a time, so it costs a
dozen short timings.  Results are cached in a JSON file keyed by grid, precision and GPU
name (CFD_TUNE_CACHE, default ~/.cache/cfd_b200/tuning.json).
"""
from __future__ import annotations

import json
import os

# A knob is one setting or a tuple of settings searched jointly: the x-line kernel and its
# radix order interact (the register-capped kernel, path 5, only pays at one split), so a
# one-at-a-time search from path 1 would not reach their best pair.
KNOBS = ((("xline_path", "xsplit"), ((6, 1), (1, 1), (1, 2), (5, 1), (5, 2), (2, 1), (3, 1), (4, 1))),
         ("xline_rows", (2, 4, 8)), ("zlines", (4, 8, 16)), ("zsplit", (1, 2)), ("rhs_chunk", (2, 4, 8, 16)),
         ("solve_cols", (64, 128, 256)))


# x-line paths that only FP32-mixed contexts run (FP64 contexts asked for them run path 1)
MIXED_ONLY_XLINE = (4, 5, 6)

# knobs that only act with another setting (the library reports them as 0 or 1 otherwise)
RELEVANT = {"xline_rows": lambda t: t.get("xline_path") != 2,
            "zsplit": lambda t: t.get("xline_path") in (1, 5, 6)}


def _cache_path() -> str:
    return os.environ.get("CFD_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cfd_b200",
                                                          "tuning.json"))


def _key(setup, precision: str, gpu: str) -> str:
    c, g = setup.cfg, setup.grid
    return f"v9|{gpu}|{c.ngal1}x{g.nyu}x{c.ngal2}|{precision}|ib{setup.ibu.n > 0}"


def time_step(setup, precision, device, tuning, steps=5, warmup=2):
    """Seconds per RK3 step of one context with the given launch shapes (CUDA events)."""
    import torch
    from .channel import Channel
    ch = Channel(setup, device=device, precision=precision, tuning=tuning)
    try:
        ch.upload_state()
        ch.step(warmup)
        stream = torch.cuda.Stream(device)
        ch.set_stream(stream.cuda_stream)
        ch.step(1)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        ch.step(steps)
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e) / 1e3 / steps, ch.tuning()
    finally:
        ch.close()


def autotune(setup, precision: str, device: int = 0, steps: int = 5, log=None):
    """Coordinate search over KNOBS from the default shapes; returns (best tuning, seconds)."""
    best_t, best = time_step(setup, precision, device, None, steps)
    tried = {json.dumps(best, sort_keys=True)}
    for name, values in KNOBS:
        for v in values:
            if name in RELEVANT and not RELEVANT[name](best):
                continue
            cand = dict(best, **(dict(zip(name, v)) if isinstance(name, tuple) else {name: v}))
            if precision == "fp64" and cand.get("xline_path") in MIXED_ONLY_XLINE:
                continue
            k = json.dumps(cand, sort_keys=True)
            if k in tried:
                continue
            tried.add(k)
            try:
                t, eff = time_step(setup, precision, device, cand, steps)
            except RuntimeError as err:  # a shape the grid cannot take
                if log:
                    log(f"skip {cand}: {err}")
                continue
            tried.add(json.dumps(eff, sort_keys=True))
            if log:
                log(f"{eff} {t * 1e3:.3f} ms/step")
            if t < best_t:
                best_t, best = t, eff
    return best, best_t


def tuned(setup, precision: str, device: int = 0):
    """The cached tuning of this grid, precision and GPU, measured (and cached) if absent."""
    import torch
    gpu = torch.cuda.get_device_name(device)
    key = _key(setup, precision, gpu)
    path = _cache_path()
    cache = {}
    if os.path.exists(path):
        with open(path) as f:
            cache = json.load(f)
    if key not in cache:
        best, t = autotune(setup, precision, device)
        cache[key] = {"tuning": best, "ms_per_step": t * 1e3}
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)  # atomic: concurrent processes never see a partial file
    return cache[key]["tuning"]


def main(argv=None):
    import argparse
    from .channel import build_channel
    from .config import preset
    ap = argparse.ArgumentParser(prog="python -m cfd_b200.autotune")
    ap.add_argument("--config", default="re550")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"])
    ap.add_argument("--steps", type=int, default=5)
    a = ap.parse_args(argv)
    cfg = preset(a.config)
    prec = a.precision or cfg.precision
    setup = build_channel(cfg)
    best, t = autotune(setup, prec, 0, a.steps, log=print)
    print(json.dumps({"config": a.config, "precision": prec, "tuning": best, "ms_per_step": t * 1e3}))


if __name__ == "__main__":
    main()
