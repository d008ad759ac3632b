"""Batched ensemble (cfd_ensemble_*): members of different sizes, precisions and IB
lattices advanced by one graph launch per RK3 step give the same fields as the same
channels stepped on their own (the kernels are deterministic, so equal to round-off 0)."""
import numpy as np
import pytest

from cfd_b200 import Channel, Ensemble, build_channel
from cfd_b200.config import tiny

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


CFGS = [tiny(24, 18, 17, precision="fp64"),
        tiny(64, 96, 17, cyl_diameter=0.3, cyl_spacing=1.5, precision="mixed", seed=11),
        tiny(96, 64, 21, cyl_diameter=0.3, cyl_spacing=1.0, precision="fp64", seed=12)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def pair(cfg):
    s = build_channel(cfg)
    out = []
    for _ in range(2):
        ch = Channel(s, device=0, precision=cfg.precision)
        ch.upload_state()
        out.append(ch)
    return s, out


def test_ensemble_matches_members(torch_cuda):
    setups, ens_m, solo = [], [], []
    for cfg in CFGS:
        s, (a, b) = pair(cfg)
        setups.append(s)
        ens_m.append(a)
        solo.append(b)
    ens = Ensemble(ens_m)
    ens.step(2)
    ens.step(1)
    for ch in solo:
        ch.step(3)
    for a, b in zip(ens_m, solo):
        sa, sb = a.download_state(), b.download_state()
        for k in sa:
            assert rel(sa[k], sb[k]) < 1e-14, k
    # a dt change of one member is picked up at the next ensemble step
    ens_m[1].set_dt(0.6 * setups[1].dt)
    solo[1].set_dt(0.6 * setups[1].dt)
    ens.step(2)
    for ch in solo:
        ch.step(2)
    for a, b in zip(ens_m, solo):
        sa, sb = a.download_state(), b.download_state()
        for k in sa:
            assert rel(sa[k], sb[k]) < 1e-14, k
    ens.close(members=True)
    for ch in solo:
        ch.close()


def test_ensemble_errors(torch_cuda):
    s = build_channel(CFGS[0])
    ch = Channel(s, device=0)
    with pytest.raises(RuntimeError, match="no state"):
        e = Ensemble([ch])
        e.step(1)
    with pytest.raises(RuntimeError, match="repeated"):
        Ensemble([ch, ch])
    ch.close()


def test_ensemble_members_vs_oracle(torch_cuda):
    """One member of each size of the uneven 16-channel ensemble (96x97x96 at Re_tau 180,
    128x129x128 at 260, 192x161x192 at 395, each with its own cylinder lattice and seed),
    advanced together by the ensemble for 10 RK3 steps, against the FP64 oracle stepping the
    same channels alone: FP64 members within 1e-10, FP32-mixed members within 1e-5 relative
    L2 on u, v, w and p."""
    from cfd_b200.config import ensemble_configs
    from oracle.oracle import OracleChannel
    cfgs = ensemble_configs(precision="fp64")
    picks = [cfgs[0], cfgs[4], cfgs[12]]   # first member of each size group
    setups = [build_channel(c) for c in picks]
    refs = []
    for s in setups:
        o = OracleChannel(s)
        o.upload_state()
        o.step(10)
        refs.append(o.download_state())
        o.close()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        members = []
        for s in setups:
            ch = Channel(s, device=0, precision=prec)
            ch.upload_state()
            members.append(ch)
        ens = Ensemble(members)
        ens.step(10)
        for s, ch, ref in zip(setups, members, refs):
            st = ch.download_state()
            for k in ("u1", "u2", "u3", "p"):
                e = rel(st[k], ref[k])
                assert e < tol, (prec, s.cfg.name, k, e)
        ens.close(members=True)
