"""GPU parity: every C-ABI entry point against the FP64 oracle on the same seeded inputs.

Tolerances: FP64 path <= 1e-10 relative L2 per field (stages and 10 RK3 steps); the
FP32-mixed path <= 1e-5 relative L2 per field (u, v, w and p) after 10 steps.
"""
import ctypes as C

import numpy as np
import pytest

from fixtures import NAMES, load

pytestmark = pytest.mark.gpu

STAGES = ("rhs0", "nonlinear", "solve_uvw", "meanflow", "solve_p", "vcorr")
FIELDS = ("u1", "u2", "u3", "p", "du1", "du2", "du3", "nu1", "nu2", "nu3", "psi")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def make(setup, precision="fp64"):
    from cfd_b200.channel import Channel
    ch = Channel(setup, device=0, precision=precision)
    ch.upload_state()
    return ch


def oracle(setup):
    from oracle.oracle import OracleChannel
    o = OracleChannel(setup)
    o.upload_state()
    return o


@pytest.mark.parametrize("name", NAMES)
def test_stage_by_stage_fp64(torch_cuda, name):
    s, _ = load(name)
    g, o = make(s), oracle(s)
    for krk in (1, 2, 3):
        for stage in STAGES:
            getattr(g, stage)(krk)
            getattr(o, stage)(krk)
            for k in FIELDS:
                e = rel(g.download(k), o.download(k))
                assert e < 1e-11, (krk, stage, k, e)
    g.close()


@pytest.mark.parametrize("name", NAMES)
def test_golden_fixture_fp64(torch_cuda, name):
    s, z = load(name)
    g = make(s)
    g.rk_substep(1)
    st = g.download_state()
    for k in st:
        assert rel(st[k], z["sub1_" + k]) < 1e-11, k
    g.close()
    g = make(s)        # fresh context: the constant-flow-rate path has advanced mpgx
    g.step(2)
    st = g.download_state()
    for k in st:
        assert rel(st[k], z["step2_" + k]) < 1e-11, k
    assert g.scalars()["mpgx"] == pytest.approx(float(z["step2_mpgx"]), rel=1e-12)
    g.close()


@pytest.mark.parametrize("cfgname", ["tiny", "tiny_ctp0", "small_ib", "re180", "re395", "re550"])
def test_ten_steps_fp64_and_mixed(torch_cuda, cfgname):
    """10 RK3 steps against the oracle: FP64 within 1e-10 relative L2 on every field, mixed
    within 1e-5 on u, v, w.  re180, re395 and re550 are the named workloads (64x97x64,
    192x193x192, 384x257x384 with their cylinder lattices); the oracle takes about a second,
    ten seconds and a minute for them on 16 host cores."""
    from cfd_b200.channel import build_channel
    from cfd_b200.config import preset, tiny
    if cfgname.startswith("re"):
        cfg = preset(cfgname)
    else:
        cfg = {"tiny": tiny(), "tiny_ctp0": tiny(flag_ctpress=0, qxt=2.0, seed=11),
               "small_ib": tiny(ngal1=48, ngal2=36, ny=33, cyl_diameter=0.3, cyl_spacing=0.9, seed=5)}[cfgname]
    s = build_channel(cfg)
    o = oracle(s)
    o.step(10)
    ref = o.download_state()
    g = make(s, "fp64")
    g.step(10)
    st = g.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-10, (k, rel(st[k], ref[k]))
    g.close()
    m = make(s, "mixed")
    m.step(10)
    st = m.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-5, (k, rel(st[k], ref[k]))
    m.close()


def test_divergence_free_after_step(torch_cuda):
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny())
    g = make(s)
    g.step(3)
    assert g.divergence_max() < 1e-12
    g.close()


def test_layouts_round_trip(torch_cuda):
    from cfd_b200 import capi
    s, _ = load("tiny_ib_ctp1")
    g = make(s)
    a = g.download("u1", capi.LAYOUT_REF)
    b = g.download("u1", capi.LAYOUT_PLANE)
    np.testing.assert_array_equal(a, b.T)
    np.testing.assert_array_equal(a, s.u1)
    g.upload("u2", s.u2.T.copy(), capi.LAYOUT_PLANE)
    np.testing.assert_array_equal(g.download("u2"), s.u2)
    g.close()


def test_plane_transforms_match_oracle(torch_cuda):
    torch = torch_cuda
    s, _ = load("tiny_ib_ctp1")
    g = make(s)
    o = oracle(s)
    cfg = s.cfg
    rng = np.random.default_rng(0)
    npl = 3
    planes = np.zeros((npl, cfg.ngal2, cfg.ngal1 + 2))
    sp = rng.standard_normal((npl, cfg.n2, cfg.nkx, 2))
    rows = [q if q < cfg.n2 // 2 else q + cfg.ngal2 - cfg.n2 for q in range(cfg.n2)]
    for q in range(cfg.n2):
        planes[:, rows[q], 0:2 * cfg.nkx:2] = sp[:, q, :, 0]
        planes[:, rows[q], 1:2 * cfg.nkx:2] = sp[:, q, :, 1]
    exp = o.four_to_phys(planes.copy(), zero_oddball=True)
    d = torch.tensor(planes, device="cuda", dtype=torch.float64)
    lib = g.lib
    assert lib.cfd_four_to_phys(g.ctx, C.c_void_p(d.data_ptr()), npl, 1) == 0
    g.synchronize()
    got = d.cpu().numpy()
    np.testing.assert_allclose(got[:, :, :cfg.ngal1], exp[:, :, :cfg.ngal1], atol=1e-12)
    back = o.phys_to_four(exp.copy())
    assert lib.cfd_phys_to_four(g.ctx, C.c_void_p(d.data_ptr()), npl) == 0
    g.synchronize()
    got = d.cpu().numpy()
    for q in range(cfg.n2):
        np.testing.assert_allclose(got[:, rows[q], :2 * cfg.nkx], back[:, rows[q], :2 * cfg.nkx], atol=1e-12)
    g.close()


def test_rft_cft_entry_points(torch_cuda):
    torch = torch_cuda
    from oracle import oracle as O
    s, _ = load("tiny_ib_ctp1")
    g = make(s)
    n1, n2 = s.cfg.ngal1, s.cfg.ngal2
    rng = np.random.default_rng(2)
    m, isa = 5, n1 + 4
    x = np.zeros((m, isa))
    x[:, :n1] = rng.standard_normal((m, n1))
    d = torch.tensor(x, device="cuda")
    assert g.lib.cfd_rft(g.ctx, C.c_void_p(d.data_ptr()), isa, m, -1) == 0
    g.synchronize()
    exp = O.rft(x.ravel().copy(), n1, isa, m, -1).reshape(m, isa)
    np.testing.assert_allclose(d.cpu().numpy()[:, :n1 + 2], exp[:, :n1 + 2], atol=1e-14)
    # inverse of the same 5 lines (transformed two per complex FFT, the last one alone):
    # against the oracle and back to the input
    dy = torch.tensor(exp, device="cuda")
    assert g.lib.cfd_rft(g.ctx, C.c_void_p(dy.data_ptr()), isa, m, +1) == 0
    g.synchronize()
    expi = O.rft(exp.ravel().copy(), n1, isa, m, +1).reshape(m, isa)
    np.testing.assert_allclose(dy.cpu().numpy()[:, :n1], expi[:, :n1], atol=1e-13)
    np.testing.assert_allclose(dy.cpu().numpy()[:, :n1], x[:, :n1], atol=1e-12)
    ise, isa2, m2 = 6, 2, 3
    c = rng.standard_normal(ise * n2 + 8)
    dc = torch.tensor(c, device="cuda")
    assert g.lib.cfd_cft(g.ctx, C.c_void_p(dc.data_ptr()), ise, isa2, m2, +1) == 0
    g.synchronize()
    expc = O.cft(c.copy(), n2, ise, isa2, m2, +1)
    np.testing.assert_allclose(dc.cpu().numpy(), expc, atol=1e-12)
    g.close()


def test_errors_are_codes_not_crashes(torch_cuda):
    from cfd_b200 import capi
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny())
    g = Channel(s)
    assert g.lib.cfd_rk_substep(g.ctx, 1) == 5          # state not uploaded
    g.upload_state()
    assert g.lib.cfd_rk_substep(g.ctx, 4) == 1          # bad krk
    assert g.lib.cfd_upload_field(g.ctx, 99, None, 0) == 1
    assert g.lib.cfd_last_error(g.ctx)                   # a message is recorded
    g.close()
    with pytest.raises(capi.CfdError, match="2\\^a\\*3\\^b"):
        Channel(build_channel(tiny(ngal1=20, posth=0.0, cyl_diameter=0.0)))   # 20 is not 2^a 3^b


# grids whose x and z lengths cover every fixed-length transform (64, 96, 128, 192, 384, 768)
FIXED_GRIDS = [(64, 96, 17), (96, 192, 13), (128, 64, 13), (192, 128, 11), (384, 768, 9), (768, 384, 9)]


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
def test_fixed_length_transforms(torch_cuda, ng1, ng2, ny):
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=ng1 + ng2))
    assert s.ibu.n > 0
    o = oracle(s)
    o.rk_substep(1)
    ref1 = o.download_state()
    o.rk_substep(2)
    o.rk_substep(3)
    ref = o.download_state()
    g = make(s, "fp64")
    g.rk_substep(1)
    st = g.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref1[k]) < 1e-11, (k, rel(st[k], ref1[k]))
    g.rk_substep(2)
    g.rk_substep(3)
    st = g.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-10, (k, rel(st[k], ref[k]))
    g.close()
    m = make(s, "mixed")
    m.step(1)
    st = m.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-5, (k, rel(st[k], ref[k]))
    m.close()


@pytest.mark.parametrize("ng1,ng2,ny", [(96, 192, 13), (384, 768, 9)])
def test_stockham_nonlinear_path(torch_cuda, monkeypatch, ng1, ng2, ny):
    """The alternative nonlinear path (per-slot interpolating z pass + shared-memory Stockham
    x-line kernel, selected with CFD_XLINE_STOCKHAM=1) on two-step lengths, both precisions."""
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    monkeypatch.setenv("CFD_XLINE_STOCKHAM", "1")
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=ng1 + 2 * ng2))
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = make(s, prec)
        g.step(1)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        g.close()


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
def test_packed_xline_path(torch_cuda, monkeypatch, ng1, ng2, ny):
    """The packed x-line kernel (1.5 inverse lines per row, CFD_XLINE_PATH=3) on every
    two-step length, FP64 (1e-10 after one RK3 step) and mixed (1e-5), against the oracle."""
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    monkeypatch.setenv("CFD_XLINE_PATH", "3")
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=ng1 + ng2))
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = make(s, prec)
        if g.tuning()["xline_path"] != 3:  # a length whose packed CTA does not fit
            g.close()
            continue
        g.step(1)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        g.close()


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
def test_pair_xline_path(torch_cuda, monkeypatch, ng1, ng2, ny):
    """The line-pair x-line kernel (packed .f32x2 DFTs, CFD_XLINE_PATH=4) on every two-step
    length: mixed within 1e-5 of the oracle after one RK3 step and within 1e-6 of the scalar
    FP32 kernel (k_xline2) on u, v, w (1e-5 on p); an FP64 context asked for it runs the
    scalar path."""
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=ng1 + 2 * ng2))
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    monkeypatch.setenv("CFD_XLINE_PATH", "1")
    g1 = make(s, "mixed")
    assert g1.tuning()["xline_path"] == 1
    g1.step(1)
    scalar = g1.download_state()
    g1.close()
    monkeypatch.setenv("CFD_XLINE_PATH", "4")
    g = make(s, "mixed")
    assert g.tuning()["xline_path"] == 4
    g.step(1)
    st = g.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-5, (k, rel(st[k], ref[k]))
        # two FP32 paths: velocities within 1e-6, the pressure (the most sensitive field)
        # within the per-field bound of the mixed path
        assert rel(st[k], scalar[k]) < (1e-5 if k == "p" else 1e-6), (k, rel(st[k], scalar[k]))
    g.close()
    g = make(s, "fp64")
    assert g.tuning()["xline_path"] == 1
    g.close()


def test_ib_velocity_after_upload(torch_cuda):
    """The IB forcing reuses the nonlinear pass's z transforms of u, v, w; a field uploaded
    between cfd_nonlinear and cfd_solve_uvw must be transformed afresh.  Stage by stage with
    a different u, v, w uploaded after the nonlinear pass, against the oracle doing the same
    (FP64, 1e-11)."""
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(96, 64, 21, cyl_diameter=0.3, cyl_spacing=1.0))
    assert s.ibu.n > 0 and s.ibv.n > 0
    other = build_channel(tiny(96, 64, 21, cyl_diameter=0.3, cyl_spacing=1.0, seed=77)).state()
    g, o = make(s), oracle(s)
    for ch in (g, o):
        ch.rhs0(1)
        ch.nonlinear(1)
        for k in ("u1", "u2", "u3"):
            ch.upload(k, other[k])
        ch.solve_uvw(1)
    for k in FIELDS:
        e = rel(g.download(k), o.download(k))
        assert e < 1e-11, (k, e)
    g.close()


def test_largest_workload_properties(torch_cuda):
    """The largest named workload (re1000: 768 x 385 x 768 + canopy planes, 131,584 columns,
    2.2 M IB points per grid), where the oracle is too slow to run: one RK3 step in FP64 is
    divergence-free to round-off with finite mean-mode scalars, and the FP32-mixed step
    agrees with it to 1e-5 (relative L2 of u, v, w and p)."""
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import preset
    s = build_channel(preset("re1000"))
    out = {}
    for prec in ("fp64", "mixed"):
        g = Channel(s, device=0, precision=prec)
        g.upload_state()
        g.step(1)
        sc = g.scalars()
        assert all(np.isfinite(v) for v in sc.values()), sc
        if prec == "fp64":
            assert g.divergence_max() < 1e-11
        out[prec] = {k: g.download(k) for k in ("u1", "u2", "u3", "p")}
        g.close()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(out["mixed"][k], out["fp64"][k]) < 1e-5, k


@pytest.mark.parametrize("name", ("tiny_ib_ctp1", "tiny_ib_ctp0"))
def test_lastplane_mode_vs_oracle(torch_cuda, name):
    """The single-slab x/z advective term (cfd_set_lastplane, the reference's 2-D scratch of
    ops_in_planes with one rank) against the oracle's emulation of the same, stage by stage
    (FP64, 1e-11) and over two RK3 steps in both precisions (1e-10 / 1e-5); switching it off
    again returns to the per-plane path."""
    from oracle.oracle import OracleChannel
    s, _ = load(name)
    g = make(s)
    g.set_lastplane(True)
    o = OracleChannel(s, quirk_lastplane=True)
    o.upload_state()
    for stage in STAGES:
        getattr(g, stage)(1)
        getattr(o, stage)(1)
        for k in FIELDS:
            e = rel(g.download(k), o.download(k))
            assert e < 1e-11, (stage, k, e)
    g.close()
    o = OracleChannel(s, quirk_lastplane=True)
    o.upload_state()
    o.step(2)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = make(s, prec)
        g.set_lastplane(True)
        g.step(2)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        g.close()
    # off again: the per-plane oracle
    plain = oracle(s)
    plain.step(2)
    ref = plain.download_state()
    g = make(s)        # fresh context: a step would advance mpgx under constant flow rate
    g.set_lastplane(True)
    g.set_lastplane(False)
    g.step(2)
    st = g.download_state()
    for k in ("u1", "u2", "u3", "p"):
        assert rel(st[k], ref[k]) < 1e-10, k
    g.close()


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
def test_transposed_splits(torch_cuda, ng1, ng2, ny):
    """The other radix order of the two-step transforms (cfd_tuning xsplit = zsplit = 2: the
    first register DFT runs over N2 points instead of N1) on every two-step length, against
    the oracle after one RK3 step: FP64 within 1e-10, FP32-mixed within 1e-5 (u, v, w, p)."""
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=3 * ng1 + ng2))
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = Channel(s, device=0, precision=prec, tuning=dict(xline_path=1, xsplit=2, zsplit=2))
        t = g.tuning()
        assert t["xsplit"] == 2 and t["zsplit"] == 2, t
        g.upload_state()
        g.step(1)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        g.close()


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
@pytest.mark.parametrize("xsplit", [1, 2])
def test_register_capped_xline(torch_cuda, monkeypatch, ng1, ng2, ny, xsplit):
    """The FP32 x-line kernel held to 64 registers (x-line path 5, k_xline2r; FP64 contexts
    run path 1) and the FP64 nonlinear z kernels held to 112 (k_zinv2sd / k_zfwd2d, the
    default for z lengths up to 384) on every two-step length and both radix orders, against
    the oracle after one RK3 step (FP64 within 1e-10, FP32-mixed within 1e-5 on u, v, w, p)."""
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    monkeypatch.setenv("CFD_Z_R112", "1")
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=5 * ng1 + ng2))
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = Channel(s, device=0, precision=prec, tuning=dict(xline_path=5, xsplit=xsplit, zsplit=xsplit))
        assert g.tuning()["xline_path"] == (5 if prec == "mixed" else 1)
        g.upload_state()
        g.step(1)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        g.close()


@pytest.mark.parametrize("ng1,ng2,ny", FIXED_GRIDS)
def test_marching_xline(torch_cuda, monkeypatch, ng1, ng2, ny):
    """The x-line pass marching in y (x-line path 6, k_xmarch; FP32-mixed only) on every
    length it takes (64, 96, 128, 192, 384; 768 and FP64 contexts run path 1), with 2 and 4
    rows per CTA and y-chunks of 2, 3 and 32 steps (chunk boundaries at every position of
    the interpolation stencil): within 1e-5 of the oracle after one RK3 step on u, v, w, p,
    and within 1e-6 of the per-slot FP32 kernel on u, v, w (1e-5 on p)."""
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(ngal1=ng1, ngal2=ng2, ny=ny, cyl_diameter=0.3, cyl_spacing=1.5, seed=3 * ng1 + ng2))
    assert s.ibu.n > 0
    o = oracle(s)
    o.step(1)
    ref = o.download_state()
    g1 = Channel(s, device=0, precision="mixed", tuning=dict(xline_path=1))
    g1.upload_state()
    g1.step(1)
    scalar = g1.download_state()
    g1.close()
    for rows in (2, 4):
        for chunk in (2, 3, 32):
            monkeypatch.setenv("CFD_XMARCH_STEPS", str(chunk))
            g = Channel(s, device=0, precision="mixed", tuning=dict(xline_path=6, xline_rows=rows))
            if ng1 == 768:
                assert g.tuning()["xline_path"] == 1
                g.close()
                return
            assert g.tuning()["xline_path"] == 6 and g.tuning()["xline_rows"] == rows
            g.upload_state()
            g.step(1)
            st = g.download_state()
            for k in ("u1", "u2", "u3", "p"):
                assert rel(st[k], ref[k]) < 1e-5, (rows, chunk, k, rel(st[k], ref[k]))
                assert rel(st[k], scalar[k]) < (1e-5 if k == "p" else 1e-6), (rows, chunk, k, rel(st[k], scalar[k]))
            g.close()
    g = Channel(s, device=0, precision="fp64", tuning=dict(xline_path=6))
    assert g.tuning()["xline_path"] == 1
    g.close()
