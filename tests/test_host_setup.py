"""Host set-up: y-grid, IB lists and initial fields keep the reference's invariants."""
import numpy as np
import pytest

from cfd_b200.channel import build_channel
from cfd_b200.config import preset, tiny
from cfd_b200.geometry import lattice_params
from cfd_b200.grid import grid_weights, wavenumbers, y_grid_rough


@pytest.mark.parametrize("ny,posth", [(17, 0.12), (97, 0.1), (33, 0.0)])
def test_y_grid_crests_and_symmetry(ny, posth):
    g = y_grid_rough(ny, 10.0, 5, posth)
    assert g.v(0) == pytest.approx(-1.0, abs=1e-14)
    assert g.v(ny - 1) == pytest.approx(1.0, abs=1e-14)
    assert g.v(g.jv0) == pytest.approx(-1.0 - posth, abs=1e-12)
    np.testing.assert_allclose(g.yu, -g.yu[::-1], atol=1e-13)
    np.testing.assert_allclose(g.yv, -g.yv[::-1], atol=1e-13)
    assert np.all(np.diff(g.yu) > 0) and np.all(np.diff(g.yv) > 0)


def test_second_derivative_exact_on_quadratics():
    g = y_grid_rough(33, 10.0, 5, 0.1)
    f = 3.0 * g.yu ** 2 - g.yu + 2.0
    for jj in range(1, g.nyu - 2):
        c = g.dyu2i[jj]
        assert c[0] * f[jj - 1] + c[1] * f[jj] + c[2] * f[jj + 1] == pytest.approx(6.0, rel=1e-8)


def test_ghost_weights_extrapolate_zero_at_wall():
    g = y_grid_rough(17, 3.0, 5, 0.12)
    gwb, gwt, _, _ = grid_weights(g)
    # u(g) = -gw u(1) puts the linear interpolant to zero at the wall face
    ug, u1 = -gwb * 1.0, 1.0
    yw, yg, y1 = g.v(g.jv0), g.u(g.ju0), g.u(g.ju0 + 1)
    assert ug + (u1 - ug) * (yw - yg) / (y1 - yg) == pytest.approx(0.0, abs=1e-14)


def test_ib_lists_sorted_in_range_and_weighted():
    s = build_channel(tiny(), with_fields=False)
    for lst in (s.ibu, s.ibv):
        idx = lst.idx
        key = (idx[:, 2].astype(np.int64) * 10000 + idx[:, 1]) * 10000 + idx[:, 0]
        assert np.all(np.diff(key) >= 0)
        for col in (0, 3, 6):
            assert idx[:, col].min() >= 1 and idx[:, col].max() <= s.cfg.ngal1
        for col in (1, 4, 7):
            assert idx[:, col].min() >= 1 and idx[:, col].max() <= s.cfg.ngal2
        inr = np.zeros(len(idx), bool)
        for side in (0, 1):
            inr |= (idx[:, 2] >= lst.jlo[side]) & (idx[:, 2] <= lst.jhi[side])
        assert inr.all()
        assert set(np.unique(lst.w[:, 0])) <= {0.0, 1.0}


@pytest.mark.parametrize("name", ["re395", "re550", "re1000"])
def test_baseline_lattices_fit(name):
    cfg = preset(name)
    ntx, ntz, dnx, dnz, r, ci, ck = lattice_params(cfg)
    assert cfg.ngal1 % ntx == 0 and ntx % 2 == 0 and cfg.ngal2 % ntz == 0
    assert r > 0.5


def test_initial_field_divergence_free_and_hermitian():
    cfg = tiny()
    s = build_channel(cfg)
    g = s.grid
    kx, kz = wavenumbers(cfg.n1, cfg.n2, cfg.alp, cfg.bet)
    i = np.arange(cfg.ncol) % cfg.nkx
    q = np.arange(cfg.ncol) // cfg.nkx
    div = (1j * kx[i][:, None] * s.u1[:, 1:-1] + 1j * kz[q][:, None] * s.u3[:, 1:-1] +
           g.dthdyu[None, 1:-1] * (s.u2[:, 1:] - s.u2[:, :-1]))
    assert np.abs(div).max() < 1e-12
    for qq in range(1, cfg.n2 // 2):
        a, b = qq * cfg.nkx, (cfg.n2 - qq) * cfg.nkx
        np.testing.assert_allclose(s.u1[a], np.conj(s.u1[b]), atol=1e-14)
    assert np.all(s.u2[:, 0] == 0) and np.all(s.u2[:, -1] == 0)
    assert s.dt > 0
