"""The oracle's emulation of the reference's single-slab x/z advective term.

ops_in_planes (FOU3D.f90:1529-1617) forms der_x/der_z of each plane's products into 2-D
scratch arrays (du1dx, du1dz, ... `:1541`) inside the plane loop and adds them into
Nu1PL/Nu3PL/Nu2PL in a second loop after it (`:1578-1585`, `:1607-1613`), so every interior
plane of a rank receives the derivative of the LAST plane of its loop: the top ghost centre
for the u/w grid (limPL_incw(ugrid,2)) and the top wall face for v.  The oracle reproduces
this for one slab (orc_set_quirk); the product path and the oracle's default use the
per-plane value.  The expected values here come from the numpy restatement's own transforms
(pocketfft), not from the oracle.
"""
import numpy as np
import pytest

from fixtures import load
from numpy_ref import NumpyChannel
from oracle.oracle import OracleChannel


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _xz_terms(n: NumpyChannel, st):
    """Per-plane x/z advective terms (der_x + der_z of the products) of state `st`."""
    g = n.g
    yu, yv = g.yu, g.yv
    u1, u2, u3 = st["u1"], st["u2"], st["u3"]
    u2i = np.zeros((n.ncol, g.nyu), np.complex128)
    for jj in range(1, g.nyu - 1):
        u2i[:, jj] = ((yu[jj] - yv[jj - 1]) * u2[:, jj] + (yv[jj] - yu[jj]) * u2[:, jj - 1]) / (yv[jj] - yv[jj - 1])
    u2i[:, 0] = n.gwib * (u2[:, 0] - u2i[:, 1]) + u2i[:, 1]
    u2i[:, -1] = n.gwit * (u2[:, -1] - u2i[:, -2]) + u2i[:, -2]
    u1i = np.zeros((n.ncol, g.nyv), np.complex128)
    u3i = np.zeros_like(u1i)
    for jj in range(g.nyv):
        w0, w1, den = yv[jj] - yu[jj], yu[jj + 1] - yv[jj], yu[jj + 1] - yu[jj]
        u1i[:, jj] = (w0 * u1[:, jj + 1] + w1 * u1[:, jj]) / den
        u3i[:, jj] = (w0 * u3[:, jj + 1] + w1 * u3[:, jj]) / den
    zrow = n.q == n.n2 // 2

    def dxz(a, b):
        v = 1j * n.kx * a + 1j * n.kz * b
        v[zrow] = 0.0
        return v
    x1 = np.zeros((n.ncol, g.nyu), np.complex128)
    x3 = np.zeros_like(x1)
    for jj in range(g.nyu):
        U, V, W = n.to_phys(u1[:, jj]), n.to_phys(u2i[:, jj]), n.to_phys(u3[:, jj])
        uu, uw, ww = n.to_spec(U * U), n.to_spec(U * W), n.to_spec(W * W)
        x1[:, jj], x3[:, jj] = dxz(uu, uw), dxz(uw, ww)
    x2 = np.zeros((n.ncol, g.nyv), np.complex128)
    for jj in range(g.nyv):
        U, V, W = n.to_phys(u1i[:, jj]), n.to_phys(u2[:, jj]), n.to_phys(u3i[:, jj])
        x2[:, jj] = dxz(n.to_spec(U * V), n.to_spec(W * V))
    return x1, x2, x3


@pytest.mark.parametrize("name", ("tiny_ib_ctp1", "tiny_smooth"))
def test_lastplane_quirk(name):
    s, _ = load(name)
    st = s.state()
    plain = OracleChannel(s)
    quirk = OracleChannel(s, quirk_lastplane=True)
    for o in (plain, quirk):
        o.upload_state(st)
        o.nonlinear(1)
    x1, x2, x3 = _xz_terms(NumpyChannel(s), st)
    for name_, x, top in (("nu1", x1, -1), ("nu3", x3, -1), ("nu2", x2, -1)):
        a, b = plain.download(name_), quirk.download(name_)
        # the y-derivative part is the same in both; the x/z part differs
        ypart = a[:, 1:-1] - x[:, 1:-1]
        got = b[:, 1:-1] - ypart
        want = np.repeat(x[:, top][:, None], got.shape[1], axis=1)
        # (the last v plane is the top wall, where v = 0: its term is exactly zero)
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(x[:, 1:-1]), name_
        # and the plain oracle really is per-plane: planes differ from the last one
        assert np.linalg.norm(a[:, 1:-1] - ypart - want) > 1e-3 * np.linalg.norm(x[:, 1:-1]), name_
        # boundary rows carry no advective term in either form
        assert np.all(b[:, 0] == 0) and np.all(b[:, -1] == 0), name_
