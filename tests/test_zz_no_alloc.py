"""The allocation-free Helmholtz solve (cfd_lusol_u_noalloc) against the context path.

It serves callers that cannot call cudaMalloc/cudaFree (device memory owned by another
allocator or capped, or loops that must not take cudaFree's implicit synchronisation).
Two calls in a row (the u and w right-hand sides of one substep) must reproduce what
cfd_solve_uvw computes for a smooth channel, where that stage is prologue + LUsolU only.
This file is collected last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-11  # FP64 relative L2, as the other FP64 parity tests


def test_noalloc_solve_matches_context_path():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cfd_b200 import capi
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    from cfd_b200.grid import grid_weights, wavenumbers

    cfg = tiny(ngal1=36, ngal2=24, ny=21, posth=0.0, cyl_diameter=0.0, seed=21)
    s = build_channel(cfg)
    ch = Channel(s, device=0, precision="fp64")
    ch.upload_state()
    ch.rhs0(1)
    ch.nonlinear(1)
    du = {k: ch.download(k, capi.LAYOUT_PLANE) for k in ("du1", "du3")}
    u = {k: ch.download(k, capi.LAYOUT_PLANE) for k in ("u1", "u3")}
    ch.solve_uvw(1)
    expect = {k: ch.download(k, capi.LAYOUT_PLANE) for k in ("u1", "u3")}
    ch.close()

    g = s.grid
    kx, kz = wavenumbers(cfg.n1, cfg.n2, cfg.alp, cfg.bet)
    gwb, gwt, _, _ = grid_weights(g)
    beta = (4.0 / 15.0) * s.dt / cfg.re_b
    dev = torch.device("cuda", 0)
    kx_d = torch.tensor(kx, dtype=torch.float64, device=dev)
    kz_d = torch.tensor(kz, dtype=torch.float64, device=dev)
    dy_d = torch.tensor(np.ascontiguousarray(g.dyu2i), dtype=torch.float64, device=dev)
    lib = capi.load()
    for a, b in (("u1", "du1"), ("u3", "du3")):
        rhs = u[a] + s.dt * du[b]          # solveU prologue (littleharsh.f90:748-753)
        rhs[0] = 0.0
        rhs[-1] = 0.0
        r_d = torch.from_numpy(np.ascontiguousarray(rhs).view(np.float64)).to(dev)
        x_d = torch.empty_like(r_d)
        st = lib.cfd_lusol_u_noalloc(cfg.nkx, cfg.n2, g.nyu, beta, gwb, gwt, kx_d.data_ptr(), kz_d.data_ptr(),
                                     dy_d.data_ptr(), r_d.data_ptr(), x_d.data_ptr(), None)
        assert st == capi.CFD_OK
        torch.cuda.synchronize()
        got = x_d.cpu().numpy().view(np.complex128).reshape(expect[a].shape)
        err = np.linalg.norm(got - expect[a]) / np.linalg.norm(expect[a])
        assert err < TOL, (a, err)
        # in place: the right-hand side buffer receives the solution
        st = lib.cfd_lusol_u_noalloc(cfg.nkx, cfg.n2, g.nyu, beta, gwb, gwt, kx_d.data_ptr(), kz_d.data_ptr(),
                                     dy_d.data_ptr(), r_d.data_ptr(), r_d.data_ptr(), None)
        assert st == capi.CFD_OK
        torch.cuda.synchronize()
        assert torch.equal(r_d, x_d), a

    # sizes above the fixed scratch are refused before any GPU work
    too_many = capi.CFD_OK
    big = (16 * 1024 * 1024) // (cfg.nkx * cfg.n2) + 2
    too_many = lib.cfd_lusol_u_noalloc(cfg.nkx, cfg.n2, big, beta, gwb, gwt, kx_d.data_ptr(), kz_d.data_ptr(),
                                       dy_d.data_ptr(), r_d.data_ptr(), x_d.data_ptr(), None)
    assert too_many == 2  # CFD_ERR_SIZE
