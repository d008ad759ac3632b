"""bench.py's compulsory-traffic model covers every kernel of the default RK3 step, so the
per-kernel HBM fractions of the bench line are never empty (CPU)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

STEP_KERNELS = ("k_zinv2s", "k_xline2", "k_zfwd2", "k_rhs", "k_solve_uvw", "k_solve_p_vcorr", "k_meanflow",
                "k_ib_zinv2", "k_ib_xinv2", "k_ib_force", "k_ib_xfwd2", "k_ib_zfwd2")


@pytest.fixture(scope="module")
def setup():
    from cfd_b200.channel import build_channel
    from cfd_b200.config import preset
    return build_channel(preset("re180"))


@pytest.mark.parametrize("mixed", (True, False))
def test_every_step_kernel_is_modelled(setup, mixed):
    import bench
    for k in STEP_KERNELS:
        b = bench.kernel_bytes(k, setup, mixed)
        assert b is not None and b > 0, k


def test_step_roofline_model(setup):
    import bench
    r = bench.step_roofline(setup, True, 1e-3, 1000.0)
    S = setup.cfg.ncol * setup.grid.nyv
    assert r["model_bytes_per_substep"] == 608 * S
    assert r["achieved_gbs"] == pytest.approx(3 * 608 * S / 1e-3 / 1e9)
