"""bench.py's compulsory-traffic model covers every kernel of the default RK3 step (both
x-line kernels: the marching one of FP32-mixed, the per-slot one of FP64), so the per-kernel
HBM fractions of the bench line are never empty (CPU)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

STEP_KERNELS = ("k_zinv2s", "k_xline2", "k_xmarch", "k_zfwd2", "k_rhs", "k_solve_uvw", "k_solve_p_vcorr",
                "k_meanflow", "k_ib_zinv2", "k_ib_xinv2", "k_ib_force", "k_ib_xfwd2", "k_ib_zfwd2")


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


class _FakeChannel:
    """Host stand-in for a Channel: records the dt of every block of steps and returns
    plane sums whose values depend on the dt sequence it was given."""

    def __init__(self, setup, dt_seq=None, fail_after=None):
        self.setup, self.dt, self.log, self.fail_after = setup, setup.dt, [], fail_after
        self.dt_seq = list(dt_seq or [])
        self.acc = None
        self.nadapt = 0
        self.uploads = []

    def upload_state(self, state=None):
        self.log.clear()
        self.started_from = state
        self.uploads.append(state)

    def download_state(self):
        import numpy as np
        return {k: np.full(3, 1.0 + len(self.log), dtype=np.complex128) for k in ("u1", "u2", "u3", "p")}

    def adapt_dt(self):
        self.dt = self.dt_seq[self.nadapt]
        self.nadapt += 1
        return self.dt

    def set_dt(self, dt):
        self.dt = dt

    def step(self, n):
        self.log.append((self.dt, n))
        if self.fail_after is not None and len(self.log) > self.fail_after:
            self.nonfinite = True

    def cfl(self):
        if getattr(self, "nonfinite", False):
            raise RuntimeError("cfl: CFD_ERR_NONFINITE: non-finite velocity in the physical planes")
        return 1.0, [1.0, 1.0, 1.0]

    def stats_configure(self, *a):
        self.acc = 0

    def stats_accumulate(self):
        self.acc += 1

    def stats_read(self):
        import numpy as np
        ny = 4
        s = float(sum(d for d, _ in self.log))
        st = {"istat": self.acc}
        for m in ("Um", "Vm", "Wm"):
            st[m] = np.full(ny, s * self.acc)
        for m in ("U2m", "V2m", "W2m"):
            st[m] = np.full(ny, 2 * s * s * self.acc)
        return st


def test_profile_error_replays_the_fp64_dt_sequence(setup):
    """The statistics window re-chooses dt from the FP64 state every nstat steps and the
    mixed path integrates with the same sequence; the caller's dt is restored after."""
    import bench
    seq = [1e-3 * (1 + 0.01 * k) for k in range(10)]
    f64, mix = _FakeChannel(setup, seq), _FakeChannel(setup)
    out = bench.profile_error({"fp64": f64, "mixed": mix}, setup, spinup=40, nsteps=60, nstat=20, shared=False)
    assert [n for _, n in f64.log] == [20] * 5 and f64.log == mix.log
    # the chaos-floor run: FP64 again, from the FP32-rounded start, with the same dt sequence
    assert mix.started_from["u1"] is setup.state()["u1"]  # both spin up from the seeded start
    assert f64.started_from["u1"].dtype == "complex128"
    assert max(out["chaos_floor_max_rel_diff"].values()) == 0.0
    assert [d for d, _ in f64.log] == seq[:5]
    assert f64.dt == setup.dt and mix.dt == setup.dt
    assert out["steps"] == 60 and out["within_bound"] and max(out["max_rel_diff"].values()) == 0.0
    assert out["dt_first_last_min_max"] == [seq[0], seq[4], seq[0], seq[4]]


def test_profile_error_shared_spinup(setup):
    """With one shared spin-up, FP64 spins up once (re-choosing dt every nstat steps), then
    FP64, mixed and the FP32-rounded FP64 run each average from the spun-up state with the
    FP64 averaging window's dt sequence."""
    import bench
    seq = [1e-3 * (1 + 0.01 * k) for k in range(10)]
    f64, mix = _FakeChannel(setup, seq), _FakeChannel(setup)
    out = bench.profile_error({"fp64": f64, "mixed": mix}, setup, spinup=40, nsteps=60, nstat=20)
    assert out["spinup"].startswith("one FP64 spin-up")
    spun = f64.uploads[1]
    assert f64.uploads[0]["u1"].shape == setup.state()["u1"].shape  # the seeded start
    assert float(spun["u1"][0].real) == 3.0       # downloaded after the 2 spin-up blocks
    assert mix.uploads == [spun]
    assert float(f64.uploads[2]["u1"][0].real) == 3.0 and f64.uploads[2]["u1"].dtype == "complex128"
    # averaging window: 3 blocks after the 2 spin-up blocks, the same dts in every run
    assert [d for d, _ in mix.log] == seq[2:5] and f64.log == mix.log
    assert out["dt_first_last_min_max"] == [seq[0], seq[4], seq[0], seq[4]]
    assert f64.dt == setup.dt and mix.dt == setup.dt and out["within_bound"]


def test_profile_error_reports_a_blow_up(setup):
    """A state that goes non-finite ends the window with the error and the block it
    happened in, instead of NaN profiles."""
    import bench
    seq = [1e-3] * 10
    for shared, fail_after in ((False, 3), (True, 1)):
        f64 = _FakeChannel(setup, seq, fail_after=fail_after)
        out = bench.profile_error({"fp64": f64, "mixed": _FakeChannel(setup)}, setup, spinup=40, nsteps=60,
                                  nstat=20, shared=shared)
        assert "error" in out and "NONFINITE" in out["error"] and "within_bound" not in out
        assert f64.dt == setup.dt


def test_top_kernel_profile_rows():
    """The roofline's ncu traffic and FP32-pipe rows of the default top kernels are committed
    (profiles/dram_traffic_re550.md, profiles/fp32_ops_re550.md)."""
    import bench
    for k in ("k_xmarch", "k_xline2"):
        assert bench.ncu_traffic("re550", k) > 0, k
        assert bench.fp32_pipe("re550", k, 0.5, {"sm_mhz": 1965.0})["fp32_ops_per_launch"] > 0, k

