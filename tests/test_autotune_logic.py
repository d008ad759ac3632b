"""The autotuner's coordinate search and cache (cfd_b200.autotune) with a fake timing model
in place of the device (CPU)."""
import json

import pytest

from cfd_b200 import autotune

DEFAULT = {"xline_path": 1, "xline_rows": 4, "zlines": 16, "solve_kind": 1, "solve_cols": 64, "rhs_chunk": 16,
           "xsplit": 1, "zsplit": 1}


def fake_model(calls, bad=()):
    """Seconds per step: a cost with its minimum at x-line path 5 with the transposed x split
    (path 5 alone and the split alone are each worse than path 1 with the default split),
    xline_rows 4, zlines 16, rhs_chunk 4, 128 threads per column-sweep CTA and the default z
    split; path 2 is slow; shapes in `bad` raise."""
    def time_step(setup, precision, device, tuning, steps=5, warmup=2):
        eff = dict(DEFAULT, **(tuning or {}))
        if eff["xline_path"] not in (1, 5):
            eff["xsplit"] = 1  # the x split acts on paths 1 and 5 only
        if eff["xline_path"] not in (1, 5, 6):
            eff["zsplit"] = 1  # the z split on paths 1, 5 and 6
        for k, v in bad:
            if eff.get(k) == v:
                raise RuntimeError(f"{k}={v} does not fit")
        calls.append(json.dumps(eff, sort_keys=True))
        t = 10.0
        t += {1: 0.0, 2: 3.0, 3: 0.5, 4: 0.8, 5: 0.2, 6: 0.1}[eff["xline_path"]]
        if eff["xline_path"] == 5 and eff["xsplit"] == 2:
            t -= 0.5   # an interaction a one-knob-at-a-time search from path 1 would miss
        t += {2: 0.4, 4: 0.0, 8: 0.2}[eff["xline_rows"]]
        t += {4: 0.5, 8: 0.3, 16: 0.0}[eff["zlines"]]
        t += {2: 0.2, 4: 0.0, 8: 0.1, 16: 0.3}[eff["rhs_chunk"]]
        t += {64: 0.1, 128: 0.0, 256: 0.05}[eff["solve_cols"]]
        t += {1: 0.1, 2: 0.0}[eff["xsplit"]] + {1: 0.0, 2: 0.2}[eff["zsplit"]]
        return t * 1e-3, eff
    return time_step


def test_coordinate_search_finds_the_separable_minimum(monkeypatch):
    calls = []
    monkeypatch.setattr(autotune, "time_step", fake_model(calls))
    best, t = autotune.autotune(None, "mixed")
    assert best["xline_path"] == 5 and best["xline_rows"] == 4 and best["zlines"] == 16
    assert best["solve_kind"] == 1 and best["rhs_chunk"] == 4 and best["solve_cols"] == 128
    assert best["xsplit"] == 2 and best["zsplit"] == 1
    assert t == pytest.approx(9.7e-3)
    assert len(calls) == len(set(calls)), "a shape was timed twice"


def test_shapes_that_do_not_fit_are_skipped(monkeypatch):
    calls = []
    monkeypatch.setattr(autotune, "time_step", fake_model(calls, bad=(("xline_rows", 2),)))
    logs = []
    best, _ = autotune.autotune(None, "mixed", log=logs.append)
    assert best["xline_rows"] == 4 and best["rhs_chunk"] == 4
    assert any(m.startswith("skip") for m in logs)


def test_cache_is_written_once_and_reused(monkeypatch, tmp_path):
    torch = pytest.importorskip("torch")
    calls = []
    monkeypatch.setattr(autotune, "time_step", fake_model(calls))
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda device=None: "FAKE B200")
    monkeypatch.setenv("CFD_TUNE_CACHE", str(tmp_path / "sub" / "tune.json"))

    class G:
        nyu = 33

    class Cfg:
        ngal1, ngal2 = 64, 96

    class IB:
        n = 5

    class S:
        cfg, grid, ibu = Cfg, G, IB

    first = autotune.tuned(S, "mixed")
    n = len(calls)
    assert n > 0 and first["xline_rows"] == 4
    again = autotune.tuned(S, "mixed")
    assert again == first and len(calls) == n, "the cached tuning was measured again"
    data = json.load(open(tmp_path / "sub" / "tune.json"))
    (key,) = data
    assert "FAKE B200" in key and "64x33x96" in key and key.endswith("ibTrue")
    other = autotune.tuned(S, "fp64")
    assert len(calls) > n and len(json.load(open(tmp_path / "sub" / "tune.json"))) == 2
    # FP64 searches the x-line paths it runs (1-3) and otherwise reaches the same shape
    assert other["xline_path"] == 1 and first["xline_path"] == 5
    assert {k: v for k, v in other.items() if k != "xline_path"} == {k: v for k, v in first.items() if k != "xline_path"}


def test_fp64_skips_the_mixed_only_xline_paths(monkeypatch):
    """FP64 contexts run x-line path 1 when asked for paths 4, 5 or 6, so the FP64 search
    does not time them."""
    calls = []
    monkeypatch.setattr(autotune, "time_step", fake_model(calls))
    autotune.autotune(None, "fp64")
    assert not any(json.loads(c)["xline_path"] in (4, 5, 6) for c in calls)
    calls.clear()
    autotune.autotune(None, "mixed")
    assert {json.loads(c)["xline_path"] for c in calls} >= {1, 2, 3, 4, 5, 6}

