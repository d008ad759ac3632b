"""Benchmark of the channel-DNS hot path on B200: RK3 steps/s and grid-point updates/s,
FP32-mixed vs FP64, with the error of the mixed path against the FP64 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config re550] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  The path does not shard (each channel lives on
one GPU), so N > 1 runs N independent replicas ("scaling": "weak"); `value` is the
aggregate over ranks, timed as the max over ranks.  Inputs (GBs of spectral state) are far
larger than the 126 MB L2, so no flush is needed between steps.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 steps/s and grid-pt updates/s: FP32-mixed vs FP64 on 1 B200 at stated error"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel (compulsory traffic: every operand read once,
# every result written once)
# ------------------------------------------------------------------------------------------
def kernel_bytes(name, setup, mixed):
    cfg, g = setup.cfg, setup.grid
    ncol, nyu, nyv, nyp = cfg.ncol, g.nyu, g.nyv, g.nyp
    cs, ct = 16, (8 if mixed else 16)
    hpl = cfg.ngal2 * cfg.nkx                 # half-physical plane (complex values)
    nslot = nyu + nyv
    nplu = sum(max(0, min(h, g.ju1 - 1) - max(l, g.ju0 + 1) + 1) for l, h in zip(setup.ibu.jlo, setup.ibu.jhi))
    nplv = sum(max(0, min(h, g.jv1 - 1) - max(l, g.jv0 + 1) + 1) for l, h in zip(setup.ibv.jlo, setup.ibv.jhi))
    phys = cfg.ngal1 * cfg.ngal2
    rt = 4 if mixed else 8
    nfp = 2 * nyu + nyv                       # field planes u, w, v
    b = {
        "k_zinv": nfp * ncol * cs + 3 * nslot * hpl * ct,
        "k_zinv2s": nfp * ncol * cs + nfp * hpl * ct,
        "k_xline": (3 * nslot + 4 * nyu + 2 * nyv) * hpl * ct,
        # reads every transformed field plane once (y-neighbours of the interpolation from L2)
        "k_xline2": (nfp + 4 * nyu + 2 * nyv) * hpl * ct,
        "k_xline4": (nfp + 4 * nyu + 2 * nyv) * hpl * ct,   # the same pass on packed line pairs
        # the pass marching in y: every field plane read once, the products written once
        "k_xmarch": (nfp + 4 * nyu + 2 * nyv) * hpl * ct,
        "k_zfwd": (4 * nyu + 2 * nyv) * (hpl + ncol) * ct,
        "k_rhs": ncol * ((2 * nyu + nyv + nyp) * cs + (2 * nyu + nyv) * ct + (4 * nyu + 2 * nyv) * ct
                         + (2 * nyu + nyv) * cs + (2 * nyu + nyv) * ct),
        "k_solve_uvw": ncol * 2 * (2 * nyu + nyv) * cs,
        "k_solve_uvw_r": ncol * 2 * (2 * nyu + nyv) * cs,   # the warp-per-column form, same bytes
        "k_solve_p": ncol * (2 * nyu + nyv + nyp + 2 * nyp) * cs,
        # fused pressure solve + correction: u, v, w read twice and written once; p read and
        # written; psi and the scaled upper diagonal (FP64 real) written and read once
        "k_solve_p_vcorr": ncol * (3 * nfp * cs + nyp * (4 * cs + 2 * 8)),
        "k_vcorr": ncol * (2 * (2 * nyu + nyv) + nyp) * cs,
        # mean mode, one thread: the flow-rate integral reads yv and u(kx=kz=0) per plane
        # (constant pressure gradient; the constant-flow-rate solve adds a one-column sweep)
        "k_meanflow": nyu * (8 + cs),
    }
    # IB kernels: average over the u-grid (2 batches: u, w) and v-grid (1 batch) launches.
    # z: the inverse transforms the right-hand sides only (the velocities' transforms come
    # from the nonlinear pass).  x: only the z rows holding a forcing or stencil point
    # (`nact` of them) make the round trip; the inverse reads the half-physical rows of the
    # right-hand side and of the velocity and writes both physical rows, the forward reads
    # the forced right-hand side row and writes its half-physical row.
    ib = []
    for npl, nb, lst in ((nplu, 2, setup.ibu), (nplv, 1, setup.ibv)):
        if npl:
            nact = int(np.unique(lst.idx[:, [1, 4, 7]]).size) if lst.n else 0
            xi = lambda rows: npl * nb * rows * (2 * cfg.nkx * ct + 2 * cfg.ngal1 * (ct // 2))
            xf = lambda rows: npl * nb * rows * (cfg.ngal1 * (ct // 2) + cfg.nkx * ct)
            # force: per point its 9 indices and 3 weights, the target's rhs and u, the two
            # stencil values of u, and the target's rhs written back (physical, real)
            ib.append({"k_ib_force": nb * lst.n * (9 * 4 + 3 * 8 + 5 * (ct // 2)),
                       "k_ib_zinv": npl * nb * (ncol * cs + hpl * ct),
                       "k_ib_zfwd": npl * nb * (hpl * ct + ncol * cs),
                       "k_ib_xinv2": xi(nact), "k_ib_xfwd2": xf(nact),          # active rows
                       "k_ib_xinv": xi(cfg.ngal2), "k_ib_xfwd": xf(cfg.ngal2)})  # every row
    for k in ("k_ib_force", "k_ib_zinv", "k_ib_zfwd", "k_ib_xinv2", "k_ib_xfwd2", "k_ib_xinv", "k_ib_xfwd"):
        if ib:
            b[k] = sum(x[k] for x in ib) / len(ib)
    if name in b:
        return b[name]
    return b.get(name[:-1]) if name.endswith("2") else None


def kernel_table(prof, setup, mixed, peak):
    """Per kernel of one RK3 step: launches, ms, and where its algorithmic bytes are modelled
    the achieved GB/s (bytes per launch / average launch time) and its fraction of `peak`."""
    out = {}
    for k, (calls, ms) in sorted(prof.items(), key=lambda kv: -kv[1][1]):
        e = {"calls": calls, "ms": ms}
        kb = kernel_bytes(k, setup, mixed)
        if kb and calls and ms > 0:
            gbs = kb / (ms / calls / 1e3) / 1e9
            e.update(algorithmic_bytes_per_launch=kb, achieved_gbs=gbs, frac=gbs / peak)
        out[k] = e
    return out


def ncu_traffic(config: str, kname: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of a kernel from the
    committed ncu summary profiles/dram_traffic_<config>.md, or None."""
    p = os.path.join(ROOT, "profiles", f"dram_traffic_{config}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 4 and cells[0].split("<")[0] == kname and "(" not in cells[0]:
            try:
                return int(cells[3])
            except ValueError:
                return None
    return None


def step_roofline(setup, mixed, seconds_per_step, peak):
    """Whole RK3 step against the compulsory-traffic model of one substep: 608 S bytes in
    FP32-mixed, 1040 S in FP64, S = columns x planes complex values per spectral field
    (every pass reads its operands once and writes its results once)."""
    S = setup.cfg.ncol * setup.grid.nyv
    per_sub = (608 if mixed else 1040) * S
    gbs = 3 * per_sub / seconds_per_step / 1e9
    return {"model_bytes_per_substep": per_sub, "achieved_gbs": gbs, "frac": gbs / peak}


def fp32_pipe(config, kname, launch_ms, clocks):
    """FP32 operations per launch of a kernel (FADD + FMUL + 2 FFMA, counted by ncu on a
    reduced-y launch and scaled to the full grid in profiles/fp32_ops_<config>.md) over its
    CUDA-event launch time, against the FP32 peak at the measured SM clock (148 SMs x 128
    lanes x 2 flops per FMA)."""
    p = os.path.join(ROOT, "profiles", f"fp32_ops_{config}.md")
    if not os.path.exists(p) or not clocks or not clocks.get("sm_mhz"):
        return None
    ops = None
    for line in open(p):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 2 and cells[0] == kname:
            try:
                ops = float(cells[-1])
            except ValueError:
                ops = None
    if not ops:
        return None
    peak = 148 * 128 * 2 * clocks["sm_mhz"] * 1e6
    achieved = ops / (launch_ms * 1e-3)
    return {"fp32_ops_per_launch": ops, "achieved_tflops": achieved / 1e12, "peak_tflops": peak / 1e12,
            "frac": achieved / peak, "source": f"profiles/fp32_ops_{config}.md"}


# ------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region: through NVML in a
    thread every 10 ms (tens of samples even for a sub-second region), else nvidia-smi
    every 200 ms.  Read-only queries; no GPU setting is touched."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index, period_s=0.01):
        self.index = index
        self.period = period_s
        self.rows = []          # (sm_mhz, sm_max_mhz, reason bits)
        self.nv = None
        self.p = None
        self.f = None
        self.thread = None
        self.stop = False

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:  # the CUDA device's PCI bus id: NVML numbers every GPU of the node
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _loop(self):
        nv, h = self.nv
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(smax), int(rs)))
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        import threading
        try:
            self.nv = self._nvml_handle()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nv = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop = True
            self.thread.join(timeout=5)
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        if self.nv is not None:
            rows = self.rows
            source = "nvml, 10 ms"
        else:
            source = "nvidia-smi, 200 ms"
            try:
                txt = open(self.f.name).read() if self.f else ""
                if self.f:
                    os.unlink(self.f.name)
            except OSError:
                return None
            rows = []
            for r in (x.split(",") for x in txt.strip().splitlines() if x.strip()):
                try:
                    bits = sum(b for (_, b), i in zip(self.REASONS, range(4))
                               if len(r) > 5 + i and "Active" in r[5 + i] and "Not" not in r[5 + i])
                    rows.append((float(r[1]), float(r[2]), bits))
                except (ValueError, IndexError):
                    continue
        if not rows:
            return None
        reasons = sorted({n for _, _, bits in rows for n, b in self.REASONS if bits & b})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "sm_mhz_min": min(r[0] for r in rows), "samples": len(rows), "reasons": reasons,
                "source": source}


# ------------------------------------------------------------------------------------------
def dist_init(backend: str = "nccl"):
    """One process per GPU (torchrun env); replicas only, so the process group carries just
    the barrier and the max-over-ranks of the timings."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        import torch
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return ws, rank, local


def aggregate_rate(ws, units_per_rank, seconds_max):
    """Whole-job throughput of independent replicas: every rank processed units_per_rank in
    its own time; the job took the slowest rank's time."""
    return ws * units_per_rank / seconds_max


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v, device):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_steps(torch, ch, stream, nsteps, ws, device):
    barrier(ws)
    torch.cuda.synchronize(device)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    ch.step(nsteps)
    e.record(stream)
    e.synchronize()
    torch.cuda.synchronize(device)
    barrier(ws)
    return max_over_ranks(ws, s.elapsed_time(e) / 1e3, device)


def profile_step(ch):
    """One RK3 step through the stage entry points with per-kernel CUDA events."""
    lib = ch.lib
    lib.cfd_profile(ch.ctx, 1)
    for k in (1, 2, 3):
        ch.rk_substep(k)
    lib.cfd_profile(ch.ctx, 0)
    buf = C.create_string_buffer(1 << 16)
    lib.cfd_profile_read(ch.ctx, buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, calls, ms = line.split()
        out[name] = (int(calls), float(ms))
    return out


def plane_profiles(st, npts):
    """Mean and rms profiles of u, v, w from accumulated plane sums (stats.f90 quantities)."""
    n = max(st["istat"], 1) * npts
    out = {}
    for f, m, m2 in (("u", "Um", "U2m"), ("v", "Vm", "V2m"), ("w", "Wm", "W2m")):
        mean = st[m] / n
        out["mean_" + f] = mean
        out["rms_" + f] = np.sqrt(np.maximum(st[m2] / n - mean * mean, 0.0))
    return out


def profile_error(chans, setup, spinup, nsteps, nstat=20, floor=True, shared=True):
    """Mean and rms velocity profiles of the mixed and FP64 paths: the flow is spun up
    `spinup` RK3 steps from the seeded start, then the on-device statistics are accumulated
    every `nstat` steps over `nsteps` steps (the reference's cadence, nstat = min(20, nwrite),
    start.f90:372).  With `shared`, one FP64 run makes the spin-up and every path averages
    from its final state; otherwise each path spins up on its own from the seeded start.
    The time step follows the reference's rule dt = min(2.5 dtv, CFL dtc) (FOU3D.f90:178-181),
    re-chosen from the FP64 state every `nstat` steps (the reference re-chooses it every
    step); the other runs replay the FP64 run's dt sequence so all integrate with the same
    steps.  Reported: the largest difference over the planes relative to the largest FP64
    value of that profile, against the 1 % bound.  With `floor`, a second FP64 run from the
    same start rounded to FP32 measures how far two FP64 trajectories that start one rounding
    apart drift in the same window (the flow is chaotic, so the profiles of any two runs
    differ by at least this much)."""
    if nsteps <= 0:
        return None
    npts = setup.cfg.ngal1 * setup.cfg.ngal2
    prof, dts = {}, []
    out = {"spinup_steps": spinup, "steps": nsteps, "nstat": nstat, "bound": 0.01,
           "spinup": "one FP64 spin-up shared by every run" if shared else "each run spins up on its own",
           "dt_rule": "min(2.5 dtv, CFL dtc) from the FP64 state every nstat steps", "max_rel_diff": {}}
    start = setup.state()
    spun = False
    if shared and spinup > 0:
        ch = chans["fp64"]
        ch.upload_state(start)
        done = 0
        try:
            while done < spinup:
                n = min(nstat, spinup - done)
                dts.append(ch.adapt_dt())
                ch.step(n)
                done += n
            ch.cfl()   # raises on a non-finite state
        except RuntimeError as e:
            out["error"] = f"fp64 spin-up: {str(e)[:160]}"
            ch.set_dt(setup.dt)
            return out
        start = ch.download_state()
        spun = True
    runs = [("fp64", chans["fp64"], start), ("mixed", chans["mixed"], start)]
    if floor:
        rounded = {k: v.astype(np.complex64).astype(np.complex128) for k, v in start.items()}
        runs.append(("fp64_from_fp32_rounded_start", chans["fp64"], rounded))
    nspin = len(dts)
    for name, ch, st in runs:
        ch.upload_state(st)
        blk = 0 if not spun else nspin
        try:
            def advance(n):
                nonlocal blk
                if name == "fp64" and blk >= len(dts):
                    dts.append(ch.adapt_dt())
                else:
                    ch.set_dt(dts[blk])
                blk += 1
                ch.step(n)
            done = 0
            while not spun and done < spinup:
                n = min(nstat, spinup - done)
                advance(n)
                done += n
            ch.stats_configure(setup.grid.jv0 - 1, 0, 0)
            done = 0
            while done < nsteps:
                n = min(nstat, nsteps - done)
                advance(n)
                done += n
                ch.stats_accumulate()
            ch.cfl()   # raises on a non-finite state
            prof[name] = plane_profiles(ch.stats_read(), npts)
        except RuntimeError as e:
            out["error"] = f"{name}: {str(e)[:160]} (after {blk} blocks of {nstat} steps)"
            return out
        finally:
            ch.set_dt(setup.dt)
    out["dt_first_last_min_max"] = [dts[0], dts[-1], min(dts), max(dts)]

    def diffs(other):
        r = {}
        for k in ("mean_u", "rms_u", "rms_v", "rms_w"):  # mean v and w are zero up to round-off
            ref = prof["fp64"][k]
            scale = max(np.abs(ref).max(), 1e-300)
            r[k] = float(np.abs(prof[other][k] - ref).max() / scale)
        return r
    out["max_rel_diff"] = diffs("mixed")
    out["within_bound"] = all(v < out["bound"] for v in out["max_rel_diff"].values())
    if floor:
        out["chaos_floor_max_rel_diff"] = diffs("fp64_from_fp32_rounded_start")
    return out


def stats_pass_timing(torch, ch, setup, stream, reps=5):
    """The statistics pass of the reference (stats.f90, every nstat steps at kRK = 1) on the
    current state: CUDA-event ms per cfd_stats_accumulate with plane sums only and with the
    conditional sums over the cylinder lattice's tile (bottom band up to the canopy top,
    as the reference's conddown/condup), its per-kernel split, and the host-timed CFL query."""
    from cfd_b200.geometry import lattice_params
    _, _, dnx, dnz, *_ = lattice_params(setup.cfg)
    g = setup.grid
    jtop = setup.ibv.jhi[0] if setup.ibv.n else g.jv0 + g.nyv // 4   # top of the bottom canopy
    out = {"tile": [dnx, dnz], "jband": int(min(jtop, g.jv1 - 1))}
    for name, jband in (("plane_sums_ms", g.jv0 - 1), ("with_conditional_ms", out["jband"])):
        ch.stats_configure(jband, dnx, dnz)
        ch.stats_accumulate()
        ch.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            ch.stats_accumulate()
        e.record(stream)
        e.synchronize()
        out[name] = s.elapsed_time(e) / reps
    ch.lib.cfd_profile(ch.ctx, 1)
    ch.stats_accumulate()
    ch.lib.cfd_profile(ch.ctx, 0)
    buf = C.create_string_buffer(1 << 16)
    ch.lib.cfd_profile_read(ch.ctx, buf, len(buf))
    out["kernels_ms"] = {ln.split()[0]: float(ln.split()[2]) for ln in buf.value.decode().splitlines()}
    ch.stats_reset()
    t0 = time.perf_counter()
    for _ in range(reps):
        ch.cfl()
    out["cfl_query_ms"] = (time.perf_counter() - t0) / reps * 1e3
    return out


def run_ensemble(torch, device, nsteps, warmup, tuning):
    """The 16-member batched ensemble (4 x 96x97x96, 8 x 128x129x128, 4 x 192x161x192, own
    seeds and cylinder diameters) in both precisions: RK3 steps/s of the whole ensemble with
    one graph launch per step (device time on the ensemble's stream), and the same members
    stepped by their own graphs one after another (host wall time), for comparison."""
    from cfd_b200 import Ensemble
    from cfd_b200.config import ensemble_configs
    out = {"members": 16, "workload": "4 x 96x97x96 Re_tau 180, 8 x 128x129x128 Re_tau 260, "
                                      "4 x 192x161x192 Re_tau 395; D ~ U[0.03, 0.06] h, spacing 4 D"}
    for prec in ("mixed", "fp64"):
        cfgs = ensemble_configs(precision=prec)
        ens = Ensemble.from_configs(cfgs, device=device.index or 0, tuning=tuning)
        gp = sum(c.ngal1 * c.ngal2 * m.setup.grid.nyv for c, m in zip(cfgs, ens.members))
        ens.step(warmup)
        ens.synchronize()
        st = torch.cuda.ExternalStream(ens.stream(), device=device)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(st)
        ens.step(nsteps)
        e.record(st)
        e.synchronize()
        t = s.elapsed_time(e) / 1e3
        for m in ens.members:
            m.step(1)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(nsteps):
            for m in ens.members:
                m.step(1)
        for m in ens.members:
            m.synchronize()
        tsep = time.perf_counter() - t0
        out[prec] = {"ensemble_steps_per_s": nsteps / t, "member_steps_per_s": 16 * nsteps / t,
                     "grid_pt_updates_per_s": gp * nsteps / t,
                     "separate_graphs_steps_per_s": nsteps / tsep}
        ens.close(members=True)
    return out


def run_e2e(torch, ch, setup, stream, steps, warmup, ws, device):
    """The step through the reference-facing C ABI with host data: every step uploads u, v,
    w, p from pinned host memory in the reference's f(j,column) layout, advances one RK3
    step and downloads them again into the same host buffers.  Timed as the host issues it
    (one synchronisation after the last step: the library orders each field's upload after
    its previous download, and the next step's uploads run while this step's downloads are
    in flight), and again with a synchronisation after every step."""
    host = {}
    nbytes = 0
    for k in ("u1", "u2", "u3", "p"):
        a = torch.from_numpy(np.ascontiguousarray(setup.state()[k]).view(np.float64).copy()).pin_memory()
        host[k] = a
        nbytes += a.numel() * 8
    lib = ch.lib
    fid = {"u1": 0, "u2": 1, "u3": 2, "p": 3}

    def e2e_step(sync):
        for k in host:
            lib.cfd_upload_field(ch.ctx, fid[k], C.cast(host[k].data_ptr(), C.POINTER(C.c_double)), 0)
        ch.step(1)
        for k in host:
            lib.cfd_download_field(ch.ctx, fid[k], C.cast(host[k].data_ptr(), C.POINTER(C.c_double)), 0)
        if sync:
            ch.synchronize()

    n = max(3, min(steps, 10))
    rates = {}
    for sync in (False, True):
        for _ in range(warmup):
            e2e_step(sync)
        ch.synchronize()
        barrier(ws)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(n):
            e2e_step(sync)
        e.record(stream)   # the context stream waits for every download's copy
        e.synchronize()
        barrier(ws)
        t = max_over_ranks(ws, s.elapsed_time(e) / 1e3, device)
        rates[sync] = aggregate_rate(ws, n, t)
    return {"value": rates[False], "unit": "RK3 steps/s", "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "steps": n, "synchronised_every_step": rates[True],
            "path": "cfd_upload_field x4 (pinned host, reference layout) + cfd_step + cfd_download_field x4, "
                    "one synchronisation after the last step (synchronised_every_step: after each)"}


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cpu_baseline(setup, budget_s=30.0):
    """FP64 oracle (C++ port of the reference step, all host threads) on a bounded sample."""
    from oracle import oracle as O
    O.build()
    nthreads = os.cpu_count() or 1
    O.set_threads(nthreads)
    o = O.OracleChannel(setup)
    o.upload_state()
    t0 = time.perf_counter()
    o.rk_substep(1)
    t_sub = time.perf_counter() - t0
    if 2 * t_sub < budget_s:
        t0 = time.perf_counter()
        o.rk_substep(2)
        o.rk_substep(3)
        t_step = t_sub + (time.perf_counter() - t0)
        sample = f"one full RK3 step of the {setup.cfg.name} grid (3 substeps)"
    else:
        t_step = 3.0 * t_sub
        sample = f"one RK3 substep (kRK=1) of the {setup.cfg.name} grid, x3 for a step"
    o.close()
    return {"value": 1.0 / t_step, "unit": "RK3 steps/s", "cores": nthreads, "kind": "port",
            "sample": sample, "seconds": t_step}


# ------------------------------------------------------------------------------------------
def workload_config(setup, ws):
    """The `config` object of both arms' JSON lines."""
    cfg = setup.cfg
    return {"workload": f"{cfg.name}: Re_tau {cfg.re_tau:g}, {cfg.ngal1}x{cfg.ny}x{cfg.ngal2} "
                        f"(+{2 * setup.grid.dny} canopy planes), cylinders H {cfg.posth} D {cfg.cyl_diameter} "
                        f"s {cfg.cyl_spacing}",
            "ny_tot": setup.grid.nyv, "ib_points_u": setup.ibu.n, "ib_points_v": setup.ibv.n,
            "dt": setup.dt, "parallelism": f"replicas x{ws}",
            "l2": "state and work buffers are GBs, far above the 126 MB L2 (no flush)"}


def run_reference(args, setup, ws, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    nth = os.cpu_count() or 1
    O.set_threads(nth)
    o = O.OracleChannel(setup)
    o.upload_state()
    budget = 120.0
    # warm-up: W full steps, stopped after 30 s (the oracle has no caches to warm beyond
    # first touch; a re550 step takes seconds on the host cores)
    warm = 0
    tw = time.perf_counter()
    while warm < args.warmup:
        for k in (1, 2, 3):
            o.rk_substep(k)
        warm += 1
        if time.perf_counter() - tw > 30.0:
            break
    done = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for k in (1, 2, 3):
            o.rk_substep(k)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = done / el
    line = {"metric": METRIC, "value": v, "unit": "RK3 steps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": done, "warmup": warm, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(setup, ws),
            "grid_pt_updates_per_s": v * setup.grid_points,
            "cpu_baseline": {"value": v, "unit": "RK3 steps/s", "cores": nth, "kind": "port",
                             "sample": f"{done} full RK3 steps of the {setup.cfg.name} grid "
                                       f"(capped at {budget:.0f} s of timed work)"},
            "e2e": {"value": v, "unit": "RK3 steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="re550")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--error-steps", type=int, default=10)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 16-member ensemble measurement")
    ap.add_argument("--no-autotune", action="store_true", help="library default launch shapes")
    ap.add_argument("--profile-steps", type=int, default=2000,
                    help="averaging steps of the mean/rms profile comparison of mixed vs FP64 (0: skip)")
    ap.add_argument("--spinup-steps", type=int, default=2000,
                    help="spin-up steps before the profile averaging window")
    ap.add_argument("--independent-spinup", action="store_true",
                    help="also compare the profiles with each precision spun up on its own")
    ap.add_argument("--sustained-steps", type=int, default=200,
                    help="steps of the longer second timing window per precision (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    from cfd_b200.channel import build_channel
    from cfd_b200.config import preset
    cfg = preset(args.config)
    ws, rank, local = dist_init() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                              int(os.environ.get("RANK", "0")), 0)
    setup = build_channel(cfg.with_(seed=cfg.seed + rank))
    if args.impl == "reference":
        run_reference(args, setup, ws, rank)
        return

    import torch
    from cfd_b200.channel import Channel
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device)
    results = {}
    chans = {}
    tuning = {}
    for prec in ("mixed", "fp64"):
        ch = Channel(setup, device=local, precision=prec, tuning=None if args.no_autotune else "auto")
        tuning[prec] = ch.tuning()
        ch.set_stream(stream.cuda_stream)
        ch.upload_state()
        ch.step(args.warmup)
        n0 = ch.launch_count()
        with ClockSampler(local) as cs:
            t = time_steps(torch, ch, stream, args.steps, ws, device)
        results[prec] = {"seconds": t, "steps_per_s": aggregate_rate(ws, args.steps, t), "clocks": cs.summary(),
                         "launches": ch.launch_count() - n0}
        chans[prec] = ch

    # error of the mixed path against the FP64 path after the same number of steps
    err = {}
    states = {}
    for prec, ch in chans.items():
        ch.upload_state()
        ch.step(args.error_steps)
        states[prec] = ch.download_state()
    for k in ("u1", "u2", "u3", "p"):
        err[k] = rel_err(states["mixed"][k], states["fp64"][k])
    fp64_div = chans["fp64"].divergence_max()
    prof_err = profile_error(chans, setup, args.spinup_steps, args.profile_steps)
    prof_err_indep = profile_error(chans, setup, args.spinup_steps, args.profile_steps, shared=False) \
        if args.independent_spinup else None
    ens = run_ensemble(torch, device, args.steps, args.warmup, None if args.no_autotune else "auto") \
        if (ws == 1 and not args.no_ensemble) else None

    # per-kernel timing (CUDA events on the launching stream) for the roofline
    hbm, peak_kind = peaks()
    prof = profile_step(chans["mixed"])
    top = max(prof.items(), key=lambda kv: kv[1][1])
    tot = sum(v[1] for v in prof.values())
    kname, (kcalls, kms) = top
    kb = kernel_bytes(kname, setup, True)
    per_launch_s = kms / kcalls / 1e3
    achieved = kb / per_launch_s / 1e9 if kb else None
    prof64 = profile_step(chans["fp64"])
    stats_t = stats_pass_timing(torch, chans["mixed"], setup, stream) if ws == 1 else None

    # end-to-end through the C ABI with pinned host buffers: H2D state, step, D2H state,
    # for both precisions (FP64 is the reference's arithmetic)
    e2e = {prec: run_e2e(torch, chans[prec], setup, stream, args.steps, args.warmup, ws, device)
           for prec in ("mixed", "fp64")}

    # the step seen over a longer window (clock record with many samples); the timed region
    # above stays exactly --steps steps
    sustained = {}
    if args.sustained_steps > 0:
        for prec, ch in chans.items():
            ch.upload_state()
            ch.step(args.warmup)
            with ClockSampler(local) as cs2:
                t2 = time_steps(torch, ch, stream, args.sustained_steps, ws, device)
            sustained[prec] = {"steps": args.sustained_steps, "steps_per_s": aggregate_rate(ws, args.sustained_steps, t2),
                               "clocks": cs2.summary()}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(setup)

    gp = setup.grid_points
    mixed, fp64 = results["mixed"], results["fp64"]
    line = {
        "metric": METRIC,
        "value": mixed["steps_per_s"],
        "unit": "RK3 steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * mixed["seconds"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32-mixed (FP32 transforms/products, FP64 solves/state)",
        "data": "synthetic (seeded perturbed Poiseuille, cylinder lattice)",
        "config": workload_config(setup, ws),
        "grid_pt_updates_per_s": mixed["steps_per_s"] * gp,
        "fp64": {"steps_per_s": fp64["steps_per_s"], "grid_pt_updates_per_s": fp64["steps_per_s"] * gp,
                 "ms_per_step": 1e3 * fp64["seconds"] / args.steps, "clocks": fp64["clocks"],
                 "max_divergence": fp64_div, "e2e": e2e["fp64"],
                 "step_roofline": step_roofline(setup, False, fp64["seconds"] / args.steps, hbm)},
        "step_roofline": step_roofline(setup, True, mixed["seconds"] / args.steps, hbm),
        "sustained": sustained or None,
        "mixed_over_fp64": mixed["steps_per_s"] / fp64["steps_per_s"],
        "error_mixed_vs_fp64": {"steps": args.error_steps, "rel_l2": err},
        "profile_error_mixed_vs_fp64": prof_err,
        "profile_error_independent_spinup": prof_err_indep,
        "statistics_pass": stats_t,
        "ensemble": dict(ens, grid_pt_rate_vs_single={
            prec: ens[prec]["grid_pt_updates_per_s"] / (results[prec]["steps_per_s"] * gp)
            for prec in ("mixed", "fp64")}) if ens else None,
        "tuning": {"source": "defaults" if args.no_autotune else "cfd_b200.autotune (coordinate search, cached)",
                   **tuning},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                     "traffic": ncu_traffic(args.config, kname), "traffic_source":
                         f"profiles/dram_traffic_{args.config}.md (ncu, bytes per launch)",
                     "algorithmic_bytes_per_launch": kb,
                     "avg_launch_ms": kms / kcalls, "share_of_step": kms / tot,
                     "fp32_pipe": fp32_pipe(args.config, kname, kms / kcalls, mixed["clocks"])},
        "kernels_mixed": kernel_table(prof, setup, True, hbm),
        "kernels_fp64": kernel_table(prof64, setup, False, hbm),
        "cpu_baseline": cpu,
        "e2e": e2e["mixed"],
        "gpu_launches": mixed["launches"],
        "launches_per_step": mixed["launches"] // max(args.steps, 1),
        "clocks": mixed["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for ch in chans.values():
        ch.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
