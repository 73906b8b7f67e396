#!/usr/bin/env python
"""Acoustic-substep throughput on B200: AcousticDynamics (fv3core's dyn_core)
on a C384 L79 cubed sphere, all six tiles on one GPU, in the mixed-precision
build (FP32 fields and arithmetic, FP64 column solves) with the plain FP64
build measured beside it, and the mixed build's error against FP64.

One step = one AcousticDynamics call = n_split (6) acoustic substeps over
the whole cube, on a Jablonowski-Williamson baroclinic-wave state with seeded
noise (synthetic data).  ``value`` is cell-levels advanced per second per
substep (6 * 384^2 * 79 cell-levels x n_split per step), device-timed with
CUDA events, inputs resident in HBM (every 3-D field is 0.59 GB, far larger
than the 126 MB L2, so no flush is needed); every step restarts from the
initial state (a device-to-device copy outside the step's events).  ``e2e``
times the same call through the package's public API with the state copied
in from pinned host memory and the results copied back every step, streamed
(two device states, the copies of one step overlapping the call of another;
``e2e.sequential`` is the one-stream loop).  ``roofline.traffic`` is the DRAM
traffic of a call as measured by ncu.

``--workload ensemble`` times the mixed-resolution ensemble (16 x C48 L79,
8 x C96 L79, 4 x C192 L63), one CUDA graph per ensemble step against eager
launches.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
N > 1 runs under torch.distributed.run: every rank advances its own replica
(the path has no data exchange between GPUs), value = all ranks' cell-levels
/ max-over-ranks time.

``--impl reference`` times the reference algorithm's CPU restatement (the
oracle) on the host cores, one worker process per core, each step a bounded
sample (one C24 L79 substep per worker).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "C384 L79 acoustic-substep cell-levels/s"
UNIT = "cell-levels/s"
# The committed ncu summary of one call's DRAM traffic (every launch, one-pass
# metrics dram__bytes_read.sum + dram__bytes_write.sum) of the current code.
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "acoustics_c128_l79_dram_traffic.md")


def dram_bytes_per_cell_level():
    """{"f32": B, "f64": B}: DRAM bytes per cell-level per substep, read from
    the profile's line ``bytes per cell-level per substep: f32 X, f64 Y``
    (None when the file or the line is missing)."""
    import re

    try:
        text = open(TRAFFIC_PROFILE).read()
    except OSError:
        return None
    m = re.search(r"bytes per cell-level per substep: f32 (\d+), f64 (\d+)", text)
    return {"f32": float(m.group(1)), "f64": float(m.group(2))} if m else None


def _env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(values, dist=None, device="cuda"):
    """Element-wise maximum of per-rank timings.  Every rank calls it at the
    same point with the same number of values (one all-reduce)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def _measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- workload
def build_problem(n, npz, n_split, seed, device="cuda", precision="f64", grid=None, state0=None):
    """GridData, AcousticDynamics and a device state for one build.  grid and
    state0 (a host baroclinic state) may be passed in to share them between
    the two builds."""
    import types

    import numpy as np
    import torch

    from fv3core_b200 import _lib
    from fv3core_b200.config import baroclinic_acoustic_config
    from fv3core_b200.grid import CubedSphereGrid
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.halo import DeviceCubedSphereCommunicator
    from fv3core_b200.initial_state import baroclinic_state
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.dyn_core import AcousticDynamics
    from fv3core_b200.storage import to_device

    grid = CubedSphereGrid(n, 3) if grid is None else grid
    st = baroclinic_state(grid, npz, seed=seed) if state0 is None else state0
    gd = GridData(grid, npz, device=device, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    cfg = baroclinic_acoustic_config(n_split=n_split)
    state = types.SimpleNamespace()
    for name in _lib.DYCORE_FIELDS:
        if name in st:
            a = st[name]
        else:
            a = np.zeros(st["phis"].shape if name == "wsd" else st["delp"].shape)
        setattr(state, name, to_device(a, dtype=dtype))
    ad = AcousticDynamics(DeviceCubedSphereCommunicator(gd.grid_indexing), sf, gd, gd, 0, False, False, cfg,
                          st["ak"], st["bk"], st["pfull"], state.phis)
    state.mdt = 225.0
    state.n_map = 1
    state.akap = 287.05 / 1004.6
    state.ptop = st["ptop"]
    state.ks = st["ks"]
    torch.cuda.synchronize()
    return gd, ad, state


# fields AcousticDynamics reads (copied in for the end-to-end timing) and writes (copied out)
E2E_IN = ("u", "v", "w", "delz", "delp", "pt", "pe", "pk", "phis", "wsd", "omga", "ua", "va", "uc", "vc", "pkz",
          "peln", "q_con", "diss_estd", "cappa")
E2E_OUT = ("u", "v", "w", "delz", "delp", "pt", "pe", "pk", "wsd", "omga", "ua", "va", "uc", "vc", "mfxd", "mfyd",
           "cxd", "cyd", "pkz", "peln", "q_con", "diss_estd")


def _compute(t, n, npz):
    h = 3
    return t[:, :npz, h:h + n, h:h + n]


def _max_rel(a, b, n, npz):
    import torch

    a, b = _compute(a, n, npz).double(), _compute(b, n, npz).double()
    return float((torch.abs(a - b) / torch.clamp(torch.abs(b), min=1e-30)).max())


def _rel_stats(a, b, n, npz):
    """(max, 99.9th percentile, count above 1e-4) of the relative difference
    over the compute domain."""
    import torch

    a, b = _compute(a, n, npz).double(), _compute(b, n, npz).double()
    r = (torch.abs(a - b) / torch.clamp(torch.abs(b), min=1e-30)).flatten()
    q = torch.kthvalue(r.cpu(), max(1, int(0.999 * r.numel()))).values.item()
    return {"max": float(r.max()), "p999": q, "above_1e-4": int((r > 1e-4).sum())}


def _rms_rel(a, b, n, npz):
    """RMS of the difference over RMS of the reference, compute domain."""
    a, b = _compute(a, n, npz).double(), _compute(b, n, npz).double()
    return float(((a - b) ** 2).mean().sqrt() / (b ** 2).mean().sqrt())


def run_cuda(args):
    import torch

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from fv3core_b200 import _lib
    from fv3core_b200.grid import CubedSphereGrid
    from fv3core_b200.initial_state import baroclinic_state

    n, npz, n_split = args.n, args.npz, args.n_split
    stream = torch.cuda.current_stream()
    cells = 6 * n * n * npz
    grid = CubedSphereGrid(n, 3)
    state0 = baroclinic_state(grid, npz, seed=1234 + rank)
    precisions = {"both": ["f32", "f64"], "mixed": ["f32"], "f64": ["f64"]}[args.precision]
    problems = {p: build_problem(n, npz, n_split, 1234 + rank, precision=p, grid=grid, state0=state0)
                for p in precisions}

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # Every step starts from the initial state.  Repeated acoustic calls
    # without the vertical remapping that follows each one in a full
    # dynamics step let the Lagrangian layers deform, and at C384 the state
    # leaves the physical range after a few calls; restarting keeps every
    # timed call on the same, valid input.  The device-to-device reset runs
    # before each call, outside that call's timing events.
    initial = {p: {k: getattr(problems[p][2], k).clone() for k in _lib.DYCORE_FIELDS} for p in precisions}

    def reset(prec):
        state = problems[prec][2]
        for k, t in initial[prec].items():
            getattr(state, k).copy_(t)

    # Error of the mixed build against FP64 after one call (one dynamics
    # step's acoustic part) from the same state.  The driver's temporaries
    # carry over between calls, as the reference's instance storages do
    # (heat_source, which d_sw accumulates into, among them), so every
    # compared run is the first call of its own AcousticDynamics.  Beside
    # it: FP64 started from the state rounded to FP32 (the mixed build's
    # input), the mixed build against that run (both start from identical
    # numbers, only the arithmetic differs), FP64's response to input
    # perturbations of relative size eps, and what the carry-over alone does
    # (a second FP64 call from the same state).
    mixed_error = None
    if len(precisions) == 2 and not args.no_error_analysis:
        fields = ("delp", "pt", "delz", "q_con")
        s32, s64 = problems["f32"][2], problems["f64"][2]
        problems["f32"][1](s32)
        problems["f64"][1](s64)
        barrier()
        ref = {k: getattr(s64, k).clone() for k in fields + ("u", "v", "w")}
        mixed = {k: _max_rel(getattr(s32, k), ref[k], n, npz) for k in fields}
        mixed_rms = {k: _rms_rel(getattr(s32, k), ref[k], n, npz) for k in fields + ("u", "v", "w")}
        reset("f64")
        problems["f64"][1](s64)
        barrier()
        carry = {k: _max_rel(getattr(s64, k), ref[k], n, npz) for k in fields}

        def first_call_f64(make_input):
            """One FP64 call on a fresh AcousticDynamics from make_input(k, t)
            applied to every initial field; returns the fresh state."""
            gd2, ad2, st2 = build_problem(n, npz, n_split, 1234 + rank, precision="f64", grid=grid, state0=state0)
            for k, t in initial["f64"].items():
                getattr(st2, k).copy_(make_input(k, t))
            ad2(st2)
            barrier()
            return gd2, st2

        gd2, st2 = first_call_f64(lambda k, t: t.float().double())
        floor = {k: _max_rel(getattr(st2, k), ref[k], n, npz) for k in fields}
        arith = {k: _max_rel(getattr(s32, k), getattr(st2, k), n, npz) for k in fields}
        gd2.close()
        del gd2, st2
        gen = torch.Generator(device="cuda").manual_seed(99)
        response = {}
        for eps in (6e-8, 6e-10, 6e-12):
            def perturbed(k, t, eps=eps):
                r = torch.rand(t.shape, device=t.device, dtype=t.dtype, generator=gen) * 2.0 - 1.0
                return t * (1.0 + eps * r)

            gd2, st2 = first_call_f64(perturbed)
            response[f"{eps:.0e}"] = {k: _rel_stats(getattr(st2, k), ref[k], n, npz) for k in ("delp", "pt")}
            gd2.close()
            del gd2, st2
        del ref
        mixed_error = {
            "mixed_vs_fp64": mixed, "mixed_vs_fp64_rms": mixed_rms, "fp64_from_fp32_rounded_input_vs_fp64": floor,
            "mixed_vs_fp64_from_same_input": arith,
            "fp64_second_call_vs_first": carry,
            "fp64_response_to_input_perturbation": {
                "per_eps": response,
                "stats": "max relative change, its 99.9th percentile, and the number of compute points above 1e-4",
            },
            "after": "one AcousticDynamics call (n_split acoustic substeps) from the same state, each compared run "
                     "the first call of its own AcousticDynamics; max relative error over the compute domain "
                     "(rms: RMS difference over RMS of the FP64 field)",
        }

    results = {}
    for prec in precisions:
        gd, ad, state = problems[prec]
        for _ in range(args.warmup):
            reset(prec)
            ad(state)
        barrier()
        launches0 = _lib.launch_count(prec)
        events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            barrier()
            torch.cuda.nvtx.range_push("timed" if prec == precisions[0] else "timed_" + prec)
            for start, stop in events:
                reset(prec)
                start.record(stream)
                ad(state)
                stop.record(stream)
            torch.cuda.nvtx.range_pop()
            barrier()
        launches = _lib.launch_count(prec) - launches0
        ms = sum(a.elapsed_time(b) for a, b in events) / args.steps
        finite = all(bool(torch.isfinite(_compute(getattr(state, k), n, npz)).all().item())
                     for k in ("u", "v", "w", "delp", "pt", "delz"))
        results[prec] = {"ms": ms, "launches": launches, "clocks": clk.summary(), "finite": finite}

    # end to end through the public API for the headline build: the state
    # copied in from pinned host memory and the results copied back, every step
    head = precisions[0]
    gd, ad, state = problems[head]
    host = {k: torch.empty(getattr(state, k).shape, dtype=getattr(state, k).dtype, pin_memory=True)
            for k in set(E2E_IN) | set(E2E_OUT)}
    for k, hb in host.items():
        hb.copy_(initial[head][k] if k in initial[head] else getattr(state, k))
    torch.cuda.synchronize()
    h2d = sum(host[k].numel() * host[k].element_size() for k in E2E_IN)
    d2h = sum(host[k].numel() * host[k].element_size() for k in E2E_OUT)
    e2e_steps = max(1, min(args.steps, args.e2e_steps))

    def e2e_step():
        for k in E2E_IN:
            getattr(state, k).copy_(host[k], non_blocking=True)
        ad(state)
        for k in E2E_OUT:
            host[k].copy_(getattr(state, k), non_blocking=True)

    # one stream, copy in -> call -> copy out, step after step
    e2e_step()  # untimed warm-up round trip
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e2e_seq_ms = e0.elapsed_time(e1) / e2e_steps

    # streamed: two device states, the copies of one state overlapped with
    # the call on the other (fv3core_b200.pipeline.StreamedAcoustics); every
    # step still copies its inputs in and its results out
    import types

    from fv3core_b200.pipeline import StreamedAcoustics

    state2 = types.SimpleNamespace(**vars(state))
    for k in _lib.DYCORE_FIELDS:
        setattr(state2, k, getattr(state, k).clone())
    streamed = StreamedAcoustics(ad, [state, state2], E2E_IN, E2E_OUT)
    host_out = {k: host[k] for k in E2E_OUT}
    streamed.run([(host, host_out)] * 2)  # untimed warm-up
    streamed.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(streamed.h2d)
    streamed.run([(host, host_out)] * e2e_steps)
    e1.record(streamed.d2h)
    streamed.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    del state2, streamed

    # max over ranks
    vals = max_over_ranks([results[p]["ms"] for p in precisions] + [e2e_seq_ms, e2e_ms], dist)
    for q, p in enumerate(precisions):
        results[p]["ms"] = vals[q]
    e2e_seq_ms, e2e_ms = vals[-2], vals[-1]
    peak, peak_kind = _measured_peak()

    per_cell = dram_bytes_per_cell_level()

    def roof(prec):
        width = 4 if prec == "f32" else 8
        sec = results[prec]["ms"] * 1e-3
        achieved = 34 * width * cells * n_split / sec / 1e9
        r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
             "traffic": None, "peak_source": peak_kind,
             "scope": f"whole AcousticDynamics call: {34 * width} B compulsory traffic per cell-level per "
                      "substep (34 field transfers at the stored width)"}
        if per_cell is not None:
            traffic = per_cell[prec] * cells * n_split
            r.update(traffic=traffic, dram_gbs_at_traffic=traffic / sec / 1e9,
                     traffic_note=f"DRAM bytes read + written per call: {per_cell[prec]:.0f} B per cell-level per "
                                  "substep (ncu, every launch of one call at C128 L79, the current code) times "
                                  "this call's cell-levels and substeps")
        return r

    ms = results[head]["ms"]
    value = world * cells * n_split / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "mixed: f32 fields and arithmetic, f64 column solves" if head == "f32" else "f64",
        "data": "synthetic (seeded baroclinic-wave state)",
        "config": {
            "workload": f"AcousticDynamics C{n} L{npz}, n_split={n_split}, 6 tiles on one GPU, nonhydrostatic, "
                        + ("mixed precision" if head == "f32" else "FP64"),
            "n": n, "npz": npz, "n_split": n_split, "dt_atmos": 225.0, "cell_levels": cells,
            "l2": "inputs larger than L2 (each 3-D field 0.29-0.59 GB at C384 L79); no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "clocks": results[head]["clocks"],
        "e2e": {"value": world * cells * n_split / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": e2e_steps,
                "mode": "streamed: two device states, copy-in / call / copy-out on three CUDA streams, the "
                        "copies of one step overlapping the call of another",
                "sequential": {"value": world * cells * n_split / (e2e_seq_ms * 1e-3), "ms_per_step": e2e_seq_ms}},
        "gpu_launches": results[head]["launches"],
        "roofline": roof(head),
        "finite": results[head]["finite"],
    }
    if "f64" in results and head != "f64":
        r = results["f64"]
        line["fp64"] = {"value": world * cells * n_split / (r["ms"] * 1e-3), "ms_per_step": r["ms"],
                        "roofline": roof("f64"), "gpu_launches": r["launches"], "clocks": r["clocks"],
                        "finite": r["finite"]}
        line["mixed_speedup_vs_fp64"] = r["ms"] / ms
    if mixed_error is not None:
        line["mixed_error_vs_fp64"] = mixed_error
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(1, args.cpu_n, args.cpu_npz)
    for gd, _, _ in problems.values():
        gd.close()
    del problems, initial, state, host, ad
    torch.cuda.empty_cache()
    if world == 1 and args.step_n > 0:
        line["step_dynamics"] = run_step_section(args, state0, grid, local)
    del state0
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ----------------------------------------------------------------------------- full dynamics step
STEP_FIELDS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp",
               "delz", "peln", "u", "v", "w", "ua", "va", "uc", "vc", "q_con", "pe", "pk", "pkz", "ps", "omga",
               "mfxd", "mfyd", "cxd", "cyd", "diss_estd")
# compulsory field transfers per cell-level of one step (k_split 1): the
# acoustic call's 34 per substep, the tracer advection's 8 tracers read and
# written plus its 5 shared fluxes (one sub-cycle), the remapping's 21
# fields read and written, the saturation adjustment's 13 read and 11
# written, the preamble's 15, post_remap's 6 and wrapup's 23
STEP_TRANSFERS_NON_ACOUSTIC = 8 * 2 + 5 + 21 * 2 + 13 + 11 + 15 + 6 + 23


def step_problem(n, npz, n_split, precision, st0, grid):
    """GridData, DynamicalCore (baroclinic namelist) and device state for a
    step_state ``st0``."""
    import torch

    from fv3core_b200.config import baroclinic_config
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.fv_dynamics import DynamicalCore
    from fv3core_b200.storage import to_device

    gd = GridData(grid, npz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    phis = to_device(st0["phis"], dtype=dtype)
    core = DynamicalCore(None, gd, sf, gd, baroclinic_config(n, npz, n_split), st0["ak"], st0["bk"], phis)
    state = {k: to_device(st0[k], dtype=dtype) for k in STEP_FIELDS}
    state["phis"] = phis
    torch.cuda.synchronize()
    return gd, core, state


def _oracle_step_worker(n, npz, n_split, q):
    """One bounded sample of the step on the host: one oracle step_dynamics
    at C{n} L{npz}; returns (cell-levels, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import cases
    import oracle_runs

    case = cases.step_case(n, npz, 5, n_split, sat_adj=True)
    t0 = time.perf_counter()
    oracle_runs.run_step(case, n, npz)
    q.put((6 * n * n * npz, time.perf_counter() - t0))


def step_cpu_sample(n, npz, n_split):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_oracle_step_worker, args=(n, npz, n_split, q))
    p.start()
    cells, sec = q.get()
    p.join()
    return {"value": cells / sec, "unit": "cell-levels/s (one dynamics step)", "cores": 1, "kind": "port",
            "sample": f"one step_dynamics (n_split {n_split}) of C{n} L{npz}, numpy FP64 oracle on one core: "
                      f"{sec:.1f} s"}


def run_step_section(args, state0, grid384, local):
    """The whole dynamics step: the plain FP64
    (and mixed) DynamicalCore.step_dynamics at C``step_n`` L79 — time per
    step, roofline, the oracle step on the host — and the mixed build's
    error against FP64 after 1 and ``error_steps`` steps at C384 L79."""
    import torch

    from fv3core_b200 import _lib
    from fv3core_b200.grid import CubedSphereGrid
    from fv3core_b200.initial_state import step_state

    n, npz, n_split = args.step_n, args.npz, args.n_split
    stream = torch.cuda.current_stream()
    cells = 6 * n * n * npz
    grid = CubedSphereGrid(n, 3)
    st0 = step_state(grid, npz, seed=4321)
    out = {"metric": f"C{n} L{npz} step_dynamics cell-levels/s", "unit": "cell-levels/s",
           "config": {"workload": f"DynamicalCore.step_dynamics C{n} L{npz}, k_split 1, n_split {n_split}, "
                                  "dt_atmos 225 s, nonhydrostatic, d_ext 0, nord 3, hord_tr 8, kord 9, 8 advected "
                                  "tracers + qcld, fast saturation adjustment (do_sat_adj)",
                      "n": n, "npz": npz, "n_split": n_split, "cell_levels": cells,
                      "reset": "every step restarts from the initial state (device copy outside the events)"}}
    peak, peak_kind = _measured_peak()
    for prec in ("f64", "f32"):
        gd, core, state = step_problem(n, npz, n_split, prec, st0, grid)
        initial = {k: v.clone() for k, v in state.items()}

        def step():
            core.step_dynamics(state, False, False, 225.0, st0["ptop"], n_split, st0["ks"])

        def reset():
            for k, v in initial.items():
                state[k].copy_(v)

        for _ in range(args.warmup):
            reset()
            step()
        torch.cuda.synchronize()
        launches0 = _lib.launch_count(prec)
        events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_push("step_timed_" + prec)
            for a, b in events:
                reset()
                a.record(stream)
                step()
                b.record(stream)
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in events) / args.steps
        launches = (_lib.launch_count(prec) - launches0) // args.steps
        width = 8 if prec == "f64" else 4
        transfers = 34 * n_split + STEP_TRANSFERS_NON_ACOUSTIC
        achieved = transfers * width * cells / (ms * 1e-3) / 1e9
        h = 3
        finite = all(bool(torch.isfinite(state[k][:, :npz, h:h + n, h:h + n]).all()) for k in
                     ("u", "v", "w", "delp", "pt", "delz", "qvapor"))
        r = {"value": cells / (ms * 1e-3), "ms_per_step": ms,
             "cell_level_substeps_per_s": cells * n_split / (ms * 1e-3), "gpu_launches_per_step": launches,
             "clocks": clk.summary(), "finite": finite,
             "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                          "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                          "scope": f"whole step: {transfers} compulsory field transfers of {width} B per "
                                   f"cell-level (34 per acoustic substep, {STEP_TRANSFERS_NON_ACOUSTIC} for the "
                                   "tracer advection, remapping with the saturation adjustment, preamble and "
                                   "epilogue)"}}
        out["fp64" if prec == "f64" else "mixed"] = r
        del initial, state, core
        gd.close()
    out["value"] = out["fp64"]["value"]
    out["mixed_speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = step_cpu_sample(12, npz, n_split)

    # mixed against FP64 after 1 and error_steps dynamics steps at C384 L79
    if args.error_steps > 0 and state0 is not None:
        ne = grid384.n
        st384 = step_state(grid384, npz, base=state0)
        snaps = {}
        keep = ("delp", "pt", "delz", "u", "v", "w", "qvapor")
        h = 3
        for prec in ("f64", "f32"):
            gd, core, state = step_problem(ne, npz, n_split, prec, st384, grid384)
            for s in range(1, args.error_steps + 1):
                core.step_dynamics(state, False, False, 225.0, st384["ptop"], n_split, st384["ks"])
                if s in (1, args.error_steps):
                    snaps[(prec, s)] = {k: state[k][:, :npz, h:h + ne, h:h + ne].double().cpu() for k in keep}
            del state, core
            gd.close()
        del st384
        err = {}
        for s in sorted({1, args.error_steps}):
            a64, a32 = snaps[("f64", s)], snaps[("f32", s)]
            entry = {}
            for k in keep:
                d = (a32[k] - a64[k]).abs()
                scale = a64[k].abs()
                with torch.no_grad():
                    rel = d / scale.clamp_min(1e-6 * float(scale.max()))
                entry[k] = {"max_rel": float(rel.max()), "max_abs_over_max": float(d.max() / scale.max()),
                            "rms_rel": float(torch.sqrt((d * d).mean() / (a64[k] * a64[k]).mean())),
                            "finite": bool(torch.isfinite(a32[k]).all() and torch.isfinite(a64[k]).all())}
            err[f"after_{s}_steps"] = entry
        out["mixed_error_vs_fp64"] = {
            "grid": f"C{ne} L{npz}", "n_split": n_split, "per_field": err,
            "metric": "max over the compute domain of |mixed - fp64| / max(|fp64|, 1e-6 max|fp64|) (max_rel; "
                      "points near zero dominate it for the winds and the tracers), of |mixed - fp64| / max|fp64| "
                      "(max_abs_over_max), and the RMS difference over the RMS of the FP64 field; both runs from "
                      "the same baroclinic-wave state",
        }
    return out


# ----------------------------------------------------------------------------- CPU oracle
def _oracle_worker(n, npz, seed, q):
    """One bounded sample: one acoustic substep of the oracle on a C{n} L{npz}
    case; returns (cell-level-substeps, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np

    import cases
    from oracle.dyn_core import AcousticDynamics

    case = cases.acoustics_case(n, npz, seed, n_split=1)
    g = cases.grid_for(n)
    cfg = {**cases.ACOUSTIC_CONFIG, **cases.RIEMANN_CONFIG, "n_split": 1, "dsw": cases.DSW_CONFIG}
    metrics = [cases.metric_namespace(n, t) for t in range(6)]
    ad = AcousticDynamics(g, metrics, cfg, case["ak"], case["bk"], case["pfull"], case["phis"], npz)
    st = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    t0 = time.perf_counter()
    with np.errstate(all="ignore"):
        ad(st)
    q.put((6 * n * n * npz, time.perf_counter() - t0))


def cpu_sample(workers, n, npz, repeats=1):
    """Oracle throughput (cell-levels/s per substep) with `workers` processes."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    total_cells, total_time = 0, 0.0
    for r in range(repeats):
        q = ctx.Queue()
        procs = [ctx.Process(target=_oracle_worker, args=(n, npz, 7 + w + 100 * r, q)) for w in range(workers)]
        for p in procs:
            p.start()
        res = [q.get() for _ in procs]
        for p in procs:
            p.join()
        total_cells += sum(c for c, _ in res)
        total_time += max(s for _, s in res)
    value = total_cells / total_time
    return {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
            "sample": f"{repeats} x {workers} worker(s), each one acoustic substep of C{n} L{npz} (numpy FP64 oracle)"}


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    try:
        import psutil

        mem_workers = int(psutil.virtual_memory().available // (3 << 30))
    except Exception:
        mem_workers = os.cpu_count() or 1
    workers = max(1, min(os.cpu_count() or 1, mem_workers, args.ref_max_workers))
    for _ in range(args.warmup):
        cpu_sample(workers, args.ref_n, args.npz)
    t0 = time.perf_counter()
    samples = [cpu_sample(workers, args.ref_n, args.npz) for _ in range(args.steps)]
    wall = time.perf_counter() - t0
    value = statistics.median(s["value"] for s in samples)
    cells_step = 6 * args.ref_n * args.ref_n * args.npz * workers
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * cells_step / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded baroclinic-wave state)",
        "impl": "reference",
        "config": {"workload": f"AcousticDynamics C{args.n} L{args.npz} (sampled at C{args.ref_n} L{args.npz}, "
                               f"one substep per worker per step)", "n": args.n, "npz": args.npz},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": samples[0]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)


def _parse_members(spec):
    """'16x48x79,8x96x79' -> [(48, 79), ... repeated]."""
    out = []
    for part in spec.split(","):
        count, n, npz = (int(x) for x in part.lower().split("x"))
        out += [(n, npz)] * count
    return out


def run_ensemble(args):
    """Ensemble of seed-perturbed members at mixed resolutions (16 x C48 L79,
    8 x C96 L79, 4 x C192 L63 by default): the members of each resolution batched in one context,
    so every kernel of an AcousticDynamics call advances all of them in one
    launch, one CUDA graph per ensemble step, optionally after the
    launch-shape autotuner; against the same members one at a time (one
    context and one call per member), eager and as one graph.  Each step
    first returns every member to its initial state (a device-to-device
    copy, inside every timing).  The two forms run in turn, so one ensemble
    is on the device at a time."""
    import torch

    from fv3core_b200 import _lib, autotune
    from fv3core_b200.ensemble import Ensemble

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    prec = "f64" if args.precision == "f64" else "f32"
    spec = _parse_members(args.members)
    members = [(n, npz, 1000 * rank + q) for q, (n, npz) in enumerate(spec)]
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(run):
        for _ in range(args.warmup):
            run()
        barrier()
        l0 = _lib.launch_count(prec)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            barrier()
            a.record(stream)
            for _ in range(args.steps):
                run()
            b.record(stream)
            barrier()
        return a.elapsed_time(b) / args.steps, (_lib.launch_count(prec) - l0) // args.steps, clk.summary()

    results = {}
    shape = _lib.get_launch_shape(prec)
    tuned = None
    cell_levels = None
    for mode in ("one_at_a_time", "batched"):
        ens = Ensemble(members, precision=prec, n_split=args.n_split, batched=(mode == "batched"))
        cell_levels = ens.cell_levels
        ens.step()  # the first call uploads per-level factors
        ens.keep_initial()
        if mode == "batched" and args.autotune:
            shape, timings = autotune.tune(lambda: ens.step(reset=True), precision=prec, repeats=1)
            tuned = {"x".join(map(str, k)): round(v, 3) for k, v in timings.items()}
        eager_ms, eager_launches, _ = timed(lambda: ens.step(reset=True))
        graph = ens.capture(reset=True)
        graph_ms, _, clocks = timed(graph.replay)
        results[mode] = {"eager_ms": eager_ms, "graph_ms": graph_ms, "launches": eager_launches, "clocks": clocks,
                         "contexts": len(ens.members)}
        del graph
        ens.close()
        torch.cuda.empty_cache()
    vals = max_over_ranks([results[m][k] for m in ("one_at_a_time", "batched") for k in ("eager_ms", "graph_ms")],
                          dist)
    results["one_at_a_time"]["eager_ms"], results["one_at_a_time"]["graph_ms"] = vals[0], vals[1]
    results["batched"]["eager_ms"], results["batched"]["graph_ms"] = vals[2], vals[3]
    cells = cell_levels * args.n_split * world
    bt, one = results["batched"], results["one_at_a_time"]
    line = {
        "metric": "ensemble acoustic-substep cell-levels/s", "value": cells / (bt["graph_ms"] * 1e-3),
        "unit": "cell-levels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": bt["graph_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed: f32 fields and arithmetic, f64 column solves" if prec == "f32" else "f64",
        "data": "synthetic (seeded baroclinic-wave states, one seed per member)",
        "config": {"workload": f"ensemble {args.members} (count x n x npz), n_split={args.n_split}: the members of "
                               "each resolution batched in one context (one launch per kernel per resolution), "
                               "one CUDA graph per ensemble step; each step resets the members to their initial "
                               "state",
                   "members": len(spec), "batched_contexts": bt["contexts"], "cell_levels": cell_levels,
                   "launch_shape": list(shape), "autotune_ms": tuned, "l2": "inputs larger than L2 in total; no flush"},
        "clocks": bt["clocks"], "gpu_launches": bt["launches"],
        "batched_eager": {"value": cells / (bt["eager_ms"] * 1e-3), "ms_per_step": bt["eager_ms"]},
        "one_at_a_time": {"value": cells / (one["eager_ms"] * 1e-3), "ms_per_step": one["eager_ms"],
                          "gpu_launches": one["launches"], "contexts": one["contexts"],
                          "graph": {"value": cells / (one["graph_ms"] * 1e-3), "ms_per_step": one["graph_ms"]}},
        "batched_speedup_vs_one_at_a_time": one["eager_ms"] / bt["graph_ms"],
        "graph_speedup_vs_eager": bt["eager_ms"] / bt["graph_ms"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _time_c_grid_chain(args, st, zh, dev, timed):
    """Forward and forward + backward times (ms) of the C-grid vertical
    chain of the acoustic loop (dyn_core.py): UpdateGeopotentialHeightOnCGrid,
    RiemannSolverC and p_grad_c, through their torch.autograd Functions."""
    import numpy as np
    import torch

    from fv3core_b200.adjoint import p_grad_c, riem_solver_c, update_dz_c
    from fv3core_b200.grid import CubedSphereGrid
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.storage import to_device

    n, npz = args.adj_n, args.npz
    grid = CubedSphereGrid(n, 3)
    gd = GridData(grid, npz)
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    ak, bk = np.asarray(st["ak"]), np.asarray(st["bk"])
    dp_ref = np.zeros(npz + 1)
    dp_ref[:npz] = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    area = np.asarray(grid.area)[:, :, :, None]
    rng = np.random.default_rng(3)
    c = {k: to_device(v) for k, v in {
        "ut": 0.02 * area * rng.standard_normal(zh.shape), "vt": 0.02 * area * rng.standard_normal(zh.shape),
        "uc": 10.0 * rng.standard_normal(zh.shape), "vc": 10.0 * rng.standard_normal(zh.shape),
        "dp_ref": dp_ref, "zs": st["phis"] * (1.0 / 9.80665), "hs": st["phis"], "ws": np.zeros(st["phis"].shape),
    }.items()}
    base = {"ut": c["ut"], "vt": c["vt"], "gz": to_device(zh), "w3": dev["w"], "delpc": dev["delp"],
            "ptc": dev["pt"], "uc": c["uc"], "vc": c["vc"]}
    x = {k: v.clone().requires_grad_(True) for k, v in base.items()}
    dt2, ptop, p_fac = 225.0 / 12, float(st["ptop"]), 0.05
    gen = torch.Generator(device="cuda").manual_seed(2)
    gu = torch.randn(c["uc"].shape, dtype=torch.float64, device="cuda", generator=gen)
    gv = torch.randn(c["vc"].shape, dtype=torch.float64, device="cuda", generator=gen)

    def chain(f):
        gz1, ws1 = update_dz_c(c["dp_ref"], c["zs"], f["ut"], f["vt"], f["gz"], c["ws"], sf, dt2)
        pef, gz2 = riem_solver_c(f["w3"], gz1, f["delpc"], f["ptc"], dev["cappa"], c["hs"], ws1, dev["q_con"],
                                 sf.grid_indexing, dt2, ptop, p_fac)
        return p_grad_c(f["uc"], f["vc"], f["delpc"], pef, gz2, sf, dt2)

    def fwd():
        with torch.no_grad():
            return chain(base)

    def fwd_bwd():
        uc, vc = chain(x)
        ((uc * gu).sum() + (vc * gv).sum()).backward()

    return timed(fwd), timed(fwd_bwd)


def run_adjoint(args):
    """Cost of the hand-written adjoints: RiemannSolver3 alone, and the C-grid
    chain UpdateGeopotentialHeightOnCGrid, RiemannSolverC, p_grad_c; forward
    alone against forward + backward through torch autograd, C48 L79 FP64 by
    default."""
    import numpy as np
    import torch

    from fv3core_b200.adjoint import riem_solver3
    from fv3core_b200.grid import CubedSphereGrid
    from fv3core_b200.initial_state import baroclinic_state
    from fv3core_b200.storage import GridIndexing, to_device

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    n, npz = args.adj_n, args.npz
    st = baroclinic_state(CubedSphereGrid(n, 3), npz, seed=7)
    gi = GridIndexing((n, n, npz), 3)
    dev = {k: to_device(st[k]) for k in ("w", "delp", "pt", "cappa", "q_con")}
    zs = st["phis"] * (1.0 / 9.80665)
    zh = np.zeros_like(st["delz"])
    zh[..., npz] = zs
    for k in range(npz - 1, -1, -1):
        zh[..., k] = zh[..., k + 1] - st["delz"][..., k]
    dev["zh"], dev["zs"], dev["wsd"] = to_device(zh), to_device(zs), to_device(np.zeros_like(zs))
    dt, ptop, p_fac = 225.0 / 6, float(st["ptop"]), 0.05
    gen = torch.Generator(device="cuda").manual_seed(1)
    gw = torch.randn(dev["w"].shape, dtype=torch.float64, device="cuda", generator=gen)
    gdz = 1e-2 * torch.randn(dev["w"].shape, dtype=torch.float64, device="cuda", generator=gen)
    x = {k: dev[k].clone().requires_grad_(True) for k in ("w", "zh", "delp", "pt")}

    def fwd():
        with torch.no_grad():
            return riem_solver3(dev["w"], dev["zh"], dev["delp"], dev["pt"], dev["cappa"], dev["zs"], dev["wsd"],
                                dev["q_con"], gi, dt, ptop, p_fac)

    def fwd_bwd():
        a, b = riem_solver3(x["w"], x["zh"], x["delp"], x["pt"], dev["cappa"], dev["zs"], dev["wsd"], dev["q_con"],
                            gi, dt, ptop, p_fac)
        ((a * gw).sum() + (b * gdz).sum()).backward()

    def timed(f):
        for _ in range(args.warmup):
            f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    torch.cuda.reset_peak_memory_stats()
    t_f = timed(fwd)
    t_fb = timed(fwd_bwd)
    peak = torch.cuda.max_memory_allocated()
    chain_f, chain_fb = _time_c_grid_chain(args, st, zh, dev, timed)
    line = {
        "metric": f"RiemannSolver3 adjoint/forward time ratio (C{n} L{npz})", "value": t_fb / t_f,
        "unit": "ratio", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fb,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded baroclinic-wave state)",
        "config": {"workload": f"RiemannSolver3 column solve, C{n} L{npz}, forward vs forward + hand-written "
                               "adjoint through torch.autograd",
                   "forward_ms": t_f, "forward_backward_ms": t_fb, "peak_memory_bytes": peak,
                   "c_grid_chain": {"stages": "UpdateGeopotentialHeightOnCGrid, RiemannSolverC, p_grad_c",
                                    "forward_ms": chain_f, "forward_backward_ms": chain_fb,
                                    "ratio": chain_fb / chain_f}},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--npz", type=int, default=79)
    ap.add_argument("--n-split", type=int, default=6)
    ap.add_argument("--precision", choices=["both", "mixed", "f64"], default="both",
                    help="both: the mixed-precision build is the headline, FP64 is measured beside it")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-n", type=int, default=48, help="resolution of the CPU baseline sample")
    ap.add_argument("--cpu-npz", type=int, default=79)
    ap.add_argument("--ref-n", type=int, default=24, help="resolution of the reference arm's per-worker sample")
    ap.add_argument("--ref-max-workers", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-error-analysis", action="store_true",
                    help="skip the mixed-vs-FP64 error analysis of the acoustic call")
    ap.add_argument("--step-n", type=int, default=128,
                    help="resolution of the full-step measurement (0: skip the step section)")
    ap.add_argument("--error-steps", type=int, default=10,
                    help="dynamics steps of the mixed-vs-FP64 comparison at the headline resolution (0: skip)")
    ap.add_argument("--workload", choices=["acoustics", "ensemble", "adjoint"], default="acoustics",
                    help="ensemble: the mixed-resolution ensemble with CUDA-graph steps; adjoint: the "
                         "RiemannSolver3 adjoint's cost")
    ap.add_argument("--adj-n", type=int, default=48, help="adjoint workload: cube resolution")
    ap.add_argument("--members", default="16x48x79,8x96x79,4x192x63")
    ap.add_argument("--autotune", action="store_true", help="ensemble: pick the launch shape by timing first")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
