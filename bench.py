#!/usr/bin/env python
"""Benchmark of the FMM evaluation pass on B200 (one JSON line on rank 0).

Workload: 64-clump Plummer mixture, N = 4,194,304, real basis, order p = 8,
leaf size 32 (the split-precision configuration the headline metric is quoted
on).  A step is one evaluation pass over the prepared topology: Morton gather
of the resident inputs, P2M -> M2M -> M2L -> L2L -> L2P + P2P, un-permute into
input order.  Prepare (tree, lists, schedules) is done once, outside the
timed region, as in the reference's prepare_state / evaluate split.

Forms, each held to p99 relative force error <= 1e-4 against an FP64 direct
sum (its accuracy parameter chosen in the run on one target sample, errors
reported on another):
  chosen  -- the error-controlled walk (the reference's Dehnen eq. 15/16a
             acceptance, adaptive_error_model="dehnen_paper") with per-pair
             gears (2, 4, 6, 8), FP32 M2L, Kahan-compensated P2P;
  plain   -- the theta walk at the maximum order, FP32 M2L and P2P;
  split_bf16, learned_gears -- reported beside (plain's lists with the
             tensor-core M2L, or with the MLP-selected gears).

`value` is particles/s of the chosen form with inputs resident in HBM, its step
(gather + pass + un-permute) replayed as a CUDA graph (Pass.capture); `e2e` is
the same metric through the public API (FastMultipoleMethod.
differentiable_accelerations on the prepared state, whose cuda_graph option
replays the same graph) from pinned host buffers, H2D + pass + D2H inside the
timed region.  Each form is also timed launching one kernel at a time with an
event between stages (`config.eager`, the stage times).  L2 is flushed
(256 MiB write) between timed steps; each step is timed with CUDA events on
its stream.

`--impl reference` times the CPU restatement of the same pass (the reference
itself is JAX, which is not installed) on the host cores.

With torchrun (N > 1 ranks) the target leaves are split into N Morton ranges;
every rank runs the (cheap, replicated) upward sweep and evaluates its own
range: no data-path collective.  Timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particles/s for accelerations at N=4M, rel err ≤1e-4: chosen vs plain, 1 B200"
WORKLOAD = {
    "workload": "clustered 64-clump Plummer mixture, N=4194304, real basis p=8, leaf 32",
    "generator": "clustered",
    "N": 4194304,
    "order": 8,
    "leaf_size": 32,
    # the 'balanced' preset's theta = 0.6 puts this workload exactly on the error
    # bound (p99 = 1.00e-4 over 32,768 targets); 0.55 meets it with margin
    "theta": 0.55,
    "seed": 0,
}
ERR_TARGETS = 32768
ERR_BOUND = 1e-4
# Each form's accuracy parameter is chosen in the run: the largest value on
# its grid whose p99 on a selection sample of ERR_TARGETS targets (and on its
# first 4,096) stays within SELECT_BOUND, refined by EPS_REFINE bisection
# steps towards the failing grid value above it; errors are then reported on
# a disjoint sample of the same size.
SELECT_BOUND = 0.9 * ERR_BOUND
THETA_GRID = (0.6, 0.59, 0.58, 0.57, 0.56, 0.55, 0.53, 0.5)
EPS_GRID = (6e-5, 5e-5, 4e-5, 3.5e-5, 3e-5, 2.5e-5, 2e-5, 1.5e-5, 1e-5)
EPS_REFINE = 2
GEARS = (2, 4, 6, 8)
# the chosen form's candidate gear sets: order 8 alone, or the gear ladder
GEAR_SETS = ((8,), GEARS)


def m2l_flops_per_pair(p: int) -> float:
    """Algorithmic flops of one rotate+scale M2L at order p: 2 x (two
    rotation blocks sum (2l+1)^2 + the z-translation terms)."""
    rot = sum((2 * ell + 1) ** 2 for ell in range(p + 1))
    zt = sum((2 if m else 1) * sum(1 for a in range(m, p + 1) for b in range(m, p + 1) if a + b <= p)
             for m in range(p + 1))
    return 2.0 * (2 * rot + zt)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 50 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows: list[list[str]] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def wait_first(self, timeout: float = 5.0) -> None:
        """Blocks until the sampler has produced a row (nvidia-smi takes a
        moment to start), so the timed region that follows is covered."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.rows and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0),
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", 1400.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


# DRAM bytes (read + write) per launch of the dominant kernels at the bench
# workload, scaled from single-launch ncu captures of a 1M-particle case by
# the units processed (far pairs / particle pairs); see profiles/.
TRAFFIC_PER_UNIT = {"k_m2l_units": 7.8, "k_m2l_units_coop": 8.9, "k_m2l_mixed": 10.7, "k_m2l_tc_units": 12.3,
                    "k_leaf_units_flat": 0.0124}


def _traffic(kernel: str, units: float | None = None):
    per = TRAFFIC_PER_UNIT.get(kernel)
    if per is None or units is None:
        return None
    return per * units


# ---------------------------------------------------------------------------
REF_THETA = 0.5875  # the theta the plain form's in-run selection picks for this workload
REF_SLICES = 8


class OracleSlices:
    """The CPU restatement of the pass (the oracle, FP32, all host threads) on
    the benchmark workload with the oracle's own tree and lists
    (oracle/tree_oracle.cpp).  A step is the pass for one of REF_SLICES
    Morton slices of the target leaves: the whole upward sweep, the M2L of
    every node whose particles meet the slice, the whole L2L cascade, then L2P
    + P2P for the slice's leaves -- a bounded sample of the workload, so that
    a run of warm-up + timed steps ends in minutes."""

    def __init__(self, n: int, theta: float = REF_THETA):
        import oracle
        from jaccpot_b200 import workloads

        oracle.build()
        self.oracle = oracle
        self.threads = oracle.set_threads(os.cpu_count() or 1)
        pos, mass = workloads.GENERATORS[WORKLOAD["generator"]](n, WORKLOAD["seed"])
        t0 = time.perf_counter()
        self.topo = oracle.tree_build(pos, mass, WORKLOAD["leaf_size"], theta)
        self.tree_s = time.perf_counter() - t0
        t = self.topo
        self.ps, self.ms = pos[t.permutation], mass[t.permutation]
        self.P = oracle.Pass(t, np.float32)
        L = t.num_leaves
        self.slices = []
        tgt = np.repeat(np.arange(t.num_nodes, dtype=np.int64), np.diff(t.far_offsets))
        for k in range(REF_SLICES):
            lo, hi = (L * k) // REF_SLICES, (L * (k + 1)) // REF_SLICES
            a = int(t.node_ranges[t.num_internal + lo, 0])
            b = int(t.node_ranges[t.num_internal + hi - 1, 1])
            keep_node = (t.node_ranges[:, 1] >= a) & (t.node_ranges[:, 0] <= b)
            keep = keep_node[tgt]
            off = np.zeros(t.num_nodes + 1, np.int64)
            np.add.at(off, tgt[keep] + 1, 1)
            self.slices.append((lo, hi, b - a + 1, np.cumsum(off), np.ascontiguousarray(t.far_sources[keep])))

    def step(self, k: int) -> int:
        """Runs slice k % REF_SLICES; returns its particle count."""
        lo, hi, count, far_off, far_src = self.slices[k % REF_SLICES]
        P, p = self.P, WORKLOAD["order"]
        centers = P.com(self.ps, self.ms)
        mult = P.upward(p, self.ps, self.ms, centers)
        P.far_off, P.far_src = far_off, far_src
        loc = P.m2l_accumulate(p, mult, centers)
        loc = P.l2l_cascade(p, centers, loc)
        P.evaluate_range(p, self.ps, self.ms, centers, loc, lo, hi, 1.0, 0.0)
        return count


def run_reference(args) -> None:
    """The reference's algorithm for the path (its CPU restatement, the oracle)
    on the benchmark workload, all host threads (see OracleSlices)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.n
    ref = OracleSlices(n)
    for k in range(args.warmup):
        ref.step(k)
    done, t_tot = 0, 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        done += ref.step(args.warmup + k)
        t_tot += time.perf_counter() - t0
    ms_step = 1e3 * t_tot / args.steps
    val = done / t_tot
    cfg = dict(WORKLOAD)
    cfg.update({"N": n, "theta": REF_THETA, "slices": REF_SLICES, "tree_s": ref.tree_s,
                "same_config": n == WORKLOAD["N"]})
    sample = (f"one of {REF_SLICES} Morton slices of the target leaves per step (whole upward sweep and L2L, M2L "
              f"of the nodes meeting the slice, L2P + P2P of its leaves), clustered N={n}, p=8, leaf 32, theta "
              f"{REF_THETA}, float32, oracle tree and lists")
    print(json.dumps({
        "metric": METRIC, "value": val, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference", "config": cfg,
        "cpu_baseline": {"value": val, "unit": "particles/s", "cores": ref.threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
def _events_ms(fn, stream, reps=10, warm=3):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def measure_prepare(pos, mass, cfg, dev, with_host: bool, fmm=None) -> dict:
    """Prepare-time tree + interaction lists for the headline workload: the GPU
    build (jb_tree_build_device; wall time around the call, which syncs: first
    call and the median of three more) and, with_host, the host build of the
    same arrays, checked identical field by field."""
    import ctypes

    import torch

    from jaccpot_b200 import _lib, tree

    lb = _lib.lib()
    p = torch.from_numpy(np.asarray(pos)).to(dev).double()
    m = torch.from_numpy(np.asarray(mass)).to(dev).double()
    st = torch.cuda.current_stream(dev).cuda_stream
    times = []
    for _ in range(4):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        h = ctypes.c_void_p()
        _lib.check(lb.jb_tree_build_device(p.shape[0], p.data_ptr(), m.data_ptr(), int(cfg["leaf_size"]),
                                           float(cfg["theta"]), st, ctypes.byref(h)), "jb_tree_build_device")
        torch.cuda.synchronize(dev)
        times.append((time.perf_counter() - t0) * 1e3)
        lb.jb_dtree_free(h)
    out = {"tree_gpu_ms_first": times[0], "tree_gpu_ms": float(np.median(times[1:])),
           "what": "Morton sort + radix split + FP64 COM/radii + dual walk + CSR lists, on the GPU"}
    if fmm is not None:  # a second prepare_state: the kernels are loaded, the pools warm
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        st2 = fmm.prepare_state(pos, mass, leaf_size=cfg["leaf_size"], max_order=cfg["order"])
        torch.cuda.synchronize(dev)
        out["prepare_state_warm_s"] = time.perf_counter() - t0
        del st2
    if with_host:
        dev_topo = tree.build_topology(p, m, leaf_size=cfg["leaf_size"], theta=cfg["theta"], device=dev)
        t0 = time.perf_counter()
        host = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=cfg["theta"])
        out["tree_host_s"] = time.perf_counter() - t0
        out["tree_host_threads"] = os.cpu_count()
        out["identical_to_host"] = all(
            np.array_equal(getattr(dev_topo, f), getattr(host, f))
            for f in ("permutation", "node_ranges", "left_child", "right_child", "parent", "node_level",
                      "level_offsets", "leaf_of_particle", "far_offsets", "far_sources", "near_offsets",
                      "near_leaves", "centers_f64", "radii_f64"))
    return out


def measure_extras(dev, stream) -> dict:
    """The other BASELINE configs on the same GPU, reported beside the headline:
    Plummer N=1,048,576, p=6, leaf 32: evaluate_prepared_state on 65,536
    int32 targets (drawn without replacement), and the adjoint of
    L = sum w . a with w ~ N(0,1)."""
    import torch

    from jaccpot_b200 import _lib, engine, tree, workloads
    from jaccpot_b200.solver import FastMultipoleMethod

    out = {}
    # config 1: uniform cube N=16,384, p=4, leaf 16, 'balanced' theta 0.6, vs FP64 direct sum (all targets)
    pos, mass = workloads.uniform_cube(16384, 0)
    fmm1 = FastMultipoleMethod(preset="balanced", G=1.0, softening=0.0, device=dev)
    st1 = fmm1.prepare_state(pos, mass, leaf_size=16, max_order=4)
    p1 = st1.pass_
    ms1 = _events_ms(lambda: p1.run(), stream)
    acc1 = p1.ws.acc4[:, :3].double().cpu().numpy()
    all_t = torch.arange(16384, dtype=torch.int32, device=dev)
    ref1 = torch.empty((16384, 4), device=dev, dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(16384, p1.ws.pos4.data_ptr(), 16384, all_t.data_ptr(), 1.0, 0.0,
                                        ref1.data_ptr(), stream.cuda_stream), "jb_direct_f64")
    e1 = workloads.relative_errors(acc1, ref1[:, :3].cpu().numpy())
    out["uniform_16k_p4"] = {"ms": ms1, "particles_per_s": 16384 / (ms1 / 1e3),
                             "err_vs_fp64_direct_p99": float(np.percentile(e1, 99)),
                             "note": "whole pass, launch-latency bound at this size"}
    n = 1048576
    pos, mass = workloads.plummer(n, 0)
    fmm = FastMultipoleMethod(preset="large_n_gpu", theta=0.6, G=1.0, softening=0.0, device=dev)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
    rng = np.random.default_rng(2)
    tg = rng.choice(n, 65536, replace=False).astype(np.int32)
    ts = torch.from_numpy(st.topology.inverse_permutation[tg].astype(np.int32)).to(dev)
    ps = st.pass_
    out_t = torch.empty((tg.size, 4), device=dev, dtype=torch.float32)
    ms_t = _events_ms(lambda: ps.evaluate_targets(ts, out=out_t), stream)
    # accuracy on 4,096 of the targets against an FP64 direct sum
    sub = ts[:4096].contiguous()
    ref = torch.empty((4096, 4), device=dev, dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(n, ps.ws.pos4.data_ptr(), 4096, sub.data_ptr(), 1.0, 0.0, ref.data_ptr(),
                                        stream.cuda_stream), "jb_direct_f64")
    got = out_t[:4096, :3].double().cpu().numpy()
    e = workloads.relative_errors(got, ref[:, :3].cpu().numpy())
    out["plummer_1M_p6_targets_65536"] = {
        "ms": ms_t, "targets_per_s": tg.size / (ms_t / 1e3),
        "err_vs_fp64_direct_p99": float(np.percentile(e, 99)),
        "note": "L2P + P2P for the targets on the prepared state (locals resident)"}
    # adjoint (config 5): forward pass + hand-written VJP, coefficients recomputed
    w = torch.from_numpy(np.random.default_rng(5).normal(size=(n, 3)).astype(np.float32)).to(dev)
    d_pos, d_mass = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    gx = torch.empty_like(d_pos)
    gm = torch.empty_like(d_mass)
    acc = torch.empty_like(d_pos)

    def fwd():
        ps.load_particles(d_pos, d_mass)
        ps.run()
        ps.unsort(acc, None)

    ms_f = _events_ms(fwd, stream, reps=5)
    ms_b = _events_ms(lambda: ps.vjp(w, gx, gm, recompute=True), stream, reps=5)
    out["plummer_1M_p6_adjoint"] = {"forward_ms": ms_f, "vjp_ms_incl_recompute": ms_b,
                                    "ratio": ms_b / ms_f,
                                    "finite": bool(torch.isfinite(gx).all() and torch.isfinite(gm).all())}
    out["gear_selector_2M"] = measure_gear_selector(dev, stream)
    return out


def measure_monitor(fmm, state, d_pos, d_mass, targets: int = 256, reps: int = 3) -> dict:
    """The facade's sampled error monitor on the chosen pass at the headline
    size: a whole re-evaluation (differentiable_accelerations on resident
    inputs) without and with one FP64 direct-sum check of `targets` random
    particles; wall clock around synchronised calls (the check reads its
    percentiles back)."""
    import torch

    from jaccpot_b200.solver import _monitor_config

    def wall(k):
        ts = []
        for _ in range(k):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fmm.differentiable_accelerations(state, d_pos, d_mass)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return 1e3 * float(np.median(ts))

    saved = fmm.error_monitor
    fmm.error_monitor = None
    off = wall(reps)
    fmm.error_monitor = _monitor_config({"targets": targets, "bound": ERR_BOUND})
    on = wall(reps)
    last = dict(fmm.error_history[-1])
    fmm.error_monitor = saved
    return {"targets": targets, "pass_ms": off, "pass_with_check_ms": on, "check_ms": on - off,
            "last_check": last, "note": "advanced={'error_monitor': ...}: FP64 direct sum on sampled targets "
                                        "after each whole-pass evaluation (jb_direct_f64), wall clock"}


def measure_gear_selector(dev, stream, n: int = 2097152, seed: int = 200, theta: float = 0.55) -> dict:
    """Config 4: the learned gear selector (MLP, gears 2/4/6/8) on the theta
    lists of a clustered system of a seed it never saw, against the plain
    maximum-order pass and against the analytic selector (the Dehnen eq. 15
    estimate at eps = the network's training budget) on the same lists:
    p99 against an FP64 direct sum on 4,096 targets, the error each adds to
    the plain pass (p99 over all particles), the gear fractions, algorithmic
    M2L flops and M2L time."""
    import torch

    from jaccpot_b200 import _lib, engine, gears, tree, workloads

    if not gears.DEFAULT_MODEL.exists():
        return None
    model = gears.GearModel.load()
    pos, mass = workloads.clustered(n, seed)
    d_pos, d_mass = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=theta, device=dev)
    ps = engine.Pass(engine.DeviceTopology(topo, dev), 8, G=1.0, eps2=0.0)
    ps.load_particles(d_pos, d_mass)
    plain = ps.run()[:, :3].clone()
    tg = np.random.default_rng(3).choice(n, 4096, replace=False)
    ts = torch.from_numpy(topo.inverse_permutation[tg].astype(np.int32)).to(dev)
    ref = torch.empty((tg.size, 4), device=dev, dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(n, ps.ws.pos4.data_ptr(), tg.size, ts.data_ptr(), 1.0, 0.0, ref.data_ptr(),
                                        stream.cuda_stream), "jb_direct_f64")
    ref = ref[:, :3].cpu().numpy()
    ps.set_gears(None, None)
    ms_plain = _events_ms(ps.m2l, stream)

    def with_gears(g):
        ps.set_gears(g, model.orders)
        acc = ps.run()[:, :3]
        add = (torch.linalg.vector_norm(acc - plain, dim=1) /
               torch.linalg.vector_norm(plain, dim=1).clamp_min(1e-30)).double().cpu().numpy()
        e = workloads.relative_errors(acc[ts.long()].double().cpu().numpy(), ref)
        gn = g.cpu().numpy()
        res = {"p99": float(np.percentile(e, 99)), "added_p99": float(np.percentile(add, 99)),
               "fraction": (np.bincount(gn, minlength=len(model.orders)) / max(1, gn.size)).tolist(),
               "m2l_flop_frac": gears.m2l_flop_fraction(gn, model.orders), "m2l_ms": _events_ms(ps.m2l, stream)}
        ps.set_gears(None, None)
        return res

    learned = with_gears(torch.as_tensor(gears.apply_gears(ps, model)).to(dev))
    ps.run()  # the plain pass's multipoles and accelerations for the analytic estimate
    analytic = with_gears(gears.analytic_gears(ps, model.budget, model.orders))
    e0 = workloads.relative_errors(plain[ts.long()].double().cpu().numpy(), ref)
    return {"N": n, "seed": seed, "theta": theta, "far_pairs": topo.num_far_pairs, "budget": model.budget,
            "plain": {"p99": float(np.percentile(e0, 99)), "m2l_ms": ms_plain},
            "learned": learned, "analytic_dehnen": analytic}


# ---------------------------------------------------------------------------
SWEEP_PLAIN_THETAS = (0.5, 0.55, 0.5875, 0.6, 0.65, 0.7)
SWEEP_ADAPTIVE = (((8,), (1e-5, 2e-5, 3e-5, 5e-5)),
                  ((2, 4, 6, 8), (1e-5, 2e-5, 3e-5, 3.24e-5, 4e-5, 5e-5, 8e-5)),
                  ((2, 4, 6, 8, 10), (3e-5, 5e-5, 8e-5, 1.2e-4)))


def run_sweep(args) -> None:
    """The accuracy / time frontier of both acceptance rules at the headline
    workload: the plain theta walk at order 8 over SWEEP_PLAIN_THETAS, and the
    error-controlled walk over eps for each gear set of SWEEP_ADAPTIVE.  One
    JSON line per point: far pairs, near interactions, stage times (CUDA
    events, L2 flushed before each step), the step as a CUDA graph, and the
    errors against an FP64 direct sum on ERR_TARGETS random targets."""
    import torch

    from jaccpot_b200 import _lib, engine, tree, workloads
    from jaccpot_b200.solver import FastMultipoleMethod

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = dict(WORKLOAD)
    n = cfg["N"] = args.n
    pos, mass = workloads.GENERATORS[cfg["generator"]](n, cfg["seed"])
    d_pos, d_mass = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    stream = torch.cuda.current_stream()
    tg = np.random.default_rng(54321).choice(n, size=min(ERR_TARGETS, n), replace=False)
    base_topo = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=0.6, device=dev)
    base = engine.Pass(engine.DeviceTopology(base_topo, dev), 1)
    base.load_particles(d_pos, d_mass)
    ts = torch.from_numpy(base_topo.inverse_permutation[tg].astype(np.int32)).to(dev)
    ref = torch.empty((tg.size, 4), device=dev, dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(n, base.ws.pos4.data_ptr(), tg.size, ts.data_ptr(), 1.0, 0.0,
                                        ref.data_ptr(), stream.cuda_stream), "jb_direct_f64")
    ref = ref[:, :3].cpu().numpy()
    del base
    acc_out = torch.empty((n, 3), device=dev, dtype=torch.float32)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)

    def measure(ps, topo, point):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        stage = np.zeros(5)
        for k in range(args.warmup + args.steps):
            flush.fill_(1.0)
            ev[0].record(stream)
            ps.load_particles(d_pos, d_mass)
            ps.upward()
            ev[1].record(stream)
            ps.m2l()
            ev[2].record(stream)
            ps.l2l()
            ev[3].record(stream)
            acc = ps.evaluate()
            ev[4].record(stream)
            ps.unsort(acc_out, None)
            ev[5].record(stream)
            torch.cuda.synchronize()
            if k >= args.warmup:
                stage += [ev[i].elapsed_time(ev[i + 1]) for i in range(5)]
        stage /= args.steps
        g = ps.capture(d_pos, d_mass, acc_out)
        per = []
        for k in range(args.warmup + args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.replay()
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= args.warmup:
                per.append(e0.elapsed_time(e1))
        del g
        ps.run()
        idx = torch.from_numpy(topo.inverse_permutation[tg].astype(np.int64)).to(dev)
        got = ps.evaluate()[idx, :3].double().cpu().numpy()
        e = workloads.relative_errors(got, ref)
        point.update({"far_pairs": int(topo.num_far_pairs), "near_interactions": int(topo.near_pair_interactions()),
                      "stage_ms": dict(zip(("upward", "m2l", "l2l", "leaf_eval", "unsort"),
                                           [round(float(x), 4) for x in stage])),
                      "graph_ms": round(float(np.mean(per)), 4), "p99": float(np.percentile(e, 99)),
                      "p50": float(np.median(e)), "meets_1e-4": bool(np.percentile(e, 99) <= ERR_BOUND)})
        print(json.dumps(point), flush=True)

    for th in SWEEP_PLAIN_THETAS:
        topo = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=th, device=dev)
        ps = engine.Pass(engine.DeviceTopology(topo, dev), cfg["order"], G=1.0, eps2=0.0)
        measure(ps, topo, {"form": "plain", "theta": th, "order": cfg["order"]})
        del ps
    for gears, eps_list in SWEEP_ADAPTIVE:
        for eps in eps_list:
            fmm = FastMultipoleMethod(theta=0.6, G=1.0, softening=0.0, adaptive_order=True, p_gears=gears,
                                      adaptive_error_model="dehnen_paper", adaptive_eps=eps,
                                      mac_force_scale_mode="paper", device=dev,
                                      advanced={"nearfield_compensated": True})
            st = fmm.prepare_state(pos, mass, leaf_size=cfg["leaf_size"], max_order=max(gears))
            per_gear = np.bincount(st.topology.far_gears, minlength=len(gears)) if st.topology.num_far_pairs else []
            measure(st.pass_, st.topology, {"form": "error-controlled", "gears": list(gears), "eps": eps,
                                            "far_pairs_per_gear": [int(c) for c in per_gear]})
            del st, fmm
    torch.cuda.synchronize()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["N"], help="particle count (default: the headline 4M)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true", help="skip the target-subset and adjoint measurements")
    ap.add_argument("--profile", choices=["chosen", "plain", "split_bf16", "learned_gears"], default=None,
                    help="after the warm-up, run one step of this form between cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--sweep", action="store_true",
                    help="instead of the bench line: the theta / eps x gear-set accuracy-time table (one GPU)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return
    if args.sweep:
        run_sweep(args)
        return

    import torch
    import torch.distributed as dist

    from jaccpot_b200 import _lib, engine, tree, workloads
    from jaccpot_b200.solver import FastMultipoleMethod

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    n = args.n
    cfg = dict(WORKLOAD)
    cfg["N"] = n
    pos, mass = workloads.GENERATORS[cfg["generator"]](n, cfg["seed"])
    d_pos = torch.from_numpy(pos).to(dev)
    d_mass = torch.from_numpy(mass).to(dev)
    if world > 1:  # sources replicated from rank 0 (one broadcast), targets sharded
        from jaccpot_b200 import sharding
        sharding.replicate_sources(d_pos, d_mass)
    stream = torch.cuda.current_stream()

    # FP64 direct-sum references on two disjoint target samples: one chooses
    # each form's accuracy parameter, the other reports the errors
    rng = np.random.default_rng(12345)
    both = rng.choice(n, size=min(2 * ERR_TARGETS, n), replace=False)
    tg_sel, tg = both[:both.size // 2], both[both.size // 2:]
    base_topo = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=0.6, device=dev)
    base_pass = engine.Pass(engine.DeviceTopology(base_topo, dev), 1)
    base_pass.load_particles(d_pos, d_mass)

    def direct_ref(targets):
        ts = torch.from_numpy(base_topo.inverse_permutation[targets].astype(np.int32)).to(dev)
        ref = torch.empty((targets.size, 4), device=dev, dtype=torch.float64)
        _lib.check(_lib.lib().jb_direct_f64(n, base_pass.ws.pos4.data_ptr(), targets.size, ts.data_ptr(), 1.0, 0.0,
                                            ref.data_ptr(), stream.cuda_stream), "jb_direct_f64")
        return ref[:, :3].cpu().numpy()

    ref_sel, ref_rep = direct_ref(tg_sel), direct_ref(tg)
    del base_pass

    def errors_of(acc4_sorted, topo, targets, ref):
        ts = torch.from_numpy(topo.inverse_permutation[targets].astype(np.int64)).to(dev)
        got = acc4_sorted[ts, :3].double().cpu().numpy()
        e = workloads.relative_errors(got, ref)
        return {"p50": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max()),
                "p99_first_4096": float(np.percentile(e[:4096], 99))}

    def meets(err) -> bool:
        return err["p99"] <= SELECT_BOUND and err["p99_first_4096"] <= SELECT_BOUND

    # plain: FP32 rotate+scale M2L + FP32 P2P at the maximum order over the
    # theta walk; theta = the largest of THETA_GRID that meets the bound on the
    # selection sample (whole-tree passes, identical on every rank)
    sel = {"bound": SELECT_BOUND, "targets": int(tg_sel.size), "plain": [], "chosen": []}
    def try_theta(th) -> bool:
        topo_t = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=th, device=dev)
        ps_t = engine.Pass(engine.DeviceTopology(topo_t, dev), cfg["order"], G=1.0, eps2=0.0)
        ps_t.load_particles(d_pos, d_mass)
        e = errors_of(ps_t.run(), topo_t, tg_sel, ref_sel)
        sel["plain"].append({"theta": th, "p99": e["p99"], "p99_first_4096": e["p99_first_4096"]})
        del ps_t
        return meets(e)

    plain_theta, failed_theta = THETA_GRID[-1], None
    for th in THETA_GRID:
        if try_theta(th):
            plain_theta = th
            break
        failed_theta = th
    for _ in range(EPS_REFINE if failed_theta is not None else 0):  # the same refinement as the chosen form's
        mid = round(0.5 * (plain_theta + failed_theta), 6)
        if try_theta(mid):
            plain_theta = mid
        else:
            failed_theta = mid
    cfg["theta"] = plain_theta

    # chosen: the error-controlled walk (Dehnen eq. 15/16a acceptance) + FP32
    # M2L + Kahan-compensated P2P, through the public API
    # (adaptive_error_model="dehnen_paper").  For each gear set of GEAR_SETS,
    # eps = the largest of EPS_GRID that meets the bound on the selection
    # sample (refined as the plain form's theta); the gear set whose step is
    # faster at its eps is the chosen form.
    def chosen_solver(eps, gears, graph=False):
        return FastMultipoleMethod(theta=0.6, G=1.0, softening=0.0, adaptive_order=True, p_gears=gears,
                                   adaptive_error_model="dehnen_paper", adaptive_eps=eps,
                                   mac_force_scale_mode="paper", device=dev,
                                   advanced={"nearfield_compensated": True, "cuda_graph": graph})

    def try_eps(eps, gears) -> bool:
        st_e = chosen_solver(eps, gears).prepare_state(pos, mass, leaf_size=cfg["leaf_size"], max_order=cfg["order"])
        e = errors_of(st_e.pass_.evaluate(), st_e.topology, tg_sel, ref_sel)
        sel["chosen"].append({"gears": list(gears), "eps": eps, "p99": e["p99"],
                              "p99_first_4096": e["p99_first_4096"]})
        del st_e
        return meets(e)

    def select_eps(gears) -> float:
        good, failed = EPS_GRID[-1], None
        for eps in EPS_GRID:
            if try_eps(eps, gears):
                good = eps
                break
            failed = eps
        # then EPS_REFINE log-space bisection steps between the passing eps and
        # the failing grid value above it
        for _ in range(EPS_REFINE if failed is not None else 0):
            mid = float(np.sqrt(good * failed))
            if try_eps(mid, gears):
                good = mid
            else:
                failed = mid
        return good

    def step_ms(eps, gears) -> float:  # the step as a CUDA graph, L2 flushed, median of 5
        st_e = chosen_solver(eps, gears).prepare_state(pos, mass, leaf_size=cfg["leaf_size"], max_order=cfg["order"])
        out = torch.empty((n, 3), device=dev, dtype=torch.float32)
        g = st_e.pass_.capture(d_pos, d_mass, out)
        fl = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)
        per = []
        for k in range(8):
            fl.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.replay()
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= 3:
                per.append(e0.elapsed_time(e1))
        del g, st_e, fl
        return float(np.median(per))

    gear_choice = []
    for gs in GEAR_SETS:
        eps_g = select_eps(gs)
        gear_choice.append({"gears": list(gs), "eps": eps_g, "step_ms": step_ms(eps_g, gs)})
    best = min(gear_choice, key=lambda c: c["step_ms"])
    if world > 1:  # every rank takes rank 0's choice (timings differ slightly between ranks)
        pick = torch.tensor([gear_choice.index(best)], device=dev)
        dist.broadcast(pick, 0)
        best = gear_choice[int(pick.item())]
    gears, chosen_eps = tuple(best["gears"]), best["eps"]
    sel["gear_sets"] = gear_choice

    fmm = chosen_solver(chosen_eps, gears, graph=True)  # the public API's deployed path: a CUDA graph of the step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    state = fmm.prepare_state(pos, mass, leaf_size=cfg["leaf_size"], max_order=cfg["order"])
    torch.cuda.synchronize()
    prep_s = time.perf_counter() - t0
    atopo = state.topology
    topo = tree.build_topology(pos, mass, leaf_size=cfg["leaf_size"], theta=plain_theta, device=dev)
    dt = engine.DeviceTopology(topo, dev)

    # leaf range of this rank (Morton order); ranks > 1 evaluate a slice
    L = topo.num_leaves
    leaf_lo, leaf_hi = (L * rank) // world, (L * (rank + 1)) // world
    forms = {
        "plain": dict(m2l_mode=_lib.JB_M2L_FP32, p2p_mode=_lib.JB_P2P_FP32),
        "split_bf16": dict(m2l_mode=_lib.JB_M2L_SPLIT_BF16, p2p_mode=_lib.JB_P2P_KAHAN),
        "learned_gears": dict(m2l_mode=_lib.JB_M2L_FP32, p2p_mode=_lib.JB_P2P_KAHAN),
    }
    passes = {k: engine.Pass(dt, cfg["order"], G=1.0, eps2=0.0, leaf_range=(leaf_lo, leaf_hi), **v)
              for k, v in forms.items()}
    if world > 1:  # the chosen pass over this rank's Morton range of the adaptive tree
        La = atopo.num_leaves
        passes["chosen"] = engine.Pass(state.device_topology, cfg["order"], G=1.0, eps2=0.0,
                                       p2p_mode=_lib.JB_P2P_KAHAN,
                                       leaf_range=((La * rank) // world, (La * (rank + 1)) // world))
        if len(gears) > 1:  # as the facade: a single order runs the plain units
            passes["chosen"].set_gears(torch.from_numpy(atopo.far_gears).to(dev), gears)
    else:
        passes["chosen"] = state.pass_
    # the learned selector (MLP gears on the theta walk), reported beside:
    # chosen once per topology from a plain pass's force scale
    from jaccpot_b200 import gears as gear_mod
    gear_info = None
    if gear_mod.DEFAULT_MODEL.exists():
        model = gear_mod.GearModel.load()
        passes["learned_gears"].load_particles(d_pos, d_mass)
        torch.cuda.synchronize()
        g0 = time.perf_counter()
        if world > 1:
            full = engine.Pass(dt, cfg["order"], G=1.0, eps2=0.0, **forms["learned_gears"])
            full.load_particles(d_pos, d_mass)
            gsel = gear_mod.apply_gears(full, model)
            passes["learned_gears"].set_gears(gsel, model.orders)
            del full
        else:
            gsel = gear_mod.apply_gears(passes["learned_gears"], model)
        torch.cuda.synchronize()
        gear_info = {"select_s": time.perf_counter() - g0, "budget": model.budget,
                     "fraction": (np.bincount(gsel, minlength=len(model.orders)) / max(1, gsel.size)).tolist(),
                     "orders": list(model.orders)}
    else:
        del passes["learned_gears"]
    acc_out = torch.empty((n, 3), device=dev, dtype=torch.float32)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)

    def step(ps: engine.Pass, ev=None):
        if ev is not None:
            ev[0].record(stream)
        ps.load_particles(d_pos, d_mass)
        ps.upward()
        if ev is not None:
            ev[1].record(stream)
        ps.m2l()
        if ev is not None:
            ev[2].record(stream)
        ps.l2l()
        if ev is not None:
            ev[3].record(stream)
        ps.evaluate()
        if ev is not None:
            ev[4].record(stream)
        ps.unsort(acc_out, None)
        if ev is not None:
            ev[5].record(stream)

    def timed(ps: engine.Pass, steps: int):
        per_step, stage = [], np.zeros(5)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(steps):
            flush.fill_(1.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
            step(ps, ev)
            torch.cuda.synchronize()
            per_step.append(ev[0].elapsed_time(ev[5]))
            stage += [ev[i].elapsed_time(ev[i + 1]) for i in range(5)]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return float(np.mean(per_step)), stage / steps

    for name, ps in passes.items():
        for _ in range(args.warmup):
            step(ps)
        torch.cuda.synchronize()
    if args.profile is not None and args.profile in passes:
        torch.cuda.profiler.start()
        step(passes[args.profile])
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    def timed_graph(g, steps: int) -> float:
        for _ in range(args.warmup):
            g.replay()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        per = []
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.replay()
            e1.record(stream)
            torch.cuda.synchronize()
            per.append(e0.elapsed_time(e1))
        if world > 1:
            dist.barrier()
        return float(np.mean(per))

    # every form timed in turn, eagerly with an event between stages; then the
    # chosen and plain steps as CUDA graphs (Pass.capture: gather + pass +
    # un-permute, the same launches); clocks sampled over all timed regions
    timings, graph_ms = {}, {}
    with ClockSampler(local) as cs:
        cs.wait_first()
        for name, ps in passes.items():
            timings[name] = timed(ps, args.steps)
            if name == "split_bf16":
                ps.check_tc_status()  # a timed-out MMA barrier voids the form's numbers
        for name in ("chosen", "plain"):
            g = passes[name].capture(d_pos, d_mass, acc_out)
            graph_ms[name] = timed_graph(g, args.steps)
            del g
    clocks = cs.summary()

    def overlap_timeline(ps: engine.Pass, steps: int = 3) -> dict:
        """When each stream's part of the two-stream step ends (events from
        the step's start; eager, median of `steps`): the near field on the
        caller's stream, the upward sweep + M2L + L2L on the pass's
        high-priority stream, and the L2P after the join."""
        far = ps.far_stream()
        rows = []
        for _ in range(steps):
            flush.fill_(1.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ps.load_particles(d_pos, d_mass)
            ev[0].record(stream)
            far.wait_stream(stream)
            ps.evaluate(stream, part="near_first")
            ev[1].record(stream)
            ps.upward(far)
            ps.downward(far)
            ev[2].record(far)
            stream.wait_stream(far)
            ps.evaluate(stream, part="far_after")
            ev[3].record(stream)
            torch.cuda.synchronize()
            rows.append([ev[0].elapsed_time(ev[i]) for i in (1, 2, 3)])
        med = np.median(np.array(rows), axis=0)
        return {"near_field_done": float(med[0]), "far_chain_done": float(med[1]), "step_done": float(med[2])}

    timeline = overlap_timeline(passes["chosen"])

    def reduce_max(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms = {k: reduce_max(v[0]) for k, v in timings.items()}
    gms = {k: reduce_max(v) for k, v in graph_ms.items()}
    ms_plain, ms_chosen = gms["plain"], gms["chosen"]  # the headline: the steps as graphs
    stage_chosen, stage_plain = timings["chosen"][1], timings["plain"][1]

    # accuracy of every form against the FP64 direct sum on the report sample
    errs = {}
    for name, ps in passes.items():
        step(ps)
        torch.cuda.synchronize()
        tp = atopo if name == "chosen" else topo
        if world > 1:  # every rank's sorted slice, reassembled (one all_gather)
            from jaccpot_b200 import sharding
            lo_, hi_ = ps.leaf_range
            b, e = sharding.particle_range(tp, lo_, hi_)
            full_acc = sharding.gather_sorted(ps.ws.acc4[b:e].contiguous(), tp)
        else:
            full_acc = ps.ws.acc4
        errs[name] = errors_of(full_acc, tp, tg, ref_rep)
    split_err = errs.pop("split_bf16")
    learned_err = errs.pop("learned_gears", None)

    # e2e through the public API from pinned host buffers
    h_pos = torch.from_numpy(pos).pin_memory()
    h_mass = torch.from_numpy(mass).pin_memory()
    h_out = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    if world > 1:
        state.pass_ = passes["chosen"]
    for _ in range(args.warmup):
        fmm.differentiable_accelerations(state, h_pos, h_mass, out=h_out)
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fmm.differentiable_accelerations(state, h_pos, h_mass, out=h_out)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e = reduce_max(float(np.mean(e2e_ms)))

    # roofline of the dominant kernel (largest stage time of the chosen form)
    peaks = _peaks()
    near_inter = atopo.near_pair_interactions()
    p2p_flops = 20.0 * near_inter
    gear_pairs = np.bincount(atopo.far_gears, minlength=len(gears)) if atopo.num_far_pairs else np.zeros(len(gears))
    m2l_flops = float(sum(int(c) * m2l_flops_per_pair(o) for c, o in zip(gear_pairs, gears)))
    m2l_flops_plain = m2l_flops_per_pair(cfg["order"]) * topo.num_far_pairs
    # measured FP32 FMA peak (in-run probe, 148 SMs x 8 blocks x 256 thr)
    sink = torch.empty(256, device=dev)
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = 4096
    _lib.lib().jb_probe_throughput(148 * 8, 64, 0, sink.data_ptr(), stream.cuda_stream)
    pe0.record(stream)
    _lib.lib().jb_probe_throughput(148 * 8, iters, 0, sink.data_ptr(), stream.cuda_stream)
    pe1.record(stream)
    torch.cuda.synchronize()
    fp32_peak = 2.0 * 148 * 8 * 256 * iters * 8 / (pe0.elapsed_time(pe1) / 1e3) / 1e12
    # the pair rate the FP32 + MUFU pipes allow for the near field's exact
    # instruction mix, on register-resident data (probe mode 3: 24 pairs per
    # thread and iteration)
    _lib.lib().jb_probe_throughput(148 * 8, 16, 3, sink.data_ptr(), stream.cuda_stream)
    pe0.record(stream)
    _lib.lib().jb_probe_throughput(148 * 8, 512, 3, sink.data_ptr(), stream.cuda_stream)
    pe1.record(stream)
    torch.cuda.synchronize()
    mix_pairs_per_s = 148 * 8 * 256 * 512 * 24 / (pe0.elapsed_time(pe1) / 1e3)
    stage_names = ["upward", "m2l", "l2l", "leaf_eval", "unsort"]
    dom = int(np.argmax(stage_chosen))
    split_m2l = False
    if stage_names[dom] == "m2l" and split_m2l:
        # tensor-core kernel: algorithmic flops against the measured bf16 peak,
        # and the same work against the FP32 pipe, where its per-pair rotations run
        ach = m2l_flops / (stage_chosen[1] / 1e3) / 1e12
        roof = {"kernel": f"k_m2l_tc_units<{cfg['order']}>", "bound": "tensor", "achieved": ach,
                "peak": peaks["bf16_tflops"], "unit": "TFLOP/s", "frac": ach / peaks["bf16_tflops"],
                "traffic": _traffic("k_m2l_tc_units", atopo.num_far_pairs), "fp32_pipe_frac": ach / fp32_peak}
    elif stage_names[dom] == "m2l":
        ach = m2l_flops / (stage_chosen[1] / 1e3) / 1e12
        kname = "k_m2l_units_coop" if len(gears) == 1 else "k_m2l_mixed"
        roof = {"kernel": f"{kname}<{cfg['order']}>", "bound": "fp32", "achieved": ach,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak,
                "traffic": _traffic(kname, atopo.num_far_pairs)}
    else:
        ach = p2p_flops / (stage_chosen[3] / 1e3) / 1e12
        pairs_per_s = near_inter / (stage_chosen[3] / 1e3)
        roof = {"kernel": "k_leaf_units_flat<kahan> (leaf stage: + k_leaf_l2p, k_leaf_reduce)", "bound": "fp32",
                "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak,
                "traffic": _traffic("k_leaf_units_flat", near_inter),
                "pairs_per_s": pairs_per_s, "mix_peak_pairs_per_s": mix_pairs_per_s,
                "frac_of_mix_peak": pairs_per_s / mix_pairs_per_s}
    roof["peak_source"] = ("measured bf16 burst (MEASURED_PEAKS.json)" if roof["bound"] == "tensor" else
                           "in-run FP32 FMA probe (MEASURED_PEAKS.json has HBM and bf16 only)")
    roof["stage_ms"] = float(stage_chosen[dom])
    roof["algorithmic"] = "P2P 20 flop/pair x near pairs; M2L 2*(2*sum(2l+1)^2 + z-terms) flop/pair"

    ms_split, stage_split = ms["split_bf16"], timings["split_bf16"][1]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ref = OracleSlices(n)
        t0 = time.perf_counter()
        cnt = ref.step(0)
        cdt = time.perf_counter() - t0
        cpu = {"value": cnt / cdt, "unit": "particles/s", "cores": ref.threads, "kind": "port",
               "sample": f"the oracle (float32, its own tree) on 1 of {REF_SLICES} Morton slices of the target "
                         f"leaves of the same workload (N={n}, theta {REF_THETA}): whole upward sweep and L2L, "
                         f"M2L of the nodes meeting the slice, L2P + P2P of its leaves"}

    extras = measure_extras(dev, stream) if (rank == 0 and world == 1 and not args.no_extras) else None
    if extras is not None:
        extras["error_monitor"] = measure_monitor(fmm, state, d_pos, d_mass)
    prep = measure_prepare(pos, mass, cfg, dev, with_host=not args.no_extras, fmm=fmm) if rank == 0 else None
    launches = passes["chosen"].launches_per_run() + 2  # + gather + unsort
    if rank == 0:
        cfg.update({
            "form": (f"chosen = error-controlled walk (Dehnen eq. 15/16a acceptance, eps={chosen_eps:g}, "
                     f"per-pair gears {gears}, chosen in the run from {GEAR_SETS}) + FP32 rotate+scale M2L + Kahan-compensated P2P; plain = theta walk "
                     f"(theta={plain_theta:g}) + FP32 M2L + FP32 P2P at the maximum order p={cfg['order']}; "
                     "split_bf16 = plain's lists with the tcgen05 split-BF16 M2L + Kahan P2P; learned_gears = "
                     "plain's lists with the MLP-selected gears + Kahan P2P"),
            "selection": sel,
            "streams": ("the graphed steps (the headline) run the near field on the caller's stream while the "
                        "upward sweep, M2L and L2L run on a high-priority stream, joined before the L2P "
                        "(Pass.overlap; the same bits as one stream)"),
            "overlap_timeline_ms_chosen": timeline,
            "chosen_vs_plain": ms_plain / ms_chosen,
            "eager": {"chosen_ms_per_step": ms["chosen"], "plain_ms_per_step": ms["plain"],
                      "chosen_vs_plain": ms["plain"] / ms["chosen"],
                      "note": "the same steps launched one kernel at a time with an event between stages "
                              "(stage_ms_* come from these runs)"},
            "chosen": {"eps": chosen_eps, "gears": list(gears), "theta_max": 1.0, "theta_prepass": 0.6,
                       "far_pairs": atopo.num_far_pairs, "far_pairs_per_gear": [int(c) for c in gear_pairs],
                       "near_leaf_pairs": atopo.num_near_pairs, "near_interactions": near_inter,
                       "m2l_algorithmic_flop": m2l_flops,
                       "m2l_kernel": "k_m2l_units_coop" if len(gears) == 1 else "k_m2l_mixed",
                       "m2l_tflops": m2l_flops / (stage_chosen[1] / 1e3) / 1e12,
                       "m2l_frac_of_fp32_probe": m2l_flops / (stage_chosen[1] / 1e3) / 1e12 / fp32_peak},
            "learned_gears": None if learned_err is None else {
                "ms_per_step": ms["learned_gears"], "particles_per_s": n / (ms["learned_gears"] / 1e3),
                "stage_ms": dict(zip(stage_names, [float(x) for x in timings["learned_gears"][1]])),
                "err_vs_fp64_direct": learned_err, "selector": gear_info},
            "split_bf16": {
                "ms_per_step": ms_split, "particles_per_s": n / (ms_split / 1e3),
                "stage_ms": dict(zip(stage_names, [float(x) for x in stage_split])),
                "err_vs_fp64_direct": split_err, "err_bound_met": bool(split_err["p99"] <= ERR_BOUND),
                "m2l_tensor_frac": m2l_flops_plain / (stage_split[1] / 1e3) / 1e12 / peaks["bf16_tflops"],
                "m2l_fp32_pipe_frac": m2l_flops_plain / (stage_split[1] / 1e3) / 1e12 / fp32_peak},
            "plain_particles_per_s": n / (ms_plain / 1e3),
            "plain_ms_per_step": ms_plain,
            "stage_ms_chosen": dict(zip(stage_names, [float(x) for x in stage_chosen])),
            "stage_ms_plain": dict(zip(stage_names, [float(x) for x in stage_plain])),
            "err_vs_fp64_direct": errs,
            "err_targets": int(tg.size),
            "err_bound_met": bool(errs["chosen"]["p99"] <= ERR_BOUND),
            "prepare_s": prep_s,  # first prepare_state of the process (kernel loading included)
            "prepare": prep,
            "num_nodes": topo.num_nodes,
            "plain_far_pairs": topo.num_far_pairs,
            "plain_near_leaf_pairs": topo.num_near_pairs,
            "plain_near_interactions": topo.near_pair_interactions(),
            "l2": "flushed (256 MiB write) between timed steps",
            "parallelism": f"target-leaf ranges over {world} rank(s)",
            "timing": ("CUDA events around each step on the launching stream (the chosen and plain steps "
                       "replayed as CUDA graphs; `eager` and the stage times from the same steps launched one "
                       "kernel at a time); max over ranks"),
        })
        line = {
            "metric": METRIC, "value": n / (ms_chosen / 1e3), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_chosen, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": n / (e2e / 1e3), "unit": "particles/s", "h2d_bytes_per_step": n * 16,
                    "d2h_bytes_per_step": n * 12, "ms_per_step": e2e},
            "gpu_launches": launches * args.steps,
            "other_configs": extras,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
