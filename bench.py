"""Benchmark: 3-D Coulomb treecode solve on one B200 (replicas on N GPUs).

Workload (the headline configuration): N = 1,048,576 points uniform in the
unit cube (seeded SplitMix64), charges uniform in [-1,1], targets = sources,
Chebyshev degree n = 8 (729 proxy points per cluster), MAC theta = 0.7, leaf
size 2000, kernel eps = 1e-4; potential + gradient (field -grad phi).

A step is one full solve (upward pass, PP/PC/CP/CC interactions, downward
pass) on device-resident inputs; L2 is flushed (256 MB write) before every
timed step, outside the timed region. ``value`` is interactions (pairwise
kernel evaluations, at each interaction's degree) per second over the whole
job; ``e2e`` is the same metric through the C ABI with pinned host buffers,
the host->device copies of coordinates and charges and the device->host copy
of the results inside the timed region.

``--impl reference`` times the reference's own CPU implementation (its
sources compiled with OpenMP against the project's Kokkos-API shim,
oracle/_ref/libbtkref.so) on this host's cores, on strided samples of the same
solve.
"""
from __future__ import annotations

import argparse
import ctypes
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

METRIC = "3D N=1M solve ms & interactions/s: learned+FP32 vs plain FP64 at 1e-6 rel L2"
N_POINTS = 1 << 20  # overridable with --points for small profiling captures
DEGREE, THETA, LEAF, EPS = 8, 0.7, 2000, 1e-4
SEED = 1
# Algorithmic flops per pairwise evaluation (FMA = 2, rsqrt/rcp = 1):
# 3-D potential 13, potential + Coulomb gradient 24.
FLOPS_PER_EVAL = {0: 13, 2: 24}


def bench_config(kind):
    """The workload both arms measure: the same object in the native and the
    reference arm's line (the form each arm computes it with is reported
    beside it, under "form")."""
    what = "potential+gradient" if kind == 2 else "potential"
    return {"workload": (f"3D Coulomb {what}, N={N_POINTS} uniform unit cube, charges U[-1,1], targets = sources, "
                         f"n={DEGREE}, theta={THETA}, leaf {LEAF}, eps {EPS}"),
            "tolerance_rel_l2": TOL,
            "value_definition": "interactions of the plain fixed-degree solve of this workload (pairwise evaluations "
                                "at n=8) divided by the solve time of the reported form"}


def workload_name(kind, precision):
    what = "potential+gradient" if kind == 2 else "potential"
    prec = "plain FP64" if precision == 0 else "mixed FP32/FP64"
    return (f"3D Coulomb {what}, N={N_POINTS} uniform unit cube, charges U[-1,1], n={DEGREE}, theta={THETA}, "
            f"leaf {LEAF}, eps {EPS}, {prec}")


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
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
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


# ---------------------------------------------------------------- distributed
def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    from barytreek_b200.distributed import reduce_over_ranks
    return reduce_over_ranks(x, "max") if world > 1 else x


# ---------------------------------------------------------------- reference arm
def reference_tree(points, threads):
    from oracle import RefLib
    ref = RefLib(threads=threads)
    return ref.create(3, points, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS)


def reference_sample(rt, q, target_seconds):
    """Strided, timed samples of the reference's own functors (OpenMP build).
    Potential + gradient = the reference's potential pass plus its gradient-type
    (velocity) pass over the same pairs. Returns dict(value, est_solve_s,
    sampled_s = wall seconds of the sample, ...)."""
    t0 = time.perf_counter()
    # calibrate the stride on a very sparse sample
    cal = 4096
    sec, scale, ev = rt.time_sample_3d(0, cal, q)
    est_full = float(np.sum(sec * scale))
    stride = max(1, int(np.ceil(2 * est_full / max(target_seconds, 1e-3))))
    total_s, evals = 0.0, 0.0
    for kind in (0, 1):
        sec, scale, ev = rt.time_sample_3d(kind, stride, q)
        total_s += float(np.sum(sec * scale))
        evals = float(ev[1])
    return {"value": evals / total_s, "est_solve_s": total_s, "sampled_s": time.perf_counter() - t0,
            "stride": stride, "evals": evals}


VALIDATION_POINTS = 65536


def reference_validation(threads):
    """The sampled estimate against one whole, unsampled reference solve
    (potential pass + velocity pass, the fixed downward pass) of the same
    workload family at N = 65,536 (3-D uniform cube, n = 8, theta 0.7, leaf
    2000): est_solve_s / full_solve_s."""
    from barytreek_b200 import datagen
    from oracle import RefLib
    ref = RefLib(threads=threads)
    pts, q = datagen.uniform_box(SEED, VALIDATION_POINTS, 3, 0.0, 1.0)
    rt = ref.create(3, pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS)
    t0 = time.perf_counter()
    rt.solve(0, q, fixed=True)
    rt.solve(1, q, fixed=True)
    full = time.perf_counter() - t0
    est = reference_sample(rt, q, 1.0)
    return {"points": VALIDATION_POINTS, "full_solve_s": full, "est_solve_s": est["est_solve_s"],
            "validated_ratio": est["est_solve_s"] / full}


def reference_config1(threads):
    """BASELINE configuration 1 in full through the reference: 2-D, N = 65,536
    uniform in [-1,1]^2, n = 8, theta 0.7, leaf 500, potential (all leaves on
    the last level: the unmodified downward pass)."""
    from barytreek_b200 import datagen
    from oracle import RefLib
    ref = RefLib(threads=threads)
    pts, q = datagen.uniform_box(SEED, 65536, 2, -1.0, 1.0)
    rt = ref.create(2, pts, degree=8, cluster_size=500, theta=0.7, eps=EPS)
    t0 = time.perf_counter()
    rt.solve(0, q, fixed=False)
    return {"workload": "2-D potential, N=65536 uniform [-1,1]^2, n=8, theta=0.7, leaf 500, plain FP64",
            "full_solve_ms": 1e3 * (time.perf_counter() - t0), "leaves_on_last_level": rt.leaves_on_last_level_only()}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    from barytreek_b200 import datagen
    from oracle import RefLib
    if not RefLib.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libbtkref.so not built (reference tree absent at build)"}
    pts, q = datagen.uniform_box(SEED, N_POINTS, 3, 0.0, 1.0)
    cores = cpu_cores()
    per_step = float(os.environ.get("BTK_REF_STEP_SECONDS", "5"))
    rt = reference_tree(pts, cores)
    vals, ests, walls = [], [], []
    for i in range(args.warmup + args.steps):
        r = reference_sample(rt, q, per_step)
        if i >= args.warmup:
            vals.append(r["value"])
            ests.append(r["est_solve_s"])
            walls.append(r["sampled_s"])
    value = statistics.median(vals)
    val = reference_validation(cores)
    sample = (f"one step = every {r['stride']}-th work item of each phase (base_pots, child_to_parent, PP, PC, CP, "
              f"CC, parent_to_child, leaf_to_point; at least 8 items per thread) of the potential pass and of the "
              f"velocity pass, timed; interactions/s = the whole solve's interactions / the work-scaled sample time")
    return {"metric": METRIC, "value": value, "unit": "interactions/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64)",
            "impl": "reference",
            "config": bench_config(2),
            "form": {"name": "reference",
                     "description": "the reference's own code, plain FP64 at n=8 on this workload: its potential pass "
                                    "and its 3-D vector-kernel (velocity) pass, which stands in for the gradient (the "
                                    "reference has no Coulomb-gradient kernel)"},
            "parallelism": "OpenMP host threads",
            "step": "a bounded sample of the solve (see cpu_baseline.sample)",
            "cpu_baseline": {"value": value, "unit": "interactions/s", "cores": cores, "kind": "reference",
                             "sample": sample, "est_solve_s": statistics.median(ests),
                             "validated_ratio": val["validated_ratio"], "validation": val},
            "configs": {"cfg1_2d_65k": reference_config1(cores)},
            "e2e": {"value": value, "unit": "interactions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------- native arm
def flush_l2(buf):
    buf.add_(1.0)


def direct_check(tc, q, kind, m=10000, eps=None):
    """FP64 direct sum (btk_direct_sum) at m seeded targets: (indices, values)."""
    import torch
    from barytreek_b200 import _lib
    L = _lib.load()
    m = min(m, tc.nt)
    idx = np.sort(np.random.default_rng(12345).choice(tc.nt, m, replace=False))
    t = [torch.from_numpy(np.ascontiguousarray(c[idx])).cuda() for c in tc.targets]
    out = torch.empty((tc.ncomp, m), dtype=torch.float64, device="cuda")
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    s = tc._s
    z = (lambda a: _lib.ptr(a[2])) if tc.dim == 3 else (lambda a: None)
    _lib.check(L.btk_direct_sum(tc.dim, kind, EPS if eps is None else eps, m, _lib.ptr(t[0]), _lib.ptr(t[1]), z(t),
                                tc.ns, _lib.ptr(s[0]), _lib.ptr(s[1]), z(s), _lib.ptr(qd), _lib.ptr(out), None))
    return idx, out.cpu().numpy()


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def event_ms(fn, flush):
    """Device time of fn() on the current stream (L2 flushed before)."""
    import torch
    flush_l2(flush)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r = fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1), r


# DRAM bytes (read + write) of one launch of the headline form's interaction
# kernel at the full workload, from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum; profiles/k_interact_mixed_learned_1m_traffic.md gives
# the command and the algorithmic bytes it compares with). None when the
# workload differs from the captured one.
TRAFFIC_BYTES = {("k_interact_mixed", "learned", 2, 1 << 20): 1730000000 + 192830000}


class Form:
    """One way of solving the workload: plain FP64 fixed degree (the reference
    method), mixed precision fixed degree, or learned degrees + mixed; the
    *_cc names apply the CC pairs as shared kernel matrices (cc_operators)."""

    def __init__(self, name, pts, args):
        import barytreek_b200 as btk
        from barytreek_b200 import selector
        self.name = name
        kind = args.kind
        self.sel = None
        if name in ("plain", "plain_cc"):
            self.tc = btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=kind,
                                   precision=btk.PREC_FP64, cc_operators=name.endswith("_cc"))
        elif name in ("mixed", "mixed_cc"):
            self.tc = btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=kind,
                                   precision=btk.PREC_MIXED, cc_operators=name.endswith("_cc"))
        else:
            self.tc = btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=kind,
                                   precision=btk.PREC_MIXED, degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4,
                                   leaf_far_pairs=True)
            self.sel = selector.Selector.load(kind=kind)
        self.report = None

    def step(self, qd, out=None, coords=None):
        """One solve; returns (total ms, interaction-kernel ms, evaluations)."""
        tc = self.tc
        if coords is not None:  # e2e: fresh device inputs
            tc._t = tc._s = coords
        if self.sel is None:
            out = tc.solve(qd, out)
            t = tc.last_timing()
            return out, t["total"], t["interaction_kernel"], tc.evals(), t
        # pair_tol=None: the plan's adaptive per-pair tolerance, steered by each solve's audit
        out, rep = tc.solve_learned(qd, self.sel, tol=TOL, pair_tol=None, degree_lo=4, out=out)
        self.report = rep
        return out, rep["ms_total"], rep["ms_kernel"], rep["evals_near"] + rep["evals_far"], rep


TOL = 1e-6
# HBM roofline denominator: MEASURED_PEAKS.json (driver-written) when present,
# else the pool's earlier copy-bandwidth measurement.
try:
    HBM_PEAK_GBS = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    HBM_PEAK_SOURCE = "MEASURED_PEAKS.json hbm_gbs (measured)"
except Exception:
    HBM_PEAK_GBS = 6650.0
    HBM_PEAK_SOURCE = "fallback 6.65 TB/s (earlier copy measurement on this pool)"


def time_form(form, qd, flush, args, world, local):
    import torch
    from barytreek_b200 import _lib
    L = _lib.load()
    for _ in range(args.warmup):
        form.step(qd)
    barrier(world)
    torch.cuda.synchronize()
    launches0 = L.btk_launch_count()
    tot, kern, evals, info = [], [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            out, t, k, e, extra = form.step(qd)
            tot.append(t)
            kern.append(k)
            evals.append(e)
            info.append(extra)
        torch.cuda.synchronize()
    launches = (L.btk_launch_count() - launches0) / max(1, args.steps)
    total = max_over_ranks(sum(tot), world)
    return {"ms": total / args.steps, "kernel_ms": statistics.mean(kern), "evals": statistics.mean(evals),
            "launches": launches, "clocks": clk.summary(), "out": out, "info": info[-1]}


def run_native(args, world, rank, local):
    import torch
    from barytreek_b200 import _lib, datagen, selector
    L = _lib.load()
    kind = args.kind
    pts, q = datagen.uniform_box(SEED, N_POINTS, 3, 0.0, 1.0)
    qd = torch.from_numpy(q).cuda()
    flush = torch.empty(32 << 20, dtype=torch.float64, device="cuda")  # 256 MB > 126 MB L2
    headline = args.form
    if headline == "learned" and not os.path.exists(selector.DEFAULT_WEIGHTS):
        headline = "mixed"
    names = (["plain", "mixed", "learned", "plain_cc", "mixed_cc"] if headline == "learned"
             else sorted({"plain", headline}))
    if args.forms:
        names = [n for n in names if n in args.forms.split(",") or n == headline]
    results, forms = {}, {}
    for name in names:
        t0 = time.time()
        forms[name] = Form(name, pts, args)
        torch.cuda.synchronize()
        setup = time.time() - t0
        results[name] = time_form(forms[name], qd, flush, args, world, local)
        results[name]["setup_s"] = setup
    plain_evals = (forms["plain"].tc if "plain" in forms else
                   btk_plan_for_count(pts, kind)).evals()
    H = results[headline]
    cold = None
    if headline == "learned":
        # the first solve on a fresh plan: the adaptive per-pair tolerance at
        # its starting point (0.05 tol), no solve before it to settle it
        fresh = Form("learned", pts, args)
        torch.cuda.synchronize()
        ms, _ = event_ms(lambda: fresh.step(qd), flush)
        rep0 = fresh.report
        cold = {"ms": ms, "audit_rel_l2": rep0["audit_rel_l2"], "fell_back": rep0["fell_back"],
                "pair_tol": rep0["pair_tol"], "evals_far": rep0["evals_far"]}
        fresh.tc.close()
    # plan set-up of the headline form with the trees and lists built on the
    # GPU (what a caller with moving points pays per rebuild), against the
    # host-built set-up timed above
    import barytreek_b200 as btk
    setup_dev = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tcd = btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=kind,
                           precision=forms[headline].tc.precision, degree_mode=forms[headline].tc.degree_mode,
                           degree_min=forms[headline].tc.degree_min, device_tree=True)
        torch.cuda.synchronize()
        setup_dev.append(time.perf_counter() - t0)
        tcd.close()
    ms_per_step = H["ms"]
    value = world * plain_evals / (ms_per_step * 1e-3)

    # e2e through the C ABI for the headline form: pinned host coordinates and
    # charges -> device, solve, results -> host, all inside the timed region.
    f = forms[headline]
    h_in = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (*pts, q)]
    d_in = [torch.empty_like(a, device="cuda") for a in h_in]
    h_out = torch.empty((f.tc.ncomp, f.tc.nt), dtype=torch.float64).pin_memory()
    d_out = torch.empty((f.tc.ncomp, f.tc.nt), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_ms = []
    keep = (f.tc._t, f.tc._s)
    for i in range(args.warmup + args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        e0.record(stream)
        for h, d in zip(h_in, d_in):
            d.copy_(h, non_blocking=True)
        f.step(d_in[3], d_out, coords=d_in[:3])
        h_out.copy_(d_out, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    f.tc._t, f.tc._s = keep
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = world * plain_evals / (e2e_total / args.steps * 1e-3)
    h2d = sum(h.numel() * h.element_size() for h in h_in)
    d2h = h_out.numel() * h_out.element_size()
    ref_out = H["out"].cpu().numpy()
    assert np.linalg.norm(h_out.numpy() - ref_out) <= 1e-6 * np.linalg.norm(ref_out)

    # every rank takes part in the batch measurement (its shard of the problems)
    batch_line = run_batch(args, flush) if not args.no_batch else None
    if rank != 0:
        return None
    idx, ds = direct_check(f.tc, q, kind)
    acc = {}
    for name in names:
        o = results[name]["out"].cpu().numpy()[:, idx]
        acc[name] = float(np.linalg.norm(o - ds) / np.linalg.norm(ds))
    per_comp = [float(np.linalg.norm(H["out"].cpu().numpy()[c, idx] - ds[c]) / np.linalg.norm(ds[c]))
                for c in range(ds.shape[0])]
    peak, peak64 = ctypes.c_double(), ctypes.c_double()
    fp32 = headline != "plain"
    _lib.check(L.btk_measure_pipe_peak(1 if fp32 else 0, ctypes.byref(peak), None))
    _lib.check(L.btk_measure_pipe_peak(0, ctypes.byref(peak64), None))
    # the FP64 and FP32 rates the SM count and clock give (64 and 128 FMA lanes per SM)
    sm_clock_ghz = H["clocks"]["sm_mhz"] / 1e3 if H["clocks"].get("sm_mhz") else 1.965
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    spec = {"fp32_tflops": n_sm * 128 * 2 * sm_clock_ghz / 1e3, "fp64_tflops": n_sm * 64 * 2 * sm_clock_ghz / 1e3}
    kernel_ms = H["kernel_ms"]
    flops = FLOPS_PER_EVAL[kind] * H["evals"]
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    kname = "k_interact_mixed" if fp32 else "k_interact_fp64"
    line = {
        "metric": METRIC, "value": value, "unit": "interactions/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if headline == "plain" else "f32+f64",
        "data": "synthetic: seeded SplitMix64, uniform unit cube, charges U[-1,1]",
        "config": bench_config(kind),
        "form": {"name": headline,
                 "description": workload_name(kind, 0 if headline == "plain" else 1) +
                 (", learned per-pair degrees 4..8 (adaptive pair tolerance; well-separated leaf pairs may be "
                  "approximated) with 1% FP64 direct-sum audit" if headline == "learned" else ""),
                 "interactions_plain": plain_evals, "interactions_evaluated": H["evals"]},
        "l2": "flushed (256 MB write) before every step",
        "parallelism": "replicas" if world > 1 else "single GPU",
        "forms": {n: {"ms_per_step": r["ms"], "interaction_kernel_ms": r["kernel_ms"], "evaluations": r["evals"],
                      "rel_l2_vs_direct_10k": acc[n], "setup_s": r["setup_s"],
                      "speedup_vs_plain_fp64": results["plain"]["ms"] / r["ms"] if "plain" in results else None}
                  for n, r in results.items()},
        "roofline": {"bound": "fp32" if fp32 else "fp64", "achieved": achieved, "peak": peak.value,
                     "unit": "TFLOP/s", "frac": achieved / peak.value,
                     "traffic": TRAFFIC_BYTES.get((kname, headline, kind, N_POINTS)),
                     "kernel": f"{kname} (persistent PP/PC/CP/CC)",
                     "kernel_ms": kernel_ms, "flops_per_launch": flops,
                     "peak_source": "measured live: btk_measure_pipe_peak FMA-chain probe on this GPU "
                                    f"({'FP32' if fp32 else 'FP64'} pipe)",
                     "frac_of_spec": achieved / spec["fp32_tflops" if fp32 else "fp64_tflops"],
                     "spec_peaks": spec, "measured_fp64_tflops": peak64.value},
        "e2e": {"value": e2e_value, "unit": "interactions/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / args.steps},
        "gpu_launches": H["launches"],
        "setup": {"host_tree_s": H["setup_s"], "device_tree_s": statistics.median(setup_dev),
                  "what": "plan creation of the headline form: tree, traversal, split, work lists, device plan"},
        "clocks": H["clocks"],
        "accuracy": {"rel_l2_vs_direct_10k": acc[headline], "per_component": per_comp,
                     "parity": "the plain FP64 potential and the reference's vector kernel match the reference's "
                               "own code to 1e-12 at this size on sampled leaves (tests/test_gpu_fullsize_parity.py);"
                               " the gradient (FIELD) has no reference counterpart: it is pinned to the C "
                               "restatement (1e-12) and the FP64 direct sum"},
    }
    if headline == "learned":
        r = forms["learned"].report
        line["learned"] = {k: r[k] for k in ("audit_rel_l2", "audit_targets", "fell_back", "evals_near", "evals_far",
                                             "ms_select", "ms_solve", "ms_kernel", "degree_hist", "pair_tol")}
        # The audit's FP64 direct sum runs as items of the same launch. On this
        # GPU FP64 and FP32 work on one SM add up (FP64 at half the FP32 rate),
        # so the launch's roofline time is FP32 flops / FP32 peak + FP64 flops /
        # FP64 peak; achieved is given in FP32-equivalent TFLOP/s (FP64 flops
        # scaled by the measured FP32/FP64 peak ratio).
        audit_evals = r["audit_targets"] * N_POINTS
        line["learned"]["evals_audit"] = audit_evals
        flops64 = FLOPS_PER_EVAL[kind] * audit_evals
        equiv = flops + flops64 * peak.value / peak64.value
        achieved = equiv / (kernel_ms * 1e-3) / 1e12
        line["roofline"].update({"achieved": achieved, "frac": achieved / peak.value, "flops_per_launch": flops,
                                 "fp64_audit_flops_per_launch": flops64, "unit": "TFLOP/s (FP32-equivalent)",
                                 "frac_of_spec": (flops / spec["fp32_tflops"] + flops64 / spec["fp64_tflops"])
                                 / 1e12 / (kernel_ms * 1e-3)})
        line["learned"]["cold_first_solve"] = cold
    updown = updown_rates(forms.get("plain"), results.get("plain"), kind)
    if updown:
        line["roofline"]["updown"] = updown
    if not args.no_configs:
        line["configs"] = run_configs(args, flush)
        line["dropin"] = run_dropin(pts, q, flush, max(1, min(args.steps, 3)))
    if batch_line is not None:
        line["batch"] = batch_line
    if world == 1 and not args.no_cpu_baseline:
        from oracle import RefLib
        if RefLib.available():
            r = reference_sample(reference_tree(pts, cpu_cores()), q,
                                 float(os.environ.get("BTK_CPU_BASELINE_SECONDS", "10")))
            line["cpu_baseline"] = {
                "value": r["value"], "unit": "interactions/s", "cores": cpu_cores(), "kind": "reference",
                "sample": (f"reference functors (OpenMP, Kokkos-API shim build) on every {r['stride']}-th work item "
                           f"of every phase (at least 8 per thread) of the potential and velocity passes, scaled by "
                           f"work; {r['sampled_s']:.1f} s of CPU work"),
                "est_solve_s": r["est_solve_s"]}
            val = reference_validation(cpu_cores())
            line["cpu_baseline"].update({"validated_ratio": val["validated_ratio"], "validation": val})
        else:
            line["cpu_baseline"] = None
    for fm in forms.values():
        fm.tc.close()
    return line


def btk_plan_for_count(pts, kind):
    """The plain fixed-degree plan of the workload (for its interaction count)."""
    import barytreek_b200 as btk
    return btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=kind)


def updown_rates(form, result, kind):
    """Achieved HBM rates of the upward and downward passes of the plain
    form (device times from btk_plan_last_timing of its last timed solve).
    Algorithmic bytes: upward = 36 B per source point (x, y, z, q, leaf id)
    + the proxy source weights written (panels x (n+1)^3 x 8 B); downward =
    24 B per target point + the leaves' proxy target weights read (leaves x
    (n+1)^3 x 8 B per component) + 8 B per point per component written."""
    if form is None or result is None:
        return None
    t = result["info"]
    tree = form.tc.tree_t
    n, ipc, nc = form.tc.nt, (DEGREE + 1) ** 3, form.tc.ncomp
    n_leaves = int(np.count_nonzero(tree.panels["is_leaf"]))
    up = 36 * n + tree.panel_count * ipc * 8
    down = 24 * n + n_leaves * ipc * 8 * nc + 8 * n * nc
    return {"upward_ms": t["upward"], "upward_bytes": up, "upward_gbs": up / (t["upward"] * 1e-3) / 1e9,
            "downward_ms": t["downward"], "downward_bytes": down,
            "downward_gbs": down / (t["downward"] * 1e-3) / 1e9,
            "hbm_peak_gbs": HBM_PEAK_GBS, "peak_source": HBM_PEAK_SOURCE,
            "form": "plain FP64 (upward: gather, leaf moments, child->parent, source proxies; downward: "
                    "parent->child, leaf->point)"}


def run_configs(args, flush):
    """The other BASELINE configurations at full size on this GPU (seeded
    synthetic inputs with their shapes and distributions):
    cfg1: 2-D potential, N = 65,536 uniform in [-1,1]^2, n = 8, theta 0.7, leaf
          500, plain FP64;
    cfg4: 3-D potential + gradient, N = 4,194,304 Plummer sphere (scale 0.1,
          r <= 2), charges U[0,1], leaf 2000, theta 0.7: learned + mixed at
          tol 1e-6 against plain FP64 at n = 10, with mixed precision at fixed
          n = 10 beside them;
    cfg5: the reference's 3-D vector kernel, eps 1e-3, N = 2,097,152 on the
          unit sphere, strengths U[-1,1], leaf 2000, theta 0.8: the same three
          forms.
    Device times (CUDA events, L2 flushed before each solve); errors against
    the FP64 direct sum at 10,000 seeded targets. The learned form reports its
    first solve on a fresh plan (cold) and its time after 3 settling solves."""
    import torch

    import barytreek_b200 as btk
    from barytreek_b200 import datagen, selector
    steps = max(1, min(args.steps, 3))
    out = {}

    def plain_leg(pts, q, kind, eps, theta, degree, leaf):
        qd = torch.from_numpy(q).cuda()
        tc = btk.Treecode(pts, degree=degree, cluster_size=leaf, theta=theta, eps=eps, kind=kind, device_tree=True)
        tc.solve(qd)
        ms = [event_ms(lambda: tc.solve(qd), flush)[0] for _ in range(steps)]
        o = tc.solve(qd).cpu().numpy()
        idx, ds = direct_check(tc, q, kind, eps=eps)
        r = {"ms": statistics.median(ms), "evaluations": tc.evals(), "rel_l2_vs_direct_10k": rel_l2(o[:, idx], ds)}
        tc.close()
        return r, idx, ds

    def mixed_leg(pts, q, kind, eps, theta, degree, leaf, idx, ds):
        qd = torch.from_numpy(q).cuda()
        tc = btk.Treecode(pts, degree=degree, cluster_size=leaf, theta=theta, eps=eps, kind=kind,
                          precision=btk.PREC_MIXED, device_tree=True)
        tc.solve(qd)
        ms = [event_ms(lambda: tc.solve(qd), flush)[0] for _ in range(steps)]
        o = tc.solve(qd).cpu().numpy()
        r = {"ms": statistics.median(ms), "evaluations": tc.evals(), "rel_l2_vs_direct_10k": rel_l2(o[:, idx], ds)}
        tc.close()
        return r

    def learned_leg(pts, q, kind, eps, theta, degree, leaf, idx, ds):
        qd = torch.from_numpy(q).cuda()
        sel = selector.Selector.load(kind=kind)
        tc = btk.Treecode(pts, degree=degree, cluster_size=leaf, theta=theta, eps=eps, kind=kind,
                          precision=btk.PREC_MIXED, degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4,
                          leaf_far_pairs=True, device_tree=True)
        cold_ms, (o, rep0) = event_ms(lambda: tc.solve_learned(qd, sel, tol=TOL), flush)
        for _ in range(2):
            tc.solve_learned(qd, sel, tol=TOL)
        ms = []
        for _ in range(steps):
            t, (o, rep) = event_ms(lambda: tc.solve_learned(qd, sel, tol=TOL), flush)
            ms.append(t)
        r = {"ms": statistics.median(ms), "cold_first_solve_ms": cold_ms, "cold_fell_back": rep0["fell_back"],
             "cold_audit_rel_l2": rep0["audit_rel_l2"], "audit_rel_l2": rep["audit_rel_l2"],
             "fell_back": rep["fell_back"], "pair_tol": rep["pair_tol"],
             "evaluations": rep["evals_near"] + rep["evals_far"],
             "rel_l2_vs_direct_10k": rel_l2(o.cpu().numpy()[:, idx], ds)}
        tc.close()
        return r

    pts, q = datagen.uniform_box(SEED, 65536, 2, -1.0, 1.0)
    r, _, _ = plain_leg(pts, q, btk.KIND_POT, EPS, 0.7, 8, 500)
    out["cfg1_2d_65k"] = {"workload": "2-D potential, N=65536 uniform [-1,1]^2, n=8, theta=0.7, leaf 500",
                          "plain_fp64": r}
    for key, what, gen, kind, eps, theta in (
            ("cfg4_plummer_4m", "3-D potential+gradient, N=4194304 Plummer sphere (a=0.1, r<=2), charges U[0,1], "
             "theta=0.7, leaf 2000, eps 1e-4", lambda: datagen.plummer(SEED, 1 << 22), btk.KIND_FIELD, 1e-4, 0.7),
            ("cfg5_sphere_2m_vel", "reference 3-D vector kernel, N=2097152 on the unit sphere, strengths U[-1,1], "
             "theta=0.8, leaf 2000, eps 1e-3", lambda: datagen.sphere_surface(SEED, 1 << 21), btk.KIND_VEL, 1e-3,
             0.8)):
        pts, q = gen()
        plain, idx, ds = plain_leg(pts, q, kind, eps, theta, 10, 2000)
        mixed = mixed_leg(pts, q, kind, eps, theta, 10, 2000, idx, ds)
        mixed["speedup_vs_plain_fp64"] = plain["ms"] / mixed["ms"]
        learned = learned_leg(pts, q, kind, eps, theta, 10, 2000, idx, ds)
        learned["speedup_vs_plain_fp64"] = plain["ms"] / learned["ms"]
        learned["cold_speedup_vs_plain_fp64"] = plain["ms"] / learned["cold_first_solve_ms"]
        # the learned solve's 1% FP64 direct-sum audit: N/100 targets x N sources
        learned["evaluations_fp64_audit"] = (len(q) // 100) * len(q)
        out[key] = {"workload": what, "plain_fp64_n10": plain, "mixed_n10": mixed, "learned_mixed": learned,
                    "tolerance_rel_l2": TOL}
    return out


def run_dropin(pts, q, flush, steps):
    """The reference-named call sequence of a solve (examples/
    example_poisson_3d.cpp:142-156: upward_pass_3d -> poisson_fmm_interactions_3d
    -> downward_pass_3d) through the drop-in entry points on device arrays in
    the reference's layouts, for the headline workload's potential (the drop-in
    interactions are the reference's potential kernel), against the plan path's
    plain FP64 potential solve. Each drop-in call synchronises its stream, as
    the reference's Kokkos calls fence; times are wall-clock around the three
    calls (after one warm-up sequence, which builds the cached plan state)."""
    import torch

    import barytreek_b200 as btk
    from barytreek_b200 import _lib
    L = _lib.load()
    cfg = btk.make_run_config(3, DEGREE, LEAF, THETA, EPS)
    tree = btk.tree_construction(cfg, pts)
    lists = btk.split_interactions(cfg, btk.dual_tree_traversal(cfg, tree))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    X = [dev(a) for a in pts]
    Q = dev(q)
    panels, leaf_of, inside = dev(tree.panels.view(np.uint8)), dev(tree.point_leaf_panel), dev(
        tree.panel_points_inside)
    Ld = [dev(l.view(np.uint8)) if len(l) else None for l in lists]
    n, P, ipc = len(q), tree.panel_count, cfg.interp_point_count
    ti = tree.tree_info()
    p = _lib.ptr
    psw = torch.empty((P, ipc), dtype=torch.float64, device="cuda")
    ptw = torch.empty((P, ipc), dtype=torch.float64, device="cuda")
    sol = torch.empty(n, dtype=torch.float64, device="cuda")

    def sequence():
        psw.zero_()
        ptw.zero_()
        sol.zero_()
        _lib.check(L.btk_upward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]), p(Q),
                                        p(panels), p(psw), p(leaf_of), n, None))
        _lib.check(L.btk_poisson_fmm_interactions_3d(
            ctypes.byref(cfg), p(X[0]), p(X[1]), p(X[2]), p(X[0]), p(X[1]), p(X[2]), p(Q), p(sol), p(inside),
            p(inside), p(psw), p(ptw), *[p(l) if l is not None else None for l in Ld], p(panels), p(panels), n, n,
            P, P, None))
        _lib.check(L.btk_downward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]), p(sol),
                                          p(panels), p(ptw), p(inside), n, None))

    t0 = time.perf_counter()
    sequence()
    torch.cuda.synchronize()
    first = time.perf_counter() - t0
    ms = []
    for _ in range(steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sequence()
        torch.cuda.synchronize()
        ms.append(1e3 * (time.perf_counter() - t0))
    out_dropin = sol.cpu().numpy()
    tc = btk.Treecode(pts, degree=DEGREE, cluster_size=LEAF, theta=THETA, eps=EPS, kind=btk.KIND_POT)
    tc.solve(Q)
    plan_ms = []
    for _ in range(steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = tc.solve(Q)
        torch.cuda.synchronize()
        plan_ms.append(1e3 * (time.perf_counter() - t0))
    agree = rel_l2(out_dropin, o.cpu().numpy()[0])
    tc.close()
    return {"workload": "3D Coulomb potential (the reference's potential path), N=%d, n=%d, theta=%g, leaf %d, "
                        "plain FP64" % (n, DEGREE, THETA, LEAF),
            "calls": "btk_upward_pass_3d -> btk_poisson_fmm_interactions_3d -> btk_downward_pass_3d",
            "ms_per_solve": statistics.median(ms), "first_call_ms": 1e3 * first,
            "plan_path_ms_per_solve": statistics.median(plan_ms),
            "ratio_to_plan_path": statistics.median(ms) / statistics.median(plan_ms),
            "rel_l2_vs_plan_path": agree}


def run_batch(args, flush):
    """The batched workload: 256 independent 3-D Coulomb potential problems,
    N log-uniform in [4096, 262144], Gaussian-mixture sources, N(0,1) charges,
    n = 6, theta = 0.6, mixed precision, leaf size and work split per size
    bucket from the autotuner's table; every solve is one captured graph."""
    import torch
    from barytreek_b200 import _lib, batch
    from barytreek_b200 import distributed as D
    L = _lib.load()
    world, rank = D.world_info()
    all_probs = batch.cfg3_problems(SEED, count=args.batch_problems)
    # one batch per rank: its size-balanced share of the problems (strong scaling)
    mine = D.shard_problems([len(p[1]) for p in all_probs], world)[rank]
    probs = [all_probs[b] for b in mine]
    coords = [p[0] for p in probs]
    q = np.ascontiguousarray(np.concatenate([p[1] for p in probs]))
    table = batch.Autotuner.load()
    t0 = time.time()
    b = batch.Batch(coords, degree=6, theta=0.6, eps=EPS, kind=0, table=table)
    setup = time.time() - t0
    qd = torch.from_numpy(q).cuda()
    out = torch.empty((1, b.n), dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        b.solve(qd, out)
    torch.cuda.synchronize()
    barrier(world)
    launches0 = L.btk_launch_count()
    ms = []
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            b.solve(qd, out)
            ms.append(b.stats()["last_ms"])
    torch.cuda.synchronize()
    launches = (L.btk_launch_count() - launches0) / args.steps
    st = b.stats()
    evals = D.reduce_over_ranks(b.evals(), "sum")
    # accuracy: 64 targets of every 16th problem against the FP64 direct sum over its own sources
    res = out.cpu().numpy()[0]
    err2 = ref2 = 0.0
    for i in range(0, len(probs), 16):
        pts, qi = probs[i]
        idx = np.linspace(0, len(qi) - 1, 64).astype(np.int64)
        t = [torch.from_numpy(np.ascontiguousarray(c[idx])).cuda() for c in pts]
        s_ = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in pts]
        o = torch.empty((1, len(idx)), dtype=torch.float64, device="cuda")
        _lib.check(L.btk_direct_sum(3, 0, EPS, len(idx), _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), len(qi),
                                    _lib.ptr(s_[0]), _lib.ptr(s_[1]), _lib.ptr(s_[2]),
                                    _lib.ptr(torch.from_numpy(qi).cuda()), _lib.ptr(o), None))
        d = o.cpu().numpy()[0]
        err2 += float(np.sum((res[b.offsets[i] + idx] - d) ** 2))
        ref2 += float(np.sum(d ** 2))
    err2, ref2 = D.reduce_over_ranks(err2, "sum"), D.reduce_over_ranks(ref2, "sum")
    m = D.reduce_over_ranks(sum(ms), "max") / len(ms)  # device time, max over ranks
    out_line = {
        "workload": f"{len(all_probs)} independent 3-D Coulomb potential problems, N log-uniform in [4096, 262144], "
                    "Gaussian mixtures of 1-8 components (sigma 0.02-0.2) in the unit cube, N(0,1) charges, "
                    "n=6, theta=0.6, mixed FP32/FP64",
        "problems": len(all_probs), "points": int(sum(len(p[1]) for p in all_probs)), "ms_per_step": m,
        "scaling": "strong", "sharding": f"problems split over {world} rank(s) by point count",
        "value": evals / (m * 1e-3), "unit": "interactions/s", "evaluations": evals,
        "graph_kernel_nodes": st["graph_kernel_nodes"], "graph_nodes": st["graph_nodes"],
        "graph_launches_per_step": 1, "kernel_launches_per_step": launches, "work_items": st["work_items"],
        "levels": st["levels"], "panels": st["panel_count"], "setup_s": setup,
        "leaf_size_by_bucket": {f"2^{k}": v[0] for k, v in sorted(table.table.items())},
        "work_split": b.work_split, "tile_targets": b.tile_targets or 256,
        "rel_l2_vs_direct_sampled": (err2 / ref2) ** 0.5 if ref2 > 0 else None,
        "clocks": clk.summary(),
    }
    b.close()
    return out_line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--kind", type=int, default=2, choices=[0, 2])
    ap.add_argument("--form", default="learned", choices=["plain", "mixed", "learned"],
                    help="the form reported as the headline (all cheaper forms are timed beside it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-problems measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations (1, 4, 5)")
    ap.add_argument("--forms", default="", help="comma list of the forms to time beside the headline (profiling)")
    ap.add_argument("--batch-only", action="store_true", help="only the batched-problems measurement (profiling)")
    ap.add_argument("--batch-problems", type=int, default=256, help="problems in the batch (profiling captures)")
    ap.add_argument("--points", type=int, default=N_POINTS, help="point count (profiling captures only)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    globals()["N_POINTS"] = args.points
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup(args.gpus)
        if args.batch_only:
            import torch
            line = run_batch(args, torch.empty(32 << 20, dtype=torch.float64, device="cuda"))
            line = line if rank == 0 else None
        else:
            line = run_native(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
