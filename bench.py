"""Benchmark of the B200 DG SN sweep (one JSON line on rank 0).

A step is one transport sweep over the whole workload: every (cell, angle,
group) of the 196,608-tet S8 G=8 Kuhn-cube workload (32^3 hexes x 6 tets,
+-0.05h jitter, lognormal sigma_t, downscatter, box source) updated once,
phi_out = D L^-1 (Q + M S phi_in).  `value` is the mixed-precision (FP32)
sweep's updates/s with inputs resident in HBM; the FP64 sweep is reported
beside it, with the phi error of the mixed-precision solve against the FP64
solve.  `e2e` is the drop-in SweeperAbstract::sweep(psi, source) through the
C ABI with host buffers (psi-sized source in, psi out, copies timed).

Two more legs ride on the same line (skip with --no-batch / --no-serve):
`batch`, 256 uneven independent instances solved together (FP64 source
iteration vs FP32-sweep iteration inside FP64 refinement, one batched pass
per step), and `serve`, Poisson-arriving solve requests (the batch size
distribution plus 5% large 48^3-hex S8 G=8 ones) admitted by device-memory
footprint against 150 GB with continuous batching, at a swept arrival rate:
p50/p99 latency, solves/s and requests in the batch of the mixed and the
FP64 service; and `large`, the 64^3 x 6-tet
S8 G=16 problem (psi 103 GB): sweep rates and the mixed-precision GMRES solve
against FP64 GMRES (skip with --no-large).

Multi-GPU: the sweep does not shard across GPUs here (one mesh partition per
GPU by design); --gpus N runs N independent replicas, one per rank, and
reports the sum of their throughputs with the max-over-ranks time.

--impl reference times the reference's own CPU sweep (SweeperTraverse::sweep
compiled from its sources, oracle/_ref/ref_dump.x) on the host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sweep cell*dir*grp updates/s (mixed-precision FP32 sweep, FP64 refinement)"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
NOMINAL_HBM_GBS = 7700.0  # B200 HBM3e, HGX figure


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="kuhn32_s8_g8")
    p.add_argument("--no-solve", action="store_true", help="skip the solve-error check")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-large", action="store_true", help="skip the 64^3 S8 G=16 leg")
    p.add_argument("--no-batch", action="store_true", help="skip the batched-instances leg")
    p.add_argument("--batch-instances", type=int, default=256)
    p.add_argument("--no-serve", action="store_true", help="skip the served-solves leg")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the oracle checks of the benchmarked solves (run after the timed legs)")
    p.add_argument("--serve-requests", type=int, default=400, help="requests per arrival rate")
    p.add_argument("--serve-rates", default="20,50,100,200",
                   help="Poisson arrival rates (requests per second), comma-separated")
    p.add_argument("--shape", default="default",
                   help="launch shape 'schedule,variant,knob[,vector[,streams]]' for both precisions "
                        "(an FP32-only vector width falls back to the widest for FP64, an FP32-only knob "
                        "to -96), default (the sweeper's own: FP32 slotted compact records, FP64 compact "
                        "records, 2 octant streams; the autotuner's pick on this workload), or auto "
                        "(run the autotuner first)")
    p.add_argument("--profile-leg", default="main", choices=["main", "batch"],
                   help="what cudaProfilerStart/Stop bracket (for ncu --profile-from-start off): the main "
                        "leg's timed steps, or steps 4-6 of each batched solve")
    return p.parse_args()


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []  # (arrival time, line)
        self.window = [None, None]

    def start(self):
        """The timed region begins: only samples from here on count."""
        self.window[0] = time.monotonic()

    def stop(self):
        self.window[1] = time.monotonic()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            time.sleep(0.5)  # sampling is running before the timed region starts
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0 = self.window[0] if self.window[0] is not None else -1e300
        t1 = self.window[1] if self.window[1] is not None else 1e300
        for t, ln in self.lines:
            if not (t0 <= t <= t1 + 0.06):  # a sample arrives up to one period late
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(nc, A, G, n_in, s):
    """Per sweep: s*G*sum_(c,a)(4 + 3 n_in) + Nc*4*G*(8+8) + Nc*208 bytes.
    psi write (4 nodal values) and upwind reads (3 per incoming interior face)
    in the sweep precision, FP64 phi in and out, per-cell geometry and tables."""
    return s * G * (4 * nc * A + 3 * n_in) + nc * 4 * G * 16 + nc * 208


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def build_problem(name):
    from tycho2_b200 import problems
    w = dict(problems.WORKLOADS[name])
    mesh, st, ss, mat, q = problems.make_problem(**w)
    return w, mesh, st, ss, mat, q


REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def reference_inputs(workload, d):
    """The workload's files for the reference, made without the product
    library: a .smesh from oracle/kuhn_problem.py, turned into the .pmesh the
    reference's TychoMesh reads by the reference's own PartitionColumns (one
    partition), and sigma_t / q as raw f64."""
    from oracle import kuhn_problem as kp
    mesh, st, q, w = kp.make_workload(workload)
    pmesh = kp.partition(mesh, d, "m", os.path.join(REF_BIN, "PartitionColumns.x"))
    st_f, q_f = os.path.join(d, "st.f64"), os.path.join(d, "q.f64")
    np.ascontiguousarray(st).tofile(st_f)
    np.ascontiguousarray(q).tofile(q_f)
    return {"pmesh": pmesh, "st": st_f, "q": q_f, "sn": w["sn"], "groups": w["groups"],
            "cells": int(mesh[0].shape[0])}


def reference_sweep(inp, steps=1, warmup=0, phi_path=None):
    """Times the reference's own SweeperTraverse::sweep (oracle/_ref/ref_dump.x
    bench) on every host core it can use: seconds per sweep, thread count and
    the hash of the last psi's bytes."""
    ncpu = os.cpu_count() or 1
    A = 2 * inp["sn"] ** 2
    # one thread per core, each bound to its core (the reference parallelises
    # over angle groups with OpenMP)
    env = dict(os.environ, OMP_NUM_THREADS=str(min(ncpu, A)))
    env.setdefault("OMP_PROC_BIND", "close")
    env.setdefault("OMP_PLACES", "cores")
    cmd = [os.path.join(REF_BIN, "ref_dump.x"), "bench", inp["pmesh"], str(inp["sn"]), str(inp["groups"]),
           inp["st"], inp["q"], str(steps), str(warmup)] + ([phi_path] if phi_path else [])
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("REFBENCH ")]
    if r.returncode != 0 or not line:
        raise RuntimeError("reference bench failed: %s" % r.stderr[-500:])
    return json.loads(line[0][len("REFBENCH "):])


def psi_hash(psi, chunk=1 << 25):
    """The hash ref_dump.x prints for a psi array: its 64-bit words x_i summed
    as x_i * (2i + 1) modulo 2^64 (equal hashes: equal bits, up to 2^-64)."""
    words = np.ascontiguousarray(psi).reshape(-1).view(np.uint64)
    h = np.uint64(0)
    with np.errstate(over="ignore"):
        for k in range(0, words.size, chunk):
            idx = np.arange(k, min(k + chunk, words.size), dtype=np.uint64)
            h = h + np.sum(words[k:k + idx.size] * (idx * np.uint64(2) + np.uint64(1)), dtype=np.uint64)
    return "%016x" % int(h)


def cpu_baseline(workload, steps=1, warmup=0):
    """Times the reference's own CPU sweep (oracle/_ref) on all host cores, one
    full sweep of the workload; falls back to the oracle restatement (on a
    mesh the product writes) where the reference was not built."""
    with tempfile.TemporaryDirectory() as d:
        if os.path.exists(os.path.join(REF_BIN, "ref_dump.x")):
            inp = reference_inputs(workload, d)
            res = reference_sweep(inp, steps, warmup)
            upd = inp["cells"] * 2 * inp["sn"] ** 2 * inp["groups"]
            return {"value": upd / res["seconds_per_sweep"], "unit": "updates/s", "cores": res["threads"],
                    "kind": "reference",
                    "sample": "%d full sweep(s) of the workload, SweeperTraverse::sweep" % steps,
                    "build": "g++ -O3 -fopenmp -ffp-contract=off (oracle/Makefile)",
                    "seconds_per_sweep": res["seconds_per_sweep"], "psi_hash": res["psi_hash"]}
        from oracle.oracle import Oracle, OracleMesh
        w, mesh, st, ss, mat, q = build_problem(workload)
        pm = os.path.join(d, "m.pmesh")
        mesh.write_pmesh(pm)
        G = w["groups"]
        o = Oracle(OracleMesh(pm), w["sn"], G)
        t0 = time.perf_counter()
        for _ in range(steps):
            psi = o.sweep(st, src_iso=np.ascontiguousarray(q))
        dt = (time.perf_counter() - t0) / steps
        return {"value": mesh.n_cells * 2 * w["sn"] ** 2 * G / dt, "unit": "updates/s",
                "cores": os.cpu_count() or 1, "kind": "port",
                "sample": "%d full sweep(s) of the workload, oracle restatement" % steps,
                "seconds_per_sweep": dt, "psi_hash": psi_hash(psi)}


def oracle_phi(params, d, name, restart=20, rtol=1e-12, iter_max=600):
    """The oracle's converged phi of one problem (its GMRES(restart), to a
    2-norm residual of rtol relative to the right-hand side), on a mesh and
    inputs written without the product library where the reference's
    PartitionColumns was built.  Returns (phi, iterations, seconds)."""
    from oracle import kuhn_problem as kp
    from oracle.oracle import Oracle, OracleMesh
    mesh, st, ss, mat, q = kp.make_problem(**params)
    pc = os.path.join(REF_BIN, "PartitionColumns.x")
    if os.path.exists(pc):
        pm = kp.partition(mesh, d, name, pc)
    else:
        from tycho2_b200 import problems
        pm = os.path.join(d, name + ".pmesh")
        problems.make_problem(**params)[0].write_pmesh(pm)
    t0 = time.perf_counter()
    o = Oracle(OracleMesh(pm), params["sn"], params["groups"])
    _, phi, it, _ = o.krylov(st, ss, scatter=mat, q_iso=np.ascontiguousarray(q), restart=restart,
                             iter_max=iter_max, rtol=rtol)
    return phi, it, time.perf_counter() - t0


def rel_l1(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).sum() / np.abs(np.asarray(b)).sum())


def parity_c1(dev):
    """The 3,072-tet S4 G=1 problem: FP64 source iteration on the GPU against
    the oracle's (same criterion, 1e-10 relative change: bit-identical
    expected) and the mixed solve against the oracle's converged phi."""
    import tycho2_b200 as ty
    from oracle import kuhn_problem as kp
    from oracle.oracle import Oracle, OracleMesh
    w = dict(kp.WORKLOADS["kuhn8_s4_g1"])
    mesh, st, ss, mat, q = ty.problems.make_problem(**w)
    sw = ty.SweeperCuda(mesh, w["sn"], w["groups"], fp32=True, device=dev)
    sw.set_cross_sections(st, ss, mat)
    sw.set_source(q, "isotropic")
    phi64, _, s64 = sw.solve("si", iter_max=2000, err_max=1e-10, want_psi=False)
    phim, _, sm = sw.solve("mixed", iter_max=500, err_max=1e-10, want_psi=False)
    sw.close()
    with tempfile.TemporaryDirectory() as d:
        pm = os.path.join(d, "c1.pmesh")
        mesh.write_pmesh(pm)
        o = Oracle(OracleMesh(pm), w["sn"], w["groups"])
        _, phi_o, it_o, _ = o.source_iteration(st, ss, scatter=mat, q_iso=np.ascontiguousarray(q),
                                               iter_max=2000, err_max=1e-10)
        phi_k, _, _ = oracle_phi(w, d, "c1k", rtol=1e-13)
    return {"workload": "kuhn8_s4_g1",
            "fp64_si_bitexact_vs_oracle_si": bool(np.array_equal(phi64.view(np.uint64), phi_o.view(np.uint64))),
            "fp64_si_phi_rel_l1_vs_oracle_si": rel_l1(phi64, phi_o),
            "fp64_si_iterations": s64["iterations"], "oracle_si_iterations": it_o,
            "fp64_si_phi_rel_l1_vs_oracle_converged": rel_l1(phi64, phi_k),
            "mixed_phi_rel_l1_vs_oracle_converged": rel_l1(phim, phi_k)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    res = cpu_baseline(args.workload, steps=steps, warmup=min(args.warmup, 1))
    v = res["value"]
    from oracle import kuhn_problem as kp
    w = kp.WORKLOADS[args.workload]
    nc, A, G = 6 * w["n"] ** 3, 2 * w["sn"] ** 2, w["groups"]
    line = {"metric": METRIC, "value": v, "unit": "updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": res["seconds_per_sweep"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "cells": nc, "angles": A, "groups": G},
            "cpu_baseline": res,
            "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


KERNELS = {
    (1, "items"): "sweep_level_kernel<{r},{k}>", (1, "tiles"): "sweep_tile_level_kernel<{r},{k}>",
    (1, "records"): "sweep_record_level_kernel<{r},{k},{vg}>",
    (2, "items"): "sweep_dataflow_kernel<{r},{k}>", (2, "tiles"): "sweep_tile_dataflow_kernel<{r},{k}>",
    (2, "records"): "sweep_record_dataflow_kernel<{r},{k},{vg}>",
    (3, "records"): "sweep_record_persist_kernel<{r},{k},{vg}>",
    (1, "direct"): "sweep_direct_level_kernel<{r},{vg},{k}>",
    (1, "compact"): "sweep_direct_level_kernel<{r},{vg},{k},compact>",
}
SCHED = {"levels": 1, "dataflow": 2, "persist": 3}


# FP32 slotted upwind rows: knob -> (threads per block, blocks per SM)
SLOT_KNOBS = {-196: (64, 10), -180: (64, 12), -172: (64, 14)}


def kernel_name(shape, fp32):
    if shape["knob"] in SLOT_KNOBS and shape["variant"] in ("direct", "compact"):
        bs, minb = SLOT_KNOBS[shape["knob"]]
        return "sweep_direct_slot_kernel<{vg},{bs},{rec},{m}>".format(
            vg=shape["vector"], bs=bs, rec="compact" if shape["variant"] == "compact" else "full", m=minb)
    return KERNELS[(SCHED[shape["schedule"]], shape["variant"])].format(
        r="float" if fp32 else "double", k=shape["knob"], vg=shape["vector"])


def traffic_family(shape, fp32):
    """What a sweep's DRAM traffic depends on: variant, precision, group vector."""
    return "%s %s vg%d" % (shape["variant"], "float" if fp32 else "double", shape["vector"])


TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of 3 mid-sweep launches of the kernel on "
                  "kuhn24_s8_g8 (warm caches), per item, times this sweep's items: profiles/sweep_traffic.md; "
                  "not measured in this run")


def profiled_traffic(workload, family):
    """DRAM bytes of one sweep from the ncu summary table in profiles/ (three
    sampled launches of the kernel, bytes per item scaled to the sweep's
    items), if that kernel family was captured for this workload; else None."""
    path = os.path.join(ROOT, "profiles", "sweep_traffic.md")
    try:
        with open(path) as f:
            for ln in f:
                cells = [c.strip() for c in ln.strip().strip("|").split("|")]
                if len(cells) >= 3 and cells[0] == workload and cells[1] == "`%s`" % family:
                    return float(cells[2])
    except (OSError, ValueError):
        pass
    return None


def batch_sample(params, k=8, seed=17):
    """Indices of the batch members checked against the oracle: the member
    with the most updates per sweep and k - 1 others drawn with a seed."""
    cost = [6 * p["n"] ** 3 * 2 * p["sn"] ** 2 * p["groups"] for p in params]
    big = int(np.argmax(cost))
    rest = [i for i in range(len(params)) if i != big]
    pick = np.random.default_rng(seed).choice(rest, size=min(k - 1, len(rest)), replace=False)
    return [big] + sorted(int(i) for i in pick)


def run_batch_leg(grp, dev, count, seed=4321, profile=False, sample=None):
    """Batched uneven instances: `count` problems (n ~ U{4..24}, G ~ U{1,2,4,8},
    S ~ U{4,6,8}, sigma_t ~ lognormal(0, 0.5), c ~ U[0.3, 0.95], q = 1, all
    seeded) solved together, FP64 source iteration vs FP32-sweep source
    iteration inside FP64 refinement, both to 1e-10 relative change."""
    import torch
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    t0 = time.perf_counter()
    sws, upd = [], 0
    params = problems.batch_instances(count, seed=seed + 7919 * grp.rank)
    for p in params:
        mesh, st, ss, mat, q = problems.make_problem(**p)
        sw = ty.SweeperCuda(mesh, p["sn"], p["groups"], fp32=True, device=dev)
        sw.set_cross_sections(st, ss, mat)
        sw.set_source(q, "isotropic")
        sws.append(sw)
        upd += mesh.n_cells * 2 * p["sn"] ** 2 * p["groups"]
    setup = time.perf_counter() - t0
    # the project's autotuner picks the batch's kernel shapes for these members
    t0 = time.perf_counter()
    tuned, tune_table = ty.BatchSolver.autotune(sws, device=dev)
    tune_s = time.perf_counter() - t0
    out, phis = {}, {}
    for method in ("si", "mixed", "si_other", "mixed_other"):
        if method.endswith("_other"):  # the form the autotuner did not pick, for comparison
            shape = {"ipw32": 0, "ipw64": 0, "persistent": not tuned["persistent"]}
        else:
            shape = tuned
        b = ty.BatchSolver(device=dev, **shape)
        method_name = method.split("_")[0]
        ids = [b.add(sw, method_name, err_max=1e-10, iter_max=5000, inner_tol=1e-5) for sw in sws]
        grp.barrier()
        t = time.perf_counter()
        steps = 0
        while True:
            if profile and steps == 3:
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            active = b.step()
            if profile and steps == 5:
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
            if active <= 0:
                break
            steps += 1
        wall = grp.max(time.perf_counter() - t)
        tm = b.timing()
        res = [b.result(i) for i in ids]
        phis[method] = [r[0] for r in res]
        swept = tm["fp64_updates"] + tm["fp32_updates"]
        out[method] = {
            "solve_wall_s": wall, "steps": steps, "updates_swept": swept,
            "solve_updates_per_s": grp.sum(swept) / wall,
            "fp64_pass_updates_per_s": tm["fp64_updates"] / (tm["fp64_ms"] * 1e-3) if tm["fp64_ms"] else None,
            "fp32_pass_updates_per_s": tm["fp32_updates"] / (tm["fp32_ms"] * 1e-3) if tm["fp32_ms"] else None,
            "sweeps_fp64": sum(r[1]["sweeps_fp64"] for r in res),
            "sweeps_fp32": sum(r[1]["sweeps_fp32"] for r in res),
            "all_converged": all(r[1]["final_error"] <= 1e-10 for r in res)}
        b.close()
    err = [float(np.abs(m - f).sum() / np.abs(f).sum()) for m, f in zip(phis["mixed"], phis["si"])]
    same = all(np.array_equal(a.view(np.uint64), b.view(np.uint64))
               for k in ("si", "mixed") for a, b in zip(phis[k], phis[k + "_other"]))
    for sw in sws:
        sw.close()
    if sample is not None:  # the members the oracle checks after the timed legs
        for i in batch_sample(params):
            sample.append((i, params[i], phis["si"][i], phis["mixed"][i]))
    return {"instances": count * grp.world, "updates_per_sweep": upd, "setup_s": setup,
            "kernel": ("batch_persist_kernel" if tuned["persistent"] else "batch_direct_level_kernel")
                      + (" (compact records)" if tuned["ipw32"] == 0 else " (ipw %d)" % tuned["ipw32"]),
            "fp64_si": out["si"], "mixed": out["mixed"],
            "autotune": {"pick": tuned, "seconds": tune_s, "table": tune_table},
            "other_form": {"form": ("one launch per level" if tuned["persistent"] else
                                    "one persistent kernel per pass, device work queue over (member, level), "
                                    "bounded grid barrier between levels") + " (the form the autotuner did not pick)",
                           "fp64_si_solve_wall_s": out["si_other"]["solve_wall_s"],
                           "mixed_solve_wall_s": out["mixed_other"]["solve_wall_s"],
                           "fp64_pass_updates_per_s": out["si_other"]["fp64_pass_updates_per_s"],
                           "fp32_pass_updates_per_s": out["mixed_other"]["fp32_pass_updates_per_s"],
                           "bit_identical_to_the_pick": same},
            "phi_rel_err_l1_max_mixed_vs_fp64": grp.max(max(err)),
            "mixed_vs_fp64_solve_speedup": out["si"]["solve_wall_s"] / out["mixed"]["solve_wall_s"],
            "mixed_vs_fp64_pass_speedup": (out["mixed"]["fp32_pass_updates_per_s"]
                                           / out["si"]["fp64_pass_updates_per_s"])}


def run_serve_leg(grp, dev, count, rates, seed=99):
    """Served solves at a swept arrival rate: `count` requests drawn like the
    batch instances plus 5% large ones (48^3 hexes x 6 tets, G=8, S8), the
    same requests at each Poisson rate (the arrival gaps of one seeded
    exponential draw, scaled by 1/rate), admitted by footprint against 150
    GB, mixed vs FP64 service: p50/p99 latency, solves/s, mean and peak
    requests in the batch."""
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    rng = np.random.default_rng(seed + grp.rank)
    params = problems.batch_instances(count, seed=seed + 31 * grp.rank)
    for k in range(count):
        if rng.random() < 0.05:
            params[k] = dict(n=48, jitter=0.05, sn=8, groups=8, sigma="lognormal", lognormal_s=0.5,
                             ratio=0.6, scatter="down", source="all", seed=5000 + k)
    probs = [problems.make_problem(**p) for p in params]
    unit_gaps = rng.exponential(1.0, count)
    out = {"requests": count * grp.world, "large": int(sum(p["n"] == 48 for p in params)),
           "budget_gb": 150.0, "rates": []}
    worst = 0.0
    for rate in rates:
        arrivals = (np.cumsum(unit_gaps) - unit_gaps[0]) / rate
        entry = {"rate_per_s": rate * grp.world}
        phis = {}
        for method, key in (("mixed", "mixed"), ("si", "fp64")):
            srv = ty.SolveServer(method=method, budget_bytes=150e9, device=dev, setup_threads=4, err_max=1e-10,
                                 inner_tol=1e-5)
            ids = [srv.submit(m, p["sn"], p["groups"], st, ss, mat, q, arrival=float(a))
                   for p, (m, st, ss, mat, q), a in zip(params, probs, arrivals)]
            grp.barrier()
            srv.run()
            info = [srv.info(i) for i in ids]
            done = [i for i in info if i["state"] == "done"]
            lat = np.array([i["latency"] for i in done])
            st_ = srv.stats()
            phis[key] = [srv.phi(i).copy() for i in ids]
            span = max(st_["makespan"], 1e-9)
            entry[key] = {"done": len(done), "p50_latency_s": grp.max(float(np.percentile(lat, 50))),
                          "p99_latency_s": grp.max(float(np.percentile(lat, 99))),
                          "solves_per_s": grp.sum(len(done)) / grp.max(st_["makespan"]),
                          "build_p50_s": float(np.percentile([i["built"] - i["admitted"] for i in done], 50)),
                          "mean_in_batch": float(sum(i["finished"] - i["built"] for i in done) / span),
                          "peak_in_batch": st_["peak_active"],
                          "peak_resident_gb": st_["peak_bytes"] / 1e9, "batch_steps": st_["steps"]}
            big = [i for p, i in zip(params, info) if p["n"] == 48 and i["state"] == "done"]
            if big:  # where the large requests' latency goes
                entry[key]["large_p50_latency_s"] = float(np.percentile([i["latency"] for i in big], 50))
            srv.close()
        entry["phi_rel_err_l1_max_mixed_vs_fp64"] = grp.max(max(
            float(np.abs(a - b).sum() / np.abs(b).sum()) for a, b in zip(phis["mixed"], phis["fp64"])))
        worst = max(worst, entry["phi_rel_err_l1_max_mixed_vs_fp64"])
        out["rates"].append(entry)
    out["phi_rel_err_l1_max_mixed_vs_fp64"] = worst
    return out


def run_large_leg(grp, dev, workload="kuhn64_s8_g16"):
    """The 64^3 x 6 = 1,572,864-tet S8 G=16 problem (lognormal(0, 1) sigma_t,
    scattering ratio 0.99): FP32 and FP64 sweep rates, then the
    mixed-precision solve (FP32-sweep GMRES(30) in FP64 refinement) against
    FP64 GMRES(30), both to 1e-10.  psi alone is 103 GB (FP64-sized), so both
    precisions sweep with compact records (the record-free warp-tile kernel
    for FP64 if those do not fit)."""
    import tycho2_b200 as ty
    w, mesh, st, ss, mat, q = build_problem(workload)
    nc, A, G = mesh.n_cells, 2 * w["sn"] ** 2, w["groups"]
    t0 = time.perf_counter()
    sw = ty.SweeperCuda(mesh, w["sn"], G, fp32=True, device=dev)
    sw.set_cross_sections(st, ss, mat)
    sw.set_source(q, "isotropic")
    setup = time.perf_counter() - t0
    info = sw.schedule_info()
    sw.configure(1, "levels", "compact", -180, 4, 2)  # the fastest slotted FP32 shape here (the autotuner's pick)
    try:  # compact FP64 records (19 GB) fit beside psi (103 GB) and the GMRES(30) basis
        sw.configure(0, "levels", "compact", -96, 2, 2)
    except ty.TychoError:
        sw.configure(0, "levels", "tiles", 4)
    sw.time_sweeps(1, 2)
    sw.time_sweeps(0, 2)
    grp.barrier()
    ms32, k32 = sw.time_sweeps(1, 3, True)
    ms64, k64 = sw.time_sweeps(0, 3, True)
    ms32, k32, ms64, k64 = (grp.max(x) for x in (ms32, k32, ms64, k64))
    upd = nc * A * G
    peak, peak_kind = hbm_peak()
    b32 = algorithmic_bytes(nc, A, G, info["n_incoming_interior"], 4)
    b64 = algorithmic_bytes(nc, A, G, info["n_incoming_interior"], 8)
    sw_shape32, sw_shape64 = sw.shape(1), sw.shape(0)
    tol, m = w.get("tol", 1e-10), w.get("restart", 30)
    phim, _, sm = sw.solve("mixed", iter_max=600, err_max=tol, restart=m, want_psi=False)
    phi64, _, s64 = sw.solve("gmres", iter_max=600, err_max=tol, restart=m, want_psi=False)
    err = float(np.abs(phim - phi64).sum() / np.abs(phi64).sum())
    sw.close()
    return {"workload": workload, "cells": nc, "angles": A, "groups": G, "levels": info["n_levels"],
            "setup_s": setup,
            "fp32": {"updates_per_s": grp.sum(upd) / (ms32 * 1e-3), "ms_per_sweep": ms32,
                     "kernel": kernel_name(sw_shape32, True), "shape": sw_shape32, "kernel_ms": k32,
                     "roofline_frac": b32 / (k32 * 1e-3) / 1e9 / peak, "peak_kind": peak_kind},
            "fp64": {"updates_per_s": grp.sum(upd) / (ms64 * 1e-3), "ms_per_sweep": ms64,
                     "kernel": kernel_name(sw_shape64, False), "shape": sw_shape64, "kernel_ms": k64,
                     "roofline_frac": b64 / (k64 * 1e-3) / 1e9 / peak},
            "mixed_solve": {"seconds": sm["seconds"], "sweeps_fp32": sm["sweeps_fp32"],
                            "sweeps_fp64": sm["sweeps_fp64"], "residual": sm["final_error"]},
            "fp64_gmres_solve": {"seconds": s64["seconds"], "sweeps_fp64": s64["sweeps_fp64"],
                                 "residual": s64["final_error"]},
            "phi_rel_err_l1_mixed_vs_fp64": grp.max(err),
            "mixed_vs_fp64_solve_speedup": s64["seconds"] / sm["seconds"]}


def run_parity(args, dev, cpu, gpu_psi_hash, phi_c2, sample, large, serve):
    """Checks of the benchmarked solves against the reference and the oracle,
    after the timed legs (relative L1 norms, the reference's diff.py norm):
    c1 the 3,072-tet problem; c2 the benchmark workload: the FP64 sweep's psi
    bits against the reference's own SweeperTraverse::sweep (hash of psi from
    ref_dump.x) and the FP64-GMRES and mixed phi against the oracle's GMRES
    to 1e-12; c3 the 64^3 problem's mixed phi against the FP64 GPU GMRES (its
    FP64 oracle does not fit host memory); c4 a seeded sample of the batch
    members (the largest included), FP64 source iteration and mixed phi
    against the oracle's GMRES to 1e-12; c5 the mixed service against the
    FP64 service."""
    out = {"norm": "relative L1", "tolerances": {"fp64_sweep": "bit-identical", "mixed_phi": 1e-8}}
    try:
        out["c1"] = parity_c1(dev)
    except Exception as e:
        out["c1"] = {"error": str(e)[:200]}
    c2 = {"workload": args.workload}
    if gpu_psi_hash and cpu and cpu.get("psi_hash"):
        c2["fp64_sweep_bitexact_vs_reference"] = gpu_psi_hash == cpu["psi_hash"]
        c2["psi_hash"] = {"gpu": gpu_psi_hash, "reference": cpu["psi_hash"]}
    if phi_c2:
        try:
            from oracle import kuhn_problem as kp
            with tempfile.TemporaryDirectory() as d:
                w = dict(kp.WORKLOADS[args.workload])
                phi_o, it, sec = oracle_phi(w, d, "c2", restart=20, rtol=1e-12)
            c2.update({"oracle_gmres_iterations": it, "oracle_seconds": sec,
                       "fp64_gmres_phi_rel_l1_vs_oracle": rel_l1(phi_c2["fp64_gmres"], phi_o),
                       "mixed_phi_rel_l1_vs_oracle": rel_l1(phi_c2["mixed"], phi_o)})
        except Exception as e:
            c2["error"] = str(e)[:200]
    out["c2"] = c2
    if large and "phi_rel_err_l1_mixed_vs_fp64" in large:
        out["c3"] = {"workload": large["workload"], "mixed_phi_rel_l1_vs_fp64_gpu": large["phi_rel_err_l1_mixed_vs_fp64"]}
    if sample:
        members, e64, emx = [], [], []
        try:
            with tempfile.TemporaryDirectory() as d:
                for i, p, phi64, phim in sample:
                    phi_o, it, sec = oracle_phi(p, d, "m%d" % i, restart=30, rtol=1e-12)
                    members.append({"index": i, "n": p["n"], "sn": p["sn"], "groups": p["groups"],
                                    "ratio": p["ratio"], "oracle_seconds": sec,
                                    "fp64_si": rel_l1(phi64, phi_o), "mixed": rel_l1(phim, phi_o)})
                    e64.append(members[-1]["fp64_si"])
                    emx.append(members[-1]["mixed"])
            out["c4"] = {"members": members, "fp64_si_max_rel_l1_vs_oracle": max(e64),
                         "mixed_max_rel_l1_vs_oracle": max(emx)}
        except Exception as e:
            out["c4"] = {"members": members, "error": str(e)[:200]}
    if serve and "phi_rel_err_l1_max_mixed_vs_fp64" in serve:
        out["c5"] = {"mixed_phi_rel_l1_max_vs_fp64_service": serve["phi_rel_err_l1_max_mixed_vs_fp64"]}
    return out


def run_b200(args):
    import torch
    import tycho2_b200 as ty
    from tycho2_b200.replicas import ReplicaGroup

    grp = ReplicaGroup()
    world, rank, dev = grp.world, grp.rank, grp.device

    w, mesh, st, ss, mat, q = build_problem(args.workload)
    nc, A, G = mesh.n_cells, 2 * w["sn"] ** 2, w["groups"]
    updates = nc * A * G
    sw = ty.SweeperCuda(mesh, w["sn"], G, fp32=True, device=dev)
    sw.set_cross_sections(st, ss, mat)
    sw.set_source(q, "isotropic")
    info = sw.schedule_info()

    # Launch shapes: the sweeper's defaults, the autotuner's pick per
    # precision, or a fixed shape.
    if args.shape == "auto":
        tuned = {1: sw.autotune(1, 5), 0: sw.autotune(0, 5)}
    elif args.shape == "default":
        tuned = {1: sw.shape(1), 0: sw.shape(0)}
    else:
        parts = args.shape.split(",")
        s, v, k = parts[:3]
        vec = int(parts[3]) if len(parts) > 3 else 0
        streams = int(parts[4]) if len(parts) > 4 else 1
        for prec in (1, 0):
            # FP32-only knobs (slotted upwind rows) fall back to -96 for FP64
            pk = -96 if prec == 0 and int(k) in SLOT_KNOBS else int(k)
            sw.configure(prec, s, v, pk, vec if (prec == 1 or vec <= 2) else 0, streams)
        tuned = {1: sw.shape(1), 0: sw.shape(0)}
    shape32, shape64 = sw.shape(1), sw.shape(0)
    launches = {1: sw.launches(1), 0: sw.launches(0)}

    # Untimed warm-up (graph capture of both precisions), then K timed steps
    # of each precision.  psi (6.4 GB FP64 / 3.2 GB FP32) is far larger than
    # L2; a 256 MB buffer is also written between steps.
    warm = max(args.warmup, 3)
    sw.time_sweeps(1, warm)
    sw.time_sweeps(0, warm)

    with Clocks(dev) as clk:
        grp.barrier()
        if args.profile_leg == "main":
            torch.cuda.profiler.start()  # ncu --profile-from-start off captures the timed steps only
        clk.start()
        t0 = time.perf_counter()
        ms32, lvl32 = sw.time_sweeps(1, args.steps, True)
        grp.barrier()
        wall32 = time.perf_counter() - t0
        ms64, lvl64 = sw.time_sweeps(0, args.steps, True)
        grp.barrier()
        clk.stop()
        if args.profile_leg == "main":
            torch.cuda.profiler.stop()
    clocks = clk.summary()

    ms32, lvl32, ms64, lvl64 = (grp.max(x) for x in (ms32, lvl32, ms64, lvl64))
    value = grp.sum(updates) / (ms32 * 1e-3)
    fp64_value = grp.sum(updates) / (ms64 * 1e-3)

    peak, peak_kind = hbm_peak()
    b32 = algorithmic_bytes(nc, A, G, info["n_incoming_interior"], 4)
    b64 = algorithmic_bytes(nc, A, G, info["n_incoming_interior"], 8)
    ach32 = b32 / (lvl32 * 1e-3) / 1e9
    ach64 = b64 / (lvl64 * 1e-3) / 1e9
    k32, k64 = kernel_name(shape32, True), kernel_name(shape64, False)

    # Solve-level check: mixed precision vs FP64 GMRES on the same problem.
    solve = None
    phi_c2 = {}
    if not args.no_solve:
        tol = w.get("tol", 1e-10)
        phi64, _, s64 = sw.solve("gmres", iter_max=500, err_max=tol, restart=w.get("restart", 20),
                                 want_psi=False)
        phim, _, sm = sw.solve("mixed", iter_max=500, err_max=tol, restart=w.get("restart", 20),
                               want_psi=False)
        err = float(np.abs(phim - phi64).sum() / np.abs(phi64).sum())
        phi_c2 = {"fp64_gmres": phi64, "mixed": phim}
        solve = {"phi_rel_err_l1_mixed_vs_fp64": err, "fp64_gmres_seconds": s64["seconds"],
                 "mixed_seconds": sm["seconds"], "fp64_sweeps": s64["sweeps_fp64"],
                 "mixed_sweeps_fp32": sm["sweeps_fp32"], "mixed_sweeps_fp64": sm["sweeps_fp64"],
                 "fp64_residual": s64["final_error"], "mixed_residual": sm["final_error"],
                 "tol": tol, "speedup": s64["seconds"] / sm["seconds"]}

    # End to end through the drop-in sweep with host buffers, in the buffer
    # kinds the reference hands it: SweeperTraverse::solve passes the
    # sweeper's own psi (c_psi, which the SweeperCuda adapter page-locks) and
    # fixedPoint's local totalSource (pageable); also both page-locked and
    # both pageable, for context.
    e2e = None
    gpu_psi_hash = None
    if not args.no_e2e:
        npsi = nc * A * 4 * G
        n_e2e = max(1, min(args.steps, 3))

        def timed(src, psi):
            src[:] = q[:, None, :, :]
            sw.sweep(psi, src)
            grp.barrier()
            t0 = time.perf_counter()
            for _ in range(n_e2e):
                sw.sweep(psi, src)
            grp.barrier()
            return grp.max((time.perf_counter() - t0) / n_e2e)

        legs = {}
        src = np.empty(sw.psi_shape)
        psi = np.empty(sw.psi_shape)
        ty.lib().tycho_host_register(psi.ctypes.data, psi.nbytes)  # the adapter's c_psi
        legs["adapter"] = timed(src, psi)
        if rank == 0 and world == 1 and not args.no_parity:
            gpu_psi_hash = psi_hash(psi)
        ty.lib().tycho_host_unregister(psi.ctypes.data)
        legs["pageable"] = timed(src, psi)
        del src, psi
        src_t = torch.empty(npsi, dtype=torch.float64, pin_memory=True)
        psi_t = torch.empty(npsi, dtype=torch.float64, pin_memory=True)
        legs["pinned"] = timed(src_t.numpy().reshape(sw.psi_shape), psi_t.numpy().reshape(sw.psi_shape))
        del src_t, psi_t
        dt = legs["adapter"]
        e2e = {"value": grp.sum(updates) / dt, "unit": "updates/s", "h2d_bytes_per_step": npsi * 8,
               "d2h_bytes_per_step": npsi * 8,
               "path": "tycho_sweeper_sweep (FP64): psi page-locked as the SweeperCuda adapter locks its c_psi, "
                       "source pageable as fixedPoint's totalSource",
               "seconds_per_step": dt,
               "by_buffers": {k: {"updates_per_s": grp.sum(updates) / v, "seconds_per_step": v}
                              for k, v in legs.items()}}

    # the batch and serve legs need the device memory of this instance
    sw.close()
    batch = serve = None
    sample = []
    if not args.no_batch:
        try:
            batch = run_batch_leg(grp, dev, args.batch_instances, profile=args.profile_leg == "batch",
                                  sample=sample)
        except Exception as e:  # reported, never fatal to the headline line
            batch = {"error": str(e)[:300]}
    if not args.no_serve:
        try:
            serve = run_serve_leg(grp, dev, args.serve_requests,
                                  [float(r) for r in args.serve_rates.split(",") if r.strip()])
        except Exception as e:
            serve = {"error": str(e)[:300]}
    large = None
    if not args.no_large:
        try:
            # a clean device for the largest problem: the earlier legs' cached
            # pool memory (and the service's reservation) goes back first
            ty.release_cached_memory(dev)
            large = run_large_leg(grp, dev)
        except Exception as e:
            large = {"error": str(e)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(args.workload, steps=1)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "error": str(e)[:200]}

    parity = None
    if rank == 0 and world == 1 and not args.no_parity:
        parity = run_parity(args, dev, cpu, gpu_psi_hash, phi_c2, sample, large, serve)

    if rank == 0:
        t32 = profiled_traffic(args.workload, traffic_family(shape32, True))
        t64 = profiled_traffic(args.workload, traffic_family(shape64, False))
        line = {
            "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms32,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "cells": nc, "angles": A, "groups": G,
                       "levels": info["n_levels"], "parallelism": "replicas" if world > 1 else "1 gpu",
                       "l2": "psi > L2 and a 256 MB flush between steps",
                       "shape_fp32": shape32, "shape_fp64": shape64,
                       "autotune_ms": ({"fp32": tuned[1]["ms"], "fp64": tuned[0]["ms"]}
                                       if args.shape == "auto" else None)},
            "fp64": {"value": fp64_value, "ms_per_step": ms64, "dtype": "f64"},
            "mixed_vs_fp64_sweep_speedup": value / fp64_value,
            "solve": solve,
            "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s",
                         "frac": ach32 / peak, "traffic": t32,
                         "traffic_source": TRAFFIC_SOURCE if t32 is not None else None, "peak_kind": peak_kind,
                         "kernel": k32, "bytes_per_sweep": b32, "kernel_ms_per_sweep": lvl32,
                         "per": "one sweep (all of its launches)",
                         "frac_of_nominal": ach32 / NOMINAL_HBM_GBS, "nominal_peak": NOMINAL_HBM_GBS,
                         "fp64": {"kernel": k64, "achieved": ach64, "frac": ach64 / peak,
                                  "bytes_per_sweep": b64, "kernel_ms_per_sweep": lvl64,
                                  "traffic": t64}},
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": e2e,
            "batch": batch,
            "serve": serve,
            "large": large,
            "gpu_launches": args.steps * (launches[1] + launches[0]),
            "clocks": clocks,
            "wall_check_s": wall32,
        }
        print(json.dumps(line), flush=True)
    grp.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
