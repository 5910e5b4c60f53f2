"""Benchmark: THERMACOND's three-phonon kappa path on B200.

Workload (one step): the full job=1 sequence -- phonons on the mesh, |V3|^2
for every IBZ q1 against every mesh q2, tetrahedron delta + Bose weights,
linewidths Q, RTA kappa, collision matrix, RHS, CG solve, kappa -- for the
rock-salt Morse crystal of the benchmark suite (2 atoms, 6 bands, 16x16x16
mesh, 276 IBZ points, T = 300 K).  Inputs are synthetic: analytic Morse
force constants written in the reference's file formats.

metric: triplet-bands per second over the whole time-to-kappa step
(triplet-bands = nibz * nkc * ndyn^3 = 2.44e8 per step), higher is better.
Both precision paths run: FP64 (every stage double) and mixed (the V3
contraction in FP32, everything else double); the line's value is the mixed
path's, the FP64 path's numbers, the speed-up and the kappa difference
between the two sit beside it.

  value  device time of K steps with the context's tables already in HBM
         (CUDA events on the stream the library runs on; max over ranks)
  e2e    the same metric through the C ABI from the input files: file
         reading, table build and host->device upload, the pipeline and the
         device->host copy of the results, per step (wall clock)

--impl reference times the reference algorithm's CPU implementation (the
oracle restatement, all host threads) on a bounded sample of IBZ rows of
the same workload and prints the same JSON line with "impl": "reference".
With torchrun (N>1) the ranks split one job by IBZ rows, as the reference's
MPI decomposition does (kappa.f90:418-431), and exchange Q and the CG
matrix-vector products with NCCL all-gathers on device buffers (strong
scaling); the reference arm runs on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "anharmonic-lattice-dynamics_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "V3 triplet-bands/s & time-to-κ: mixed vs FP64 GPU path, 1 B200, κ err≤1e-4"
UNIT = "triplet-bands/s"
# --workload: the benchmark suite's configuration 1 (the metric's own) or
# configuration 2 (the large single structure); mesh edge, description
WORKLOADS = {
    "rocksalt": (16, "rocksalt-Morse NaCl-type, 2 atoms (6 bands), %dx%dx%d q-mesh, tetrahedron delta, T=300 K"),
    "lj-argon": (32, "fcc LJ argon, 1 atom (3 bands), %dx%dx%d q-mesh, Gaussian 0.05 THz, CG to residual 1e-8, "
                     "T=300 K"),
    "rocksalt-192": (4, "rocksalt-Morse 2x2x2 conventional supercell as one 64-atom cell (192 bands), structure 0 "
                        "of the batched suite, %dx%dx%d q-mesh, tetrahedron delta, T=300 K"),
}
CONFIG_OF = {"rocksalt": 1, "lj-argon": 2, "rocksalt-192": 4}
# the batched suites: many structures of uneven size in one ald_kappa_batched call
SUITES = {
    "suite3": "64 LJ argon mass superlattices, fcc conventional cell x p along x (p = 1..8, 8 structures each, "
              "12-96 bands, layer masses U[20,80] amu from seed 20261203 + s), (ceil(12/p) >= 2) x 12 x 12 mesh, "
              "lattice IBZ (none for the odd 3 x 12 x 12 meshes of p = 4, 5), Gaussian 0.1 THz, T=300 K",
    "suite4": "rock-salt Morse 64-atom cells (192 bands) with seeded jitter (D +-20 %%, alpha +-10 %%, masses "
              "U[10,130] amu), %d structures, %dx%dx%d mesh, tetrahedron delta, T=300 K",
}


def suite_dirs(root: str, suite: str, nstruct: int = 0, mesh_edge: int = 0):
    """Input directories of a batched suite (written once under root)."""
    from ald import inputs as I
    out = []
    if suite == "suite3":
        k = 0
        for p in range(1, 9):
            for j in range(8):
                st, rp = I.config(3, p=p, s=k)
                if rp.mesh[0] % 2:
                    rp.ibz = "none"
                d = os.path.join(root, "s3_%02d" % k)
                I.write_inputs(st, rp, d)
                out.append(d)
                k += 1
    else:
        n = nstruct or 2
        m = mesh_edge or 4
        for k in range(n):
            st, rp = I.config(4, mesh=(m, m, m), s=k)
            d = os.path.join(root, "s4_%02d" % k)
            I.write_inputs(st, rp, d)
            out.append(d)
    return out


def run_suite(args, suite: str):
    """A batched suite: ald_kappa_batched over all structures (mixed and FP64)
    against the same structures one after another; aggregate triplet-bands/s
    of the whole batch, device time of the call (CUDA events bracket it on the
    default stream after a device synchronize)."""
    import numpy as np
    import torch

    import ald
    tmp = tempfile.TemporaryDirectory()
    dirs = suite_dirs(tmp.name, suite, args.suite_n, args.mesh)
    res = {}
    nf = min(len(dirs), args.suite_fp64) if args.suite_fp64 > 0 else len(dirs)
    for prec, name in ((ald.MIXED, "mixed"), (ald.FP64, "fp64")):
        # the FP64 leg may run on the first nf structures only (the 192-band cells take seconds each)
        sel = dirs if name == "mixed" else dirs[:nf]
        ctxs = [ald.Context(d, ald.default_options(precision=prec, delta=ald.DELTA_TETRA if suite == "suite4"
                                                   else ald.DELTA_GAUSS)) for d in sel]
        tempk = [c.info.tempk for c in ctxs]
        out, st = ald.kappa_batched(ctxs, tempk)  # warm-up: phonons, workspaces, graphs
        tb = sum(o["triplet_bands"] for o in out)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out, st = ald.kappa_batched(ctxs, tempk)
        torch.cuda.synchronize()
        tbat = time.perf_counter() - t0
        t0 = time.perf_counter()
        seq = []
        for c, tk in zip(ctxs, tempk):  # one after another, each keeping device memory only for its run
            seq.append(c.kappa_pipeline(tk, want_modes=False))
            c.release_workspaces()
        torch.cuda.synchronize()
        tseq = time.perf_counter() - t0
        res[name] = {"structures": len(sel), "triplet_bands": tb, "batched_s": tbat, "sequential_s": tseq, "batched_value": tb / tbat,
                     "sequential_value": tb / tseq, "speedup_batched_vs_sequential": tseq / tbat,
                     "status": st, "kappa_trace_over_3": [float(np.trace(o["kappa_cg"]) / 3) for o in out],
                     "kappa_rel_diff_batched_vs_sequential": float(max(
                         np.abs(o["kappa_cg"] - q["kappa_cg"]).max() / np.abs(q["kappa_cg"]).max()
                         for o, q in zip(out, seq)))}
        for c in ctxs:
            c.close()
        ald.release_cached_memory()
    km, kf = np.array(res["mixed"]["kappa_trace_over_3"][:nf]), np.array(res["fp64"]["kappa_trace_over_3"])
    desc = SUITES[suite] if suite == "suite3" else SUITES[suite] % (len(dirs), args.mesh or 4, args.mesh or 4,
                                                                     args.mesh or 4)
    line = {"metric": METRIC, "value": res["mixed"]["batched_value"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "mixed (tensor-core V3 above 12 bands) and f64", "data": "synthetic (analytic FC2/FC3)",
            "config": {"workload": desc, "structures": len(dirs), "triplet_bands": res["mixed"]["triplet_bands"]},
            "mixed": res["mixed"],
            "fp64": res["fp64"],
            # time per structure, one structure after another: FP64 over mixed
            "mixed_speedup_vs_fp64_per_structure": (res["fp64"]["sequential_s"] / nf) /
                                                   (res["mixed"]["sequential_s"] / len(dirs)),
            "kappa_rel_err_mixed_vs_fp64": float(np.abs(km - kf).max() / np.abs(kf).max())}
    print(json.dumps(line))
    tmp.cleanup()


def _peaks():
    """Roofline denominators: MEASURED_PEAKS.json (written on this pool's
    B200s) when present, else the pool's earlier measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d.get("hbm_gbs", 6650.0)), "bf16_tflops": float(d.get("bf16_tflops", 1590.0)),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0))),
                "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a while to start: wait for its first line, then
            # keep only the samples taken from here on (the timed region)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines = []
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9 or f[0] != str(self.index):
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(d: str, mesh=(16, 16, 16), workload: str = "rocksalt"):
    from ald import inputs as I
    st, rp = I.config(CONFIG_OF[workload], mesh=mesh)
    I.write_inputs(st, rp, d)
    return rp


def workload_options(ald, rp, workload: str, **kw):
    """Library options of a workload: configuration 1 runs the defaults (tetrahedron delta, the
    reference's CG stop rule); configuration 2 the Gaussian delta and CG to a residual."""
    if workload != "lj-argon":
        return ald.default_options(**kw)
    return ald.default_options(delta=ald.DELTA_GAUSS, cg_stop=ald.CG_RESIDUAL, cg_tol=rp.cg_tol,
                               width_cm=rp.width_cm, **kw)


def cpu_baseline(d: str, rows: int = 0, gauss: bool = False):
    """The oracle (literal CPU restatement of the reference) on a bounded sample of IBZ rows:
    V3 + tetrahedron (or Gaussian) FGR + tauRTA for `rows` rows, all host threads."""
    import oracle_py
    oracle_py.build()
    nthreads = os.cpu_count() or 1
    O = oracle_py.Oracle(d, nthreads)
    t0 = time.time()
    O.mesh()
    O.phonons()
    O.tet()
    t_setup = time.time() - t0
    rows = rows or min(O.nibz, nthreads)
    t0 = time.time()
    v33 = O.v3(1, rows)
    P1, P2 = O.fgr(1, rows, v33, gauss=gauss)
    O.distribution(300.0)
    O.tau(1, rows, 300.0, P1, P2, want_p=False)
    dt = time.time() - t0
    tb = rows * O.nkc * O.ndyn ** 3
    return {"value": tb / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": "%d of %d IBZ rows of the same workload: V3 + %s FGR + tauRTA (%.1f s); "
                      "mesh/IBZ/phonon setup %.1f s not counted" % (rows, O.nibz, "Gaussian" if gauss else
                                                                    "tetrahedron", dt, t_setup),
            "seconds": dt, "nibz": O.nibz, "nkc": O.nkc, "ndyn": O.ndyn}


def arm_config(workload_desc, mesh, nibz, nkc, b, tb, world, mixed_head):
    """The workload of the bench line: both arms (the GPU path and the
    reference's CPU path) print this same dict for the same arguments."""
    return {"workload": workload_desc, "mesh": list(mesh), "nibz": nibz, "nkc": nkc, "ndyn": b,
            "triplet_bands_per_step": tb, "precision": "mixed" if mixed_head else "fp64",
            "l2": "working set > L2 (R1/R2 %.0f MB, collision matrix %.0f MB)" % (
                2 * nibz * nkc * b * b * 8 / 1e6, (3 * b * nibz) ** 2 * (4 if mixed_head else 8) / 1e6),
            "parallelism": ("dp%d: IBZ rows sharded as the reference's MPI split, NCCL all-gathers "
                            "of Q and the CG products" % world) if world > 1 else "single GPU"}


# DRAM bytes (read + write) of one launch from ncu captures of this workload
# (profiles/), keyed by (stage, nkc, bands, rows per launch)
# (stage, nkc, bands, precision, rows per launch): DRAM read + write of one launch
# (profiles/kappa_pipeline_nacl_morse_mesh16.md)
NCU_TRAFFIC = {("delta", 4096, 6, "mixed", 276): 1579.93e6, ("delta", 4096, 6, "fp64", 75): 587.54e6,
               ("v3", 4096, 6, "mixed", 276): 930.17e6}


def roofline(stage_ms, launches, nibz, nkc, b, peaks, cg_iters=1, cm_bytes=8, rows_per_launch=None,
             precision="mixed"):
    """The dominant device stage against its ceiling.

    achieved = algorithmic bytes per launch / device time per launch (the
    stage's CUDA events over the timed steps, divided by its launches).
    Algorithmic bytes of the tetrahedron delta: R1/R2 written once,
    2 nibz nkc b^2 8 bytes per step; `wide_bytes` adds the |V3|^2 read (FP32
    in the mixed path) and the R1/R2 read-modify-write of the fused kernel."""
    stages = {k: v for k, v in stage_ms.items() if k != "total"}
    dom = max(stages, key=stages.get)
    n = launches.get(dom, 1) or 1
    ms = stages[dom] / n
    N = 3 * b * nibz
    b3 = b ** 3
    vb = 4 if precision == "mixed" else 8  # the mixed pipeline keeps |V3|^2 in FP32
    alg = {
        "delta": 2 * nibz * nkc * b * b * 8 / n,
        "v3": nibz * nkc * (b3 * vb) / n,
        "collision": N * N * cm_bytes / n,
        "cg": N * N * cm_bytes,
    }
    wide = {"delta": nibz * nkc * (b3 * vb + 2 * 2 * b * b * 8) / n,
            "v3": nibz * nkc * (b3 * vb + 2 * b * b * 16) / n}
    if dom == "cg":
        ms = stages[dom] / max(1, cg_iters)
    by = alg.get(dom)
    if by is None or ms <= 0:
        return {"bound": "hbm", "achieved": None, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": None,
                "traffic": None, "kernel": dom}
    ach = by / (ms * 1e-3) / 1e9
    traffic = None
    rpl = rows_per_launch or max(1, nibz // n)
    for (st, nk, bb, pr, rows), t in NCU_TRAFFIC.items():
        if st == dom and nk == nkc and bb == b and pr == precision:
            traffic = t * rpl / rows  # DRAM traffic grows with the rows of a launch
    out = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": ach / peaks["hbm_gbs"], "traffic": traffic, "kernel": dom, "ms_per_launch": ms,
           "launches_per_step": n, "algorithmic_bytes": by, "peak_source": peaks["src"] + " (copy bandwidth)"}
    if dom in wide:
        out["wide_bytes"] = wide[dom]
        out["wide_frac"] = wide[dom] / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"]
    return out


def v3_roofline(stage_ms, launches, nibz, nkc, b, peaks, where):
    """V3 against the dense tensor-core peak: the algorithmic 24 b^4 real
    flops per (q1, q2) pair of the three complex mode products, over the V3
    stage's device time."""
    ms = stage_ms.get("v3", 0.0)
    flops = 24.0 * b ** 4 * nibz * nkc
    if ms <= 0:
        return None
    ach = flops / (ms * 1e-3) / 1e12
    pk = peaks["bf16_tflops"]
    return {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s", "frac": ach / pk,
            "kernel": "v3", "flops_per_step": flops, "ms_per_step": ms, "launches_per_step": launches.get("v3"),
            "peak_source": peaks["src"] + " (dense bf16 GEMM, burst)", "where": where}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ald", choices=["ald", "reference"])
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="both: time the FP64 and the mixed path; the line's value is the mixed path's")
    ap.add_argument("--suite-n", type=int, default=0, help="suite4: number of structures (default 2)")
    ap.add_argument("--suite-fp64", type=int, default=0,
                    help="suites: the FP64 leg on the first K structures only (default: all)")
    ap.add_argument("--workload", default="rocksalt", choices=sorted(WORKLOADS) + sorted(SUITES),
                    help="rocksalt: the metric's configuration (default); lj-argon: the large single structure")
    ap.add_argument("--mesh", type=int, default=0, help="mesh edge (default: the workload's own)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-cache", default="",
                    help="the autotuner's cache file (default: a fresh one in the workload's directory)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the extra driver-timed workloads (32^3 argon, the 192-band cell)")
    args = ap.parse_args()

    if args.workload in SUITES:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched suites are timed on the GPU only"}))
            return
        return run_suite(args, args.workload)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    mesh = (args.mesh or WORKLOADS[args.workload][0],) * 3
    workload_desc = WORKLOADS[args.workload][1] % mesh

    if args.impl == "reference":
        if rank != 0:
            return
        with tempfile.TemporaryDirectory() as d:
            make_workload(d, mesh, args.workload)
            vals = []
            cb = None
            for _ in range(args.warmup + args.steps):
                # two IBZ rows per step keep the whole run within a few minutes
                cb = cpu_baseline(d, rows=2, gauss=args.workload == "lj-argon")
                vals.append(cb["value"])
            v = sorted(vals[args.warmup:])[len(vals[args.warmup:]) // 2] if args.steps else vals[-1]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (analytic %s FC2/FC3, reference file formats)" % (
                    "Lennard-Jones" if args.workload == "lj-argon" else "Morse"),
                "config": arm_config(workload_desc, mesh, cb["nibz"], cb["nkc"], cb["ndyn"],
                                     float(cb["nibz"] * cb["nkc"] * cb["ndyn"] ** 3), world,
                                     args.precision != "fp64"),
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch

    import ald

    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)
    tmp = tempfile.TemporaryDirectory()
    d = tmp.name
    rp = make_workload(d, mesh, args.workload)
    stream = torch.cuda.Stream(device=dev)

    def timed_path(precision, d=d, rp=rp, workload=args.workload, steps=args.steps, warmup=args.warmup, det=None):
        """K timed steps of one precision path on a context whose tables are in HBM.
        det: the options' deterministic field (None: the library's default,
        deterministic for FP64, FP64 atomics for the mixed path)."""
        opts = workload_options(ald, rp, workload, device=dev, precision=precision)
        if det is not None:
            opts.deterministic = det
        ctx = ald.Context(d, opts)
        ctx.set_stream(stream.cuda_stream)
        tempk = ctx.info.tempk
        # the library's autotuner picks the launch shapes (outside the timed
        # region; its cache file lives in the workload's directory)
        tuning = ctx.autotune(args.tune_cache or os.path.join(d, "ald_tune.txt"), budget_s=30) if world == 1 else None

        ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # several GPUs: the reference's MPI row split, one rank per GPU, with
        # the Q and CG exchanges as NCCL all-gathers on device buffers
        gdev = ald.torch_allgather_device() if world > 1 else None

        def step():
            # the eigensolve (get_frequencies) runs before the pipeline call;
            # its time joins the pipeline's own "phonons" stage
            ev_a.record(stream)
            ctx.invalidate_phonons()
            ev_b.record(stream)
            if gdev is not None:
                out = ctx.kappa_pipeline_sharded(rank, world, gdev, tempk, device=True)
            else:
                out = ctx.kappa_pipeline(tempk, want_modes=False)
            out["stage_ms"]["phonons"] += ev_a.elapsed_time(ev_b)
            out["stage_ms"]["total"] += ev_a.elapsed_time(ev_b)
            return out

        for _ in range(warmup):
            out = step()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        stage_sum = {k: 0.0 for k in ald.STAGES}
        launches = 0
        with ClockSampler(dev) as clk:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                out = step()
                for k, v in out["stage_ms"].items():
                    stage_sum[k] += v
                launches += out["launches"]["total"] + 3  # + the eigensolver launches of get_frequencies
            e1.record(stream)
            torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ms = e0.elapsed_time(e1)
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_max = float(t.item())
        res = {"ms": ms_max, "steps": steps, "stage": {k: v / steps for k, v in stage_sum.items()},
               "launch_counts": dict(out["launches"]), "launches": launches, "out": out, "clocks": clk.summary(),
               "tempk": tempk, "nibz": ctx.nibz, "nkc": ctx.nkc, "b": ctx.ndyn, "opts": opts, "tuning": tuning}
        ctx.close()
        return res

    precisions = {"fp64": [ald.FP64], "mixed": [ald.MIXED], "both": [ald.FP64, ald.MIXED]}[args.precision]
    runs = {p: timed_path(p) for p in precisions}
    # the FP64 path with FP64 atomics in the delta (not bitwise repeatable), for comparison
    fp64_atomic = timed_path(ald.FP64, steps=min(args.steps, 5), det=0) if world == 1 and ald.FP64 in runs else None
    head = runs[precisions[-1]]  # the mixed path when both run
    nibz, nkc, b = head["nibz"], head["nkc"], head["b"]
    out = head["out"]
    tb = out["triplet_bands"]
    ms_max = head["ms"]
    # one job split over the ranks (strong scaling): the job's triplet-bands
    # per second of the slowest rank
    value = tb * args.steps / (ms_max * 1e-3)
    per_step = head["stage"]
    per_launch_counts = head["launch_counts"]
    launches = head["launches"]
    clk_summary = head["clocks"]
    opts = head["opts"]
    tempk = head["tempk"]

    # ---- end to end through the C ABI from the input files (headline path)
    e2e_times, h2d, d2h = [], 0.0, 0.0
    gdev_e2e = ald.torch_allgather_device() if world > 1 else None
    for i in range(max(2, min(args.steps, 5)) + 1):
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c2 = ald.Context(d, opts)
        if world == 1:  # the tuned launch shapes, read from the cache file
            c2.autotune(args.tune_cache or os.path.join(d, "ald_tune.txt"))
        if gdev_e2e is not None:
            c2.set_stream(stream.cuda_stream)
            o2 = c2.kappa_pipeline_sharded(rank, world, gdev_e2e, tempk, device=True)
        else:
            o2 = c2.kappa_pipeline(tempk, want_modes=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        h2d, d2h = c2.h2d_bytes(), o2["d2h_bytes"] + 9 * 2 * 8
        c2.close()
        if i > 0:
            e2e_times.append(dt)
    e2e = tb / (sorted(e2e_times)[len(e2e_times) // 2])
    if world > 1:  # the slowest rank's time
        te = torch.tensor([e2e], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MIN)
        e2e = float(te.item())

    # ---- configuration 1's three temperatures on one context: new eigenpairs,
    # then 100, 300 and 600 K (|V3|^2 formed once and kept across the calls)
    temps3 = {}
    if world == 1 and args.workload == "rocksalt":
        for pp in precisions:
            opts3 = workload_options(ald, rp, args.workload, device=dev, precision=pp)
            c3 = ald.Context(d, opts3)
            c3.set_stream(stream.cuda_stream)
            c3.autotune(args.tune_cache or os.path.join(d, "ald_tune.txt"))
            for _ in range(2):  # the second round is timed
                ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ea.record(stream)
                c3.invalidate_phonons()
                o3 = [c3.kappa_pipeline(T, want_modes=False) for T in (100.0, 300.0, 600.0)]
                eb.record(stream)
                torch.cuda.synchronize()
            temps3[pp] = {"ms_three_temperatures": ea.elapsed_time(eb),
                          "v3_launches_per_temperature": [o["launches"]["v3"] for o in o3],
                          "kappa_cg_trace_over_3": [float(np.trace(o["kappa_cg"]) / 3) for o in o3]}
            c3.close()

    # ---- extra workloads, driver-timed beside the headline (single GPU only):
    # the large single structure (32^3 argon, 3-band tensor-core class sums)
    # and the 192-band cell (both mode products on the tensor cores)
    extras = {}
    if world == 1 and not args.no_extra:
        peaks0 = _peaks()
        for wl, st_, wu in (("lj-argon", 5, 3), ("rocksalt-192", 2, 1)):
            try:
                t2 = tempfile.TemporaryDirectory()
                m2 = (WORKLOADS[wl][0],) * 3
                rp2 = make_workload(t2.name, m2, wl)
                rr = {pp: timed_path(pp, d=t2.name, rp=rp2, workload=wl, steps=st_, warmup=wu)
                      for pp in (ald.FP64, ald.MIXED)}
                f, m = rr[ald.FP64], rr[ald.MIXED]
                tb2 = m["out"]["triplet_bands"]
                kf, km = np.asarray(f["out"]["kappa_cg"]), np.asarray(m["out"]["kappa_cg"])
                extras[wl] = {
                    "workload": WORKLOADS[wl][1] % m2, "steps": st_, "warmup": wu,
                    "nibz": m["nibz"], "nkc": m["nkc"], "ndyn": m["b"],
                    "mixed": {"value": tb2 * st_ / (m["ms"] * 1e-3), "unit": UNIT, "ms_per_step": m["ms"] / st_,
                              "stage_ms_per_step": {k: round(v, 4) for k, v in m["stage"].items()},
                              "roofline_v3": v3_roofline(m["stage"], m["launch_counts"], m["nibz"], m["nkc"], m["b"],
                                                         peaks0, "mixed path")},
                    "fp64": {"value": tb2 * st_ / (f["ms"] * 1e-3), "unit": UNIT, "ms_per_step": f["ms"] / st_,
                             "stage_ms_per_step": {k: round(v, 4) for k, v in f["stage"].items()}},
                    "mixed_speedup_vs_fp64": f["ms"] / m["ms"],
                    "mixed_v3_speedup_vs_fp64": f["stage"]["v3"] / max(m["stage"]["v3"], 1e-9),
                    "kappa_rel_err_mixed_vs_fp64": float(np.abs(km - kf).max() / np.abs(kf).max()),
                    "clocks": m["clocks"], "tuning": {"mixed": m["tuning"], "fp64": f["tuning"]}}
                t2.cleanup()
            except Exception as ex:  # reported beside the headline, never required
                extras[wl] = {"failed": str(ex)[:300]}

    line = None
    if rank == 0:
        peaks = _peaks()
        mixed_head = precisions[-1] == ald.MIXED
        rf = roofline(per_step, per_launch_counts, nibz, nkc, b, peaks, cg_iters=max(1, out["cg_iters"]),
                      cm_bytes=4 if mixed_head else 8, precision="mixed" if mixed_head else "fp64")
        rf_v3 = v3_roofline(per_step, per_launch_counts, nibz, nkc, b, peaks,
                            "mixed path" if mixed_head else "fp64 path")
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cb = cpu_baseline(d, gauss=args.workload == "lj-argon")
                cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as ex:  # the baseline is reported, never required
                cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": "failed: %s" % ex}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": ("mixed: V3 class sums split-f16 on tensor cores (3 bands) or f32, mode products, delta "
                          "weights and CG matrix f32; eigensolve, sums, CG vectors and kappa f64")
                if mixed_head else "f64",
                "data": "synthetic (analytic %s FC2/FC3 written in the reference's file formats)" % (
                    "Lennard-Jones" if args.workload == "lj-argon" else "Morse"),
                "config": arm_config(workload_desc, mesh, nibz, nkc, b, tb, world, mixed_head),
                "time_to_kappa_ms": ms_max / args.steps,
                "stage_ms_per_step": {k: round(v, 4) for k, v in per_step.items()},
                "kappa_cg_trace_over_3": float(np.trace(out["kappa_cg"]) / 3),
                "cg_iters": out["cg_iters"],
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "seconds_per_step": sorted(e2e_times)[len(e2e_times) // 2]},
                "gpu_launches": launches, "roofline": rf, "roofline_v3": rf_v3, "cpu_baseline": cb,
                "tuning": head["tuning"],
                "clocks": clk_summary}
        if ald.FP64 in runs and ald.MIXED in runs:
            f, m = runs[ald.FP64], runs[ald.MIXED]
            kf, km = np.asarray(f["out"]["kappa_cg"]), np.asarray(m["out"]["kappa_cg"])
            krf, krm = np.asarray(f["out"]["kappa_rta"]), np.asarray(m["out"]["kappa_rta"])
            line["fp64"] = {"value": tb * args.steps / (f["ms"] * 1e-3), "unit": UNIT,
                            "ms_per_step": f["ms"] / args.steps,
                            "stage_ms_per_step": {k: round(v, 4) for k, v in f["stage"].items()},
                            "tuning": f["tuning"],
                            "clocks": f["clocks"], "delta": "deterministic (the FP64 default)"}
            if fp64_atomic is not None:
                a_ = fp64_atomic
                line["fp64"]["atomic_delta"] = {
                    "ms_per_step": a_["ms"] / a_["steps"],
                    "stage_ms_per_step": {k: round(v, 4) for k, v in a_["stage"].items()},
                    "note": "ald_options.deterministic = 0: FP64 atomics, last bits vary between runs"}
            line["mixed_speedup_vs_fp64"] = f["ms"] / m["ms"]
            line["mixed_v3_speedup_vs_fp64"] = f["stage"]["v3"] / m["stage"]["v3"]
            line["kappa_rel_err_mixed_vs_fp64"] = {
                "cg": float(np.abs(km - kf).max() / np.abs(kf).max()),
                "rta": float(np.abs(krm - krf).max() / np.abs(krf).max())}
        if temps3:
            line["temperatures_100_300_600K"] = {("mixed" if k == ald.MIXED else "fp64"): v for k, v in temps3.items()}
        if extras:
            line["extra_workloads"] = extras
        print(json.dumps(line))
    tmp.cleanup()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
