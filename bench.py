#!/usr/bin/env python
"""Benchmark of the B200 tidal forward path: seconds per complex edge-FEM solve to a 1e-8 FP64 true residual.

One step = one pass of the forward path over one batch: assemble the
Nedelec system (K, M and the sigma(v x F) right-hand sides) from the
resident mesh, solve it with COCG to a true residual <= 1e-8, evaluate B and
E at the sites.  The workload is the 96x96x64-hex model (3,538,944 tets,
4,193,536 edges, log-normal subsurface, M2 source, 400 sites), synthetic
and seeded (no dataset exists for it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--method METHOD]
  python bench.py --impl reference ...   # the CPU reference path (oracle restatement)

Methods (preconditioner, precision, systems per step): plain = SSOR-COCG
FP64, one system (the reference's solver on the device, natural row order);
plain-mc = the multicolour SSOR; hybrid = multicolour SSOR plus the
gradient-space (nodal) correction; mixed = hybrid with FP32 inner COCG
under FP64 refinement; *-pc32 = FP64 COCG with the preconditioner in FP32;
batched / batched-mixed / batched-pc32 = 8 tidal periods x 2 source patterns =
16 systems per solve (batched-pc32 is the default); learned* = flexible COCG with the learned
network (flexible COCG, z = H(r) + N(r) over the gradient-corrected SSOR H when
that checkpoint exists); packed = 24 uneven meshes (n x n x 3n/4, n in 8..32)
in one solve.

Prints ONE JSON line on rank 0.  Under torchrun every rank solves its own
independent systems (replicas; weak scaling), the time is the max over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s per complex edge-FEM solve to 1e-8 residual: learned+batched vs plain COCG"
# The reference's own solver (COCG13_single with SSOR, natural row order) on the
# 96x96x64 model, run once on a B200 through the COCG13_single seam: it had not
# reached 1e-8 after 30,000 iterations (recursive = true residual 6.843e-5),
# 15.862 ms per iteration.  Its iteration count is therefore a lower bound.
PLAIN_96 = {"iterations": 30000, "converged": False, "resid_true_at_cap": 6.843e-05, "ms_per_iteration": 15.862,
            "seconds_at_cap": 475.9}
UNIT = "s/solve"
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of a kernel, from a
# one-pass ncu capture of the 96x96x64 batch itself (4,193,536 rows; two iterations, the mean):
# `python bench.py --profile-case --workload large --maxit 60 --spmv-rpw 8` under
# `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum`.  Scaled by rows for other models.
_T96 = "ncu one-pass dram bytes of a launch on this 96x96x64 batch (profile case, FP32 preconditioner)"
TRAFFIC = {
    "cocg_spmv_fp64pc32_ns16_rpw8": {"bytes": 4.085e9, "rows": 4193536, "source": _T96},
    "cocg_fwd_sweep_mc_fp64pc32_ns16": {"bytes": 5.877e9, "rows": 4193536, "source": _T96},
    "cocg_bwd_sweep_mc_fp64pc32_ns16": {"bytes": 3.163e9, "rows": 4193536, "source": _T96},
    "cocg_p_update_fp64pc32_ns16": {"bytes": 4.931e9, "rows": 4193536, "source": _T96},
    "cocg_nodal_correction_fp64pc32_ns16": {"bytes": 1.991e9, "rows": 4193536, "source": _T96},
}
DEFAULT_METHOD = "batched-pc32"
TOL = 1e-8
FALLBACK_HBM_GBS = 6650.0


# ----------------------------------------------------------------------------- helpers
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1])); smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def widths(name: str):
    """(COCG real bytes, preconditioner real bytes) from a kernel name's precision tag."""
    if "_fp64pc32_" in name:
        return 8, 4
    if "_fp32_" in name:
        return 4, 4
    return 8, 8


def kernel_bytes(name: str, n: int, nnz: int, ns: int, ntet: int = 0, nsrc: int = 1, node: int = 0, nodes: int = 0,
                 mc: bool = False, fold: bool = False) -> float:
    """Algorithmic bytes of one launch of the named kernel (values read/written once).

    mc: multicolour iteration (x += alpha p moves from the forward sweep to the p
    update); fold: the hybrid's z += G u is formed inside the p update.  The COCG
    vectors (r, p, q) and the SpMV use the COCG width, the preconditioner's matrix
    copies and vectors (y, z, nodal t, u) the preconditioner width (the name's tag)."""
    rb, pb = widths(name)
    if "_seg" in name:
        ns = 1  # packed batch: one system per row
    ent = 2 * rb + 4                  # (K, M) pair + column index per stored entry
    pent = 2 * pb + 4                 # the same in the preconditioner's copy
    vec = 2 * rb * ns                 # one complex COCG value per system per row
    pvec = 2 * pb * ns                # one complex preconditioner value per system per row
    off = (nnz - n) // 2              # strictly lower (= strictly upper) entries
    if name.startswith("cocg_fwd_sweep_mc"):
        # colour-ordered split rows: the earlier-colour half, position pointers and row ids, the
        # FP64 (K, M) diagonal pair; r read/write, q read, y write (x is updated in the p update)
        return pent * off + 8 * n + 16 * n + n * (3 * vec + pvec)
    if name.startswith("cocg_bwd_sweep_mc"):
        # the later-colour half, pointers, ids, diagonal pair; y read, z write (in place);
        # rho from the diagonal, packed batches read r instead for their per-mesh rho
        b = pent * off + 8 * n + 16 * n + n * 2 * pvec
        return b + n * vec if "_seg" in name else b
    if name.startswith("cocg_nodal_correction"):
        nnz_n = node + 2 * n          # node graph: the node and its edge neighbours
        pvn = pvec                    # nodal vectors have the edge vectors' width
        gt = 4 * (node + 1) + 8 * n + n + n * vec + node * pvn
        # two sweeps, each over its half of the off-diagonal entries, with pointers and ids;
        # forward: t, dd read, y write; backward: y read and write, dd read
        sweeps = 2 * (pent * (nnz_n - node) // 2 + 4 * (node + 1) + 4 * node + 3 * node * pvn)
        if fold:  # the backward nodal sweep also reads t for t^T u
            return gt + sweeps + node * pvn
        gadd = 8 * n + n + 2 * n * pvec + n * vec + node * pvn
        return gt + sweeps + gadd
    if name.startswith("cocg_fwd_sweep"):
        # L entries, rowptr+diagpos, flag write; r r/w, q, p, x r/w (FP64), DD, y write, y gather
        return ent * off + 12 * n + n * (vec * 6 + 32 * ns)
    if name.startswith("cocg_bwd_sweep"):
        # U entries, rowptr+diagpos, flag write; y read, z write, DD, z gather, r read
        return ent * off + 12 * n + n * vec * 5
    if name.startswith("cocg_spmv"):
        # all entries, rowptr; p gather, p own read (p^T q), q write
        return ent * nnz + 4 * (n + 1) + n * vec * 3
    if name.startswith("cocg_p_update"):
        b = n * (pvec + 2 * vec)            # z read, p read and write
        if mc:
            b += n * 32 * ns                # x read and write (FP64)
        if fold:
            b += 8 * n + n + node * pvec    # line, bc, u (each node once)
        return b
    if name.startswith("assemble_rows"):
        # tetrahedron data (n4, n6line, tag, sigma), node coordinates, adjacency, pattern, values, rhs
        return ntet * (16 + 24 + 4 + 8) + 24 * node + 24 * ntet + 4 * (n + 1) + 4 * nnz + 16 * nnz + 16 * n * nsrc \
            + nodes * (24 + 48) * nsrc
    return 0.0


# ----------------------------------------------------------------------------- workloads
METHODS = {
    # method: (preconditioner, precision, batched)
    "plain": ("SSOR", "fp64", False),          # the reference's COCG13_single with SSOR, natural row order
    "plain-mc": ("SSOR_MC", "fp64", False),
    "hybrid": ("HYBRID", "fp64", False),
    "mixed": ("HYBRID", "mixed", False),
    "batched": ("HYBRID", "fp64", True),
    "batched-mixed": ("HYBRID", "mixed", True),
    "batched-pc32": ("HYBRID", "pc32", True),
    "hybrid-pc32": ("HYBRID", "pc32", False),
    "learned": ("LEARNED", "fp64", False),
    "learned-batched": ("LEARNED", "fp64", True),
    "learned-batched-mixed": ("LEARNED", "mixed", True),
    "packed": ("HYBRID", "fp64", False),
    "packed-pc32": ("HYBRID", "pc32", False),
}


def build_workload(method: str, rank: int, workload: str = "large"):
    from actfemtide_b200 import synth

    def make(seed):
        if workload == "large":
            return synth.large_model(seed=seed)
        if workload == "medium":  # matrix ~0.17 GB: larger than L2, small enough for ncu captures
            return synth.tidal_box(48, 48, 32, seed=seed, grf=True, block=False, name="box48x48x32")
        return synth.small_model(seed=seed)
    m = make(rank)
    if METHODS[method][2]:
        m2 = make(seed=1000 + rank)
        freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
        f = np.concatenate([freqs, freqs])
        src = np.repeat([0, 1], 8).astype(np.int32)
        sources = [(m.F, m.v), (m2.F, m2.v)]
    else:
        f = np.array([1.0 / synth.M2_PERIOD_S])
        src = np.zeros(1, np.int32)
        sources = [(m.F, m.v)]
    return m, f, src, sources


def solve_kwargs(method: str, precond: str | None = None):
    pc, prec, _ = METHODS[method]
    return dict(precond=precond or pc, precision=prec)


# ----------------------------------------------------------------------------- GPU arm
class Job:
    """The inputs of one step's problem as host arrays, and how to load them through the C ABI."""

    def __init__(self, method: str, rank: int, workload: str):
        from actfemtide_b200 import synth
        self.method = method
        if method == "packed":
            self.pk = synth.pack(synth.uneven_models(24, seed=rank))
            self.parts = self.pk.parts
            self.freqs = np.array([m.freqs[0] for m in self.parts])
            self.srcs = np.zeros(len(self.parts), np.int32)
            self.sites = self.parts[0].sites
            self.ntet = int(self.pk.n4.shape[0])
            self.node = int(self.pk.xyz.shape[0])
            self.nodes = int(sum(m.nodes for m in self.parts))
            self.nsrc = 1
            dims = sorted(m.dims[0] for m in self.parts)
            self.desc = (f"24 packed uneven meshes n x n x round(3n/4), n in {dims[0]}..{dims[-1]}: "
                         f"{self.ntet} tets, {{n}} edges, nnz {{nnz}}, {self.sites.shape[0]} sites per mesh")
        else:
            m, self.freqs, self.srcs, self.sources = build_workload(method, rank, workload)
            self.m = m
            self.sites = m.sites
            self.ntet, self.node, self.nodes, self.nsrc = m.ntet, m.node, m.nodes, len(self.sources)
            self.desc = (f"{m.dims[0]}x{m.dims[1]}x{m.dims[2]} hex box: {m.ntet} tets, {{n}} edges, nnz {{nnz}}, "
                         f"{m.sites.shape[0]} sites")

    @property
    def ns(self):
        return len(self.freqs)

    def host_arrays(self, pin, line=None, n6=None):
        if self.method == "packed":
            pk = self.pk
            return dict(xyz=pin(pk.xyz), n4=pin(pk.n4), tag=pin(pk.tag), sig=pin(pk.sigma_tet), F=[pin(pk.F)],
                        v=[pin(pk.v)], sites=pin(self.sites), node_ptr=pin(pk.node_ptr))
        m = self.m
        return dict(xyz=pin(m.xyz), n4=pin(m.n4), tag=pin(m.tag), line=pin(line), n6=pin(n6), sig=pin(m.sigma_land),
                    F=[pin(F) for F, _ in self.sources], v=[pin(v) for _, v in self.sources], sites=pin(m.sites))

    def load(self, fw, h=None):
        """Load the problem (from the job's arrays, or from the host buffers h)."""
        if self.method == "packed":
            if h is None:
                fw.load_packed(self.pk)
                return
            fw.set_mesh(h["xyz"], h["n4"], h["tag"])
            fw.set_segments(h["node_ptr"])
            fw.set_sigma(h["sig"])
            fw.set_source(h["F"][0], h["v"][0], 0)
            b = self.pk.bounds
        else:
            m = self.m
            if h is None:
                fw.load_model(m, sources=self.sources)
                return
            fw.set_mesh(h["xyz"], h["n4"], h["tag"], h["line"], h["n6"])
            fw.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=h["sig"])
            for k in range(len(h["F"])):
                fw.set_source(h["F"][k], h["v"][k], k)
            b = m.bounds
        fw.set_bounds(b["zmin"], b["zmax"], b["xout"], b["yout"])


def shared_config(desc: str, ns: int, ws: int, nnz: int) -> dict:
    """The workload description both arms print (the GPU solve and the reference's CPU solver)."""
    return {"workload": desc, "solves_per_step": ns,
            "systems": ("8 tidal periods (12.4206, 12.0000, 12.6583, 11.9672, 23.9345, 25.8193, 24.0659, 26.8684 h) "
                        "x 2 seeded source-velocity patterns") if ns == 16 else f"{ns} system(s)",
            "tol_true_residual": TOL, "parallelism": f"replicas x{ws}",
            "l2": "working set > 126 MB L2 (matrix alone %.2f GB)" % (nnz * 20 / 1e9)}


def c1_desc() -> str:
    """The 96x96x64 workload's description (sizes from the Kuhn split: 6 tets per hex)."""
    return "96x96x64 hex box: 3538944 tets, 4193536 edges, nnz 68152576, 400 sites"


def run_gpu(args):
    import torch
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from actfemtide_b200 import capi
    from actfemtide_b200.forward import Forward

    job = Job(args.method, rank, args.workload)
    fw = Forward(local)
    job.load(fw)
    if "learned" in args.method:
        # the network over the gradient-corrected SSOR when that checkpoint exists, else the Jacobi-base one
        from actfemtide_b200 import learned
        ckpt = args.ckpt or (learned.HYBRID_CKPT if os.path.exists(learned.HYBRID_CKPT + ".json")
                             else learned.DEFAULT_CKPT)
        fw.mpnn_set_params(learned.load(ckpt))
        fw.mpnn_set_base(learned.load_base(ckpt) == 1)
    if args.spmv_rpw:
        fw.set_spmv_rows_per_warp(args.spmv_rpw)
    n = fw.nline
    INU, IAU, INL, IAL = fw.export_pattern()
    nnz = n + 2 * len(IAU)
    ns = job.ns
    kw = solve_kwargs(args.method, args.precond)
    stream = torch.cuda.ExternalStream(fw.stream_ptr(), device=local)

    def step(maxit=args.maxit):
        fw.assemble()
        res = fw.solve(job.freqs, srcs=job.srcs, tol=TOL, maxit=maxit, **kw)
        out = fw.sites(job.sites, nsys=ns)
        return res, out

    if args.profile_case:
        # profiler case: one assembly + solve (capped at --maxit) + sites, no timing, no JSON bench line
        res, _ = step()
        print(f"profile case {args.workload}: iterations {res.iterations}, true residual {res.resid_true:.3e}, "
              f"status {res.status}", flush=True)
        fw.close()
        return

    for _ in range(args.warmup):
        res, _ = step()
        if not res.ok and not args.allow_unconverged:
            raise SystemExit(f"warm-up solve failed: {res}")
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = capi.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    iters, resid, refs = [], [], []
    for _ in range(args.steps):
        res, out = step()
        iters.append(res.iterations)
        resid.append(res.resid_true)
        refs.append(res.refinements)
        if not res.ok and not args.allow_unconverged:
            raise SystemExit(f"timed solve failed: {res}")
    e1.record(stream)
    torch.cuda.synchronize()
    launches = capi.launch_count() - l0
    if ws > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)

    # ---- per-kernel device times: a separate, bounded pass with CUDA events around every kernel
    fw.set_profiling(True)
    step(maxit=args.prof_iters)
    prof = fw.profile()
    prof = {k: v for k, v in prof.items() if not k.startswith("host_")}  # kernels only
    fw.set_profiling(False)

    # ---- end to end through the C ABI with pinned host buffers, copies inside the timed region
    line, n6 = fw.lines()
    h = job.host_arrays(lambda a: _pinned(torch, a), line, n6)
    h2d = sum(int(a.nbytes) for k, a in h.items() if not isinstance(a, list)) + \
        sum(int(a.nbytes) for a in h["F"]) + sum(int(a.nbytes) for a in h["v"])
    d2h = 16 * 5 * job.sites.shape[0] * ns
    e2e_steps = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        job.load(fw, h)
        fw.assemble()
        r2 = fw.solve(job.freqs, srcs=job.srcs, tol=TOL, maxit=args.maxit, **kw)
        out = fw.sites(h["sites"], nsys=ns)
        if not r2.ok and not args.allow_unconverged:
            raise SystemExit(f"e2e solve failed: {r2}")
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    # max over ranks
    times = np.array([ms / 1e3, e2e_s], dtype=np.float64)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor(times, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times = t.cpu().numpy()
        dist.barrier()
    total_solves = args.steps * ns * ws
    value = times[0] / total_solves
    e2e_value = times[1] / (e2e_steps * ns * ws)

    # ---- roofline of the dominant kernel
    peak, peak_kind = peaks()
    dom, dom_ms, dom_n = None, 0.0, 0
    for name, (kms, cnt) in prof.items():
        if kms > dom_ms:
            dom, dom_ms, dom_n = name, kms, cnt
    pc = kw["precond"]
    mc = pc in ("SSOR_MC", "HYBRID") or "learned" in args.method
    fold = pc == "HYBRID" and not args.method.startswith("packed")
    per_launch = kernel_bytes(dom or "", n, nnz, ns, job.ntet, job.nsrc, job.node, job.nodes, mc=mc, fold=fold)
    achieved = per_launch / (dom_ms / max(1, dom_n) / 1e3) / 1e9 if dom_ms > 0 else 0.0
    traffic, traffic_src = None, None
    tr = TRAFFIC.get(dom or "")
    if tr and job.method != "packed":
        traffic = tr["bytes"] * n / tr["rows"]
        traffic_src = tr["source"]
    kernels = {}
    total_ms = sum(x[0] for x in prof.values())
    for k, (kms, cnt) in sorted(prof.items(), key=lambda kv: -kv[1][0]):
        b = kernel_bytes(k, n, nnz, ns, job.ntet, job.nsrc, job.node, job.nodes, mc=mc, fold=fold)
        avg = kms / max(1, cnt)
        kernels[k] = {"share": round(kms / max(1e-9, total_ms), 4), "avg_ms": round(avg, 5), "launches": cnt,
                      "bytes_per_launch": b, "gbs": round(b / (avg / 1e3) / 1e9, 1) if avg > 0 else None,
                      "frac": round(b / (avg / 1e3) / 1e9 / peak, 3) if avg > 0 and b else None}

    # ---- the reference's own solvers on the same GPU and model (bounded), and a converged pair on C0
    plain = None
    if rank == 0 and ws == 1 and args.plain_iters > 0 and not args.method.startswith("packed"):
        plain = plain_same_gpu(fw, job, args.plain_iters)
    pair = None
    if rank == 0 and ws == 1 and args.c0_pair and not args.method.startswith("packed"):
        pair = converged_pair_c0(local, kw, args.c0_threads)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.method.startswith("packed"):
        cpu = cpu_baseline(job, args.cpu_seconds, plain)
    fw.close()
    line_out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp64": "complex-f64", "pc32": "complex-f64 COCG, complex-f32 preconditioner",
                  "mixed": "complex-f32 inner COCG / f64 refinement"}[kw["precision"]],
        "data": "synthetic (seeded Kuhn-split boxes, log-normal subsurface, tidal sources)",
        "config": (shared_config(job.desc.format(n=n, nnz=nnz), ns, ws, nnz) if not job.method.startswith("packed")
                   else {"workload": job.desc.format(n=n, nnz=nnz), "solves_per_step": ns,
                         "parallelism": f"replicas x{ws}"}),
        "method": {"name": args.method, "preconditioner": kw["precond"], "precision": kw["precision"],
                   "note": "batched gradient-corrected (Hiptmair hybrid) multicolour-SSOR COCG; the learned network "
                           "is not in this method (it does not pay on these models)" if "learned" not in args.method
                   else "flexible COCG with the learned correction"},
        "solver": {"iterations_median": int(np.median(iters)), "refinements_median": int(np.median(refs)),
                   "true_residual_max": float(max(resid))},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "includes": "set_mesh (upload, numbering, pattern) + cond + source + assemble + "
                                                "solve + sites, through the C ABI from pinned host buffers"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "peak_kind": peak_kind,
                     "bytes_per_launch": per_launch, "avg_launch_ms": dom_ms / max(1, dom_n), "traffic": traffic,
                     "traffic_source": traffic_src,
                     "profile_pass": f"one step with the iteration cap at {args.prof_iters}, CUDA events around "
                                     "every kernel (graphs off), outside the timed region",
                     "kernels": kernels},
        "gpu_launches": int(launches),
        "clocks": clk,
        "plain_same_gpu": plain,
        "like_for_like_c0": pair,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line_out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


_PINNED = []  # pinned host tensors behind the numpy views handed out by _pinned


def _pinned(torch, a):
    """A pinned (page-locked) host copy of a, so the host->device copies of the e2e pass are DMA copies."""
    a = np.ascontiguousarray(a)
    t = torch.empty(a.shape, dtype=getattr(torch, {"float64": "float64", "int32": "int32", "complex128": "complex128"}[
        str(a.dtype)]), pin_memory=True)
    out = t.numpy()
    out[...] = a
    _PINNED.append(t)
    return out


def plain_same_gpu(fw, job, cap):
    """The reference's solver (COCG13_single: FP64, natural row order) with SSOR and with its
    diagonal-modified IC(0), system 0 of the workload alone, capped at `cap` iterations."""
    out = {"system": "system 0 of the batch alone", "cap": cap}
    for pc in ("SSOR", "IC"):
        fw.assemble()
        r = fw.solve(job.freqs[:1], srcs=job.srcs[:1], precond=pc, precision="fp64", tol=TOL, maxit=cap)
        out[pc] = {"iterations": r.iterations, "converged": bool(r.ok), "resid_true": r.resid_true,
                   "seconds": r.seconds, "ms_per_iteration": 1e3 * r.seconds / max(1, r.iterations),
                   "status": capi_status(r.status)}
    return out


def capi_status(code):
    from actfemtide_b200 import capi
    return capi.STATUS.get(code, code)


def _assemble_batch(of, m, m2, freqs, threads):
    """Oracle systems of the 8 x 2 batch: A(omega_k) with pattern 1's b, and pattern 2's b."""
    import concurrent.futures as cf
    import dataclasses
    from oracle import oracle as O
    mk2 = dataclasses.replace(m, F=m2.F, v=m2.v)

    def one(f):
        A = of.assemble(f)
        b2 = O.forward_assemble(mk2, of.line, of.n6line, of.pat, f, of.sigma_tet).b
        return A, b2
    with cf.ThreadPoolExecutor(max_workers=max(1, min(threads, 4))) as ex:
        return list(ex.map(one, freqs))


def converged_pair_c0(local, kw, threads):
    """A like-for-like pair of finished solves on the 20x20x20 model, where the reference's solver converges:
    the same 16 systems (8 periods x 2 patterns) to an FP64 residual of 1e-8, on the GPU (this method) and with
    the oracle's COCG13_single + SSOR on the host's cores, both timed here."""
    import concurrent.futures as cf
    import torch
    from actfemtide_b200 import synth
    from actfemtide_b200.forward import Forward
    from oracle import oracle as O
    m = synth.small_model(seed=0)
    m2 = synth.tidal_box(20, 20, 20, seed=1000, name="box20")
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    f = np.concatenate([freqs, freqs])
    src = np.repeat([0, 1], 8).astype(np.int32)
    with Forward(local) as fw:
        fw.load_model(m, sources=[(m.F, m.v), (m2.F, m2.v)])
        for _ in range(2):
            fw.assemble()
            fw.solve(f, srcs=src, tol=TOL, **kw)
        torch.cuda.synchronize()
        reps = 5
        t0 = time.perf_counter()
        for _ in range(reps):
            fw.assemble()
            r = fw.solve(f, srcs=src, tol=TOL, **kw)
            out = fw.sites(m.sites, nsys=16)
        torch.cuda.synchronize()
        gpu_s = (time.perf_counter() - t0) / (reps * 16)
        gpu_it = r.iterations
        gpu_ok = bool(r.ok)
    nthr = max(1, min(threads, os.cpu_count() or 1))
    of = O.OracleForward(m)
    t0 = time.perf_counter()
    systems = _assemble_batch(of, m, m2, freqs, nthr)
    t_asm = time.perf_counter() - t0

    def solve(k):
        A, b2 = systems[k % 8]
        r_ = O.cocg13_single(A, b=None if src[k] == 0 else b2, precond="SSOR", resid=TOL, maxit=200000)
        return r_
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=nthr) as ex:
        sols = list(ex.map(solve, range(16)))
    cpu_s = (time.perf_counter() - t0 + t_asm) / 16
    cpu_it = sorted(s_["iter"] for s_ in sols)
    tr = O.true_residual(systems[0][0], sols[0]["x"])
    ref, _, _ = of.sites(sols[0]["x"], f[0])
    diff = float(np.abs(out[0] - ref[0]).max() / np.abs(ref[0]).max())
    return {"workload": f"20x20x20 hex box: {m.ntet} tets, 59660 edges, 25 sites; the same 16 systems (8 periods x 2 "
                        "patterns) on both sides",
            "gpu": {"s_per_solve": gpu_s, "iterations": gpu_it, "converged": gpu_ok,
                    "timed": "wall clock of assemble + solve + sites, 5 batches after 2 untimed"},
            "cpu_reference": {"s_per_solve": cpu_s, "iterations_min": cpu_it[0], "iterations_max": cpu_it[-1],
                              "converged": all(s_["error"] == 0 for s_ in sols), "threads": nthr,
                              "true_residual_system0": tr,
                              "timed": "wall clock of the oracle's assembly of the 8 x 2 systems + 16 COCG13_single "
                                       "(SSOR) solves to a recursive residual of 1e-8, one per thread"},
            "speedup": cpu_s / gpu_s, "site_rel_diff_system0": diff}


def cpu_baseline(job, seconds, plain):
    """The reference's solver (the oracle's COCG13_single with SSOR, one thread) on a bounded sample of the same
    workload: system 0 for about `seconds`, its measured time per iteration scaled by the iterations the same
    solver ran on the GPU in this run without converging (a lower bound on s/solve)."""
    from oracle import oracle as O
    m = job.m
    of = O.OracleForward(m)
    t0 = time.perf_counter()
    A = of.assemble(job.freqs[0])
    t_asm = time.perf_counter() - t0
    run = O.CocgSlices(A, precond="SSOR")
    t0 = time.perf_counter()
    run.advance(1)
    per = time.perf_counter() - t0
    k = max(3, int(seconds / max(per, 1e-6)))
    t0 = time.perf_counter()
    run.advance(k)
    per_it = (time.perf_counter() - t0) / k
    resid = run.resid
    run.close()
    it_gpu = plain["SSOR"]["iterations"] if plain else None
    conv = plain["SSOR"]["converged"] if plain else False
    value = t_asm + per_it * it_gpu if it_gpu else None
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "lower_bound": not conv,
            "ms_per_iteration": per_it * 1e3, "assembly_s": t_asm,
            "sample": f"oracle GENMAT+COPY_UL+BC of system 0 ({t_asm:.2f} s) + {k + 1} COCG13_single (SSOR) iterations "
                      f"on 1 thread ({per_it * 1e3:.1f} ms/iteration, recursive residual {resid:.3g} after them), "
                      f"scaled by the {it_gpu} iterations the same solver ran on the GPU in this run "
                      + ("to converge" if conv else "without converging (so a lower bound)")}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's solver (the oracle's COCG13_single with SSOR: the reference's CPU path for this
    step) on the GPU arm's workload: the same 16 systems, one Krylov run per system, spread over the
    host's threads.  The reference does not reach 1e-8 on this model within any bounded sample, so each
    step advances every system's run by a slice of iterations (the state carries over), and `value` is
    the measured time per system of the timed steps: a lower bound on its s/solve."""
    import concurrent.futures as cf
    ws, rank, _ = dist_info()
    if rank != 0:
        return
    from actfemtide_b200 import synth
    from oracle import oracle as O
    t_all = time.perf_counter()
    m = synth.large_model(seed=0)
    m2 = synth.large_model(seed=1000)
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    src = np.repeat([0, 1], 8)
    threads = max(1, min(16, os.cpu_count() or 1))
    of = O.OracleForward(m)
    systems = _assemble_batch(of, m, m2, freqs, threads)
    runs = [O.CocgSlices(systems[k % 8][0], b=None if src[k] == 0 else systems[k % 8][1], precond="SSOR")
            for k in range(16)]
    n = of.line.shape[0]
    nnz = n + 2 * len(of.pat[1])
    pool = cf.ThreadPoolExecutor(max_workers=threads)

    def advance_all(k):
        list(pool.map(lambda r: r.advance(k), runs))

    # calibrate the slice on the first warm-up step (one iteration of every system)
    t0 = time.perf_counter()
    advance_all(1)
    t1 = time.perf_counter() - t0
    slice_ = max(1, int(round(args.ref_step_seconds / max(t1, 1e-6))))
    for _ in range(max(0, args.warmup - 1)):
        advance_all(slice_)
    it0 = runs[0].iterations
    step_s = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        advance_all(slice_)
        step_s.append(time.perf_counter() - t0)
    timed = float(sum(step_s))
    its = runs[0].iterations - it0
    resid = [r.resid for r in runs]
    x0 = runs[0].close()
    for r in runs[1:]:
        r.close()
    tr0 = O.true_residual(systems[0][0], x0)
    pool.shutdown()
    value = timed / 16.0  # every system ran the whole timed region without converging
    per_it = timed / (16.0 * its)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * timed / args.steps, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "complex-f64" + (" COCG, complex-f32 preconditioner" if args.mt_precision == "pc32" else ""),
           "data": "synthetic (seeded Kuhn-split boxes, log-normal subsurface, tidal sources)",
           "config": shared_config(c1_desc(), 16, ws, nnz),
           "method": {"name": "reference", "solver": "COCG13_single with SSOR (the reference's iterative solver; "
                                                     "its production solver, MKL PARDISO, is a closed binary)",
                      "threads": threads},
           "impl": "reference",
           "lower_bound": True,
           "converged": False,
           "solver": {"iterations_per_system_timed": its, "iterations_per_system_total": its + it0,
                      "slice_iterations_per_step": slice_, "resid_recursive_min": float(min(resid)),
                      "resid_recursive_max": float(max(resid)), "true_residual_system0": tr0,
                      "ms_per_iteration_per_solve": 1e3 * per_it},
           "value_basis": (f"timed region {timed:.1f} s: {args.steps} steps x {slice_} iterations of all 16 systems on "
                           f"{threads} threads ({1e3 * per_it:.1f} ms per iteration per solve); value = timed / 16 "
                           f"solves, none converged (recursive residual {min(resid):.3g} to {max(resid):.3g}), so the "
                           "reference's s/solve is above it"),
           "extrapolated": {"s_per_solve": per_it * PLAIN_96["iterations"],
                            "basis": f"{1e3 * per_it:.1f} ms per iteration per solve x {PLAIN_96['iterations']} "
                                     "iterations, at which the same solver on a B200 had still not converged "
                                     "(residual 6.8e-5): also a lower bound"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{args.steps} timed slices of {slice_} iterations of the 16 systems"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "wall_s": time.perf_counter() - t_all}
    print(json.dumps(out), flush=True)


def mt_model(workload: str):
    """The MT workload: a Kuhn box with graded vertical cells, a log-normal earth around 10 Ohm m
    and a 2 Ohm m block, 8 frequencies from 1 mHz to 0.3 Hz, sites on a 20 x 20 grid."""
    from actfemtide_b200 import synth
    # cell growth per region chosen so the first cells at the surface are about 0.5 km (large),
    # 1 km (medium) thick, near the horizontal cell size
    dims, ra, re_ = {"large": ((96, 96, 24, 40), 1.11, 1.042), "medium": ((48, 48, 12, 20), 1.2, 1.1),
                     "small": ((20, 20, 8, 12), 1.25, 1.15)}[workload]
    freqs = np.logspace(-3, np.log10(0.3), 8)
    grid = np.linspace(-40.0, 40.0, 20)
    return synth.mt_box(*dims, ratio_air=ra, ratio_earth=re_, grf=True, seed=0, block_sigma=0.5, freqs=freqs,
                        site_grid=grid, name="mt%dx%dx%d" % (dims[0], dims[1], dims[2] + dims[3]))


def run_mt(args):
    """The 3-D MT forward (afem_mt_forward): per call the four side faces' 2-D TM solves at every
    frequency, the lifted 3-D systems of both polarisations, their batched solve, the sites and
    the impedances.  Inputs resident on the device; the call returns the impedances to the host."""
    import torch
    from actfemtide_b200 import synth
    from actfemtide_b200.forward import MTForward
    from oracle import oracle as O
    t_all = time.perf_counter()
    m = mt_model(args.workload)
    fw = MTForward(0)
    fw.load_mt_model(m)
    kw = dict(precond=args.precond or "HYBRID", precision=args.mt_precision, tol=TOL, maxit=args.maxit)
    for _ in range(args.warmup):
        r = fw.mt_forward(m.freqs, m.sites, **kw)
    torch.cuda.synchronize()
    clk = ClockSampler(0)
    clk.start()
    times, res = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = fw.mt_forward(m.freqs, m.sites, **kw)
        times.append(time.perf_counter() - t0)
        res.append(r.solve)
    clocks = clk.stop()
    # one more call with per-kernel events (outside the timed region)
    fw._check(fw._L.afem_set_profiling(fw.ctx, 1))
    fw.mt_forward(m.freqs, m.sites, **kw)
    prof = {}
    for i in range(fw._L.afem_profile_count(fw.ctx)):
        import ctypes as C
        buf = C.create_string_buffer(128); ms = C.c_double(); nl = C.c_long()
        fw._L.afem_profile_entry(fw.ctx, i, buf, 128, C.byref(ms), C.byref(nl))
        if not buf.value.decode().startswith("host_"):
            prof[buf.value.decode()] = round(ms.value, 3)
    fw._check(fw._L.afem_set_profiling(fw.ctx, 0))
    fw.close()
    ok = all(x.ok for x in res)
    pair = None
    if args.mt_pair:
        # a converged GPU / CPU pair on the 10 x 10 x 18 half-space model: the device against the oracle
        # with a direct (SuperLU) solve, the PARDISO stand-in of the reference
        ms_ = synth.mt_box(10, 10, 6, 12, sigma=0.1, freqs=[0.01], site_grid=(-20.0, 0.0, 20.0))
        with MTForward(0) as f2:
            f2.load_mt_model(ms_)
            f2.mt_forward(ms_.freqs, ms_.sites, **kw)
            t0 = time.perf_counter()
            rg = f2.mt_forward(ms_.freqs, ms_.sites, **kw)
            gpu_s = time.perf_counter() - t0
        line, n6 = O.mkline(ms_.node, ms_.n4)
        t0 = time.perf_counter()
        ro = O.MTOracle(ms_, line, n6).forward(ms_.freqs, ms_.sites)
        cpu_s = time.perf_counter() - t0
        pair = {"workload": "10x10x18 half-space, 1 frequency, 9 sites", "gpu_s": gpu_s, "cpu_oracle_direct_s": cpu_s,
                "z_rel_diff": float(np.abs(rg.z - ro["z"]).max() / np.abs(ro["z"]).max())}
    value = statistics.mean(times)
    out = {"metric": "s per 3-D MT forward (8 frequencies x 2 polarisations to 1e-8, 400 sites)",
           "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * value, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "complex-f64" + (" COCG, complex-f32 preconditioner" if args.mt_precision == "pc32" else ""),
           "data": "synthetic (seeded graded Kuhn box, log-normal earth, 2 Ohm m block)",
           "config": {"workload": f"{m.name}: {m.ntet} tets, 8 frequencies {m.freqs[0]:.3g}..{m.freqs[-1]:.3g} Hz, "
                                  f"{m.sites.shape[0]} sites", "method": kw["precond"],
                      "l2": "working set > 126 MB L2"},
           "solver": {"iterations": [x.iterations for x in res], "resid_true_max": max(x.resid_true for x in res),
                      "converged": ok},
           "phases_ms": prof, "clocks": clocks,
           "like_for_like_small": pair,
           "wall_s": time.perf_counter() - t_all}
    print(json.dumps(out), flush=True)
    if not ok and not args.allow_unconverged:
        sys.exit(3)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--method", default=DEFAULT_METHOD, choices=sorted(METHODS))
    p.add_argument("--precond", default=None, choices=["IC", "SSOR", "DIAG", "NONE", "LEARNED", "SSOR_MC", "HYBRID"],
                   help="override the method's preconditioner")
    p.add_argument("--prof-iters", type=int, default=256,
                   help="iteration cap of the per-kernel profiling pass (outside the timed region)")
    p.add_argument("--workload", default="large", choices=["large", "medium", "small"],
                   help="large: 96x96x64 hexes (the measured workload); medium: 48x48x32 (profiler captures); "
                        "small: 20x20x20 (quick checks)")
    p.add_argument("--allow-unconverged", action="store_true",
                   help="profiling runs with a small --maxit: accept solves stopped by the cap (not a bench number)")
    p.add_argument("--maxit", type=int, default=200000)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--plain-iters", type=int, default=1000,
                   help="cap of the bounded runs of the reference's solvers (SSOR, IC) on the same GPU; 0: skip")
    p.add_argument("--c0-pair", type=int, default=1, help="1: time the converged 20x20x20 GPU/CPU pair")
    p.add_argument("--c0-threads", type=int, default=16)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--ref-step-seconds", type=float, default=8.0,
                   help="reference arm: wall seconds of one step's slice of iterations")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--spmv-rpw", type=int, default=0, help="pin the SpMV's rows per warp (1, 2, 4, 8); 0: tuned")
    p.add_argument("--ckpt", default=None, help="learned methods: checkpoint path (without extension)")
    p.add_argument("--profile-case", action="store_true",
                   help="for profiler captures: one assembly and solve capped at --maxit, then exit (no bench line)")
    p.add_argument("--mt", action="store_true",
                   help="time the 3-D MT forward (afem_mt_forward) instead of the tidal step")
    p.add_argument("--mt-precision", default="pc32", choices=["fp64", "pc32"],
                   help="--mt: the preconditioner's precision (FP32 preconditioner by default, as the tidal step)")
    p.add_argument("--mt-pair", type=int, default=1, help="--mt: 1 times the converged GPU/CPU pair on a small model")
    args = p.parse_args()
    if args.mt:
        run_mt(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
