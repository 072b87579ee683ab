"""Benchmark of the per-level LBM step on B200 (one JSON line on rank 0).

Workload (the throughput roofline configuration): periodic 256^3 uniform box,
16.8M cells, one level, D3Q19 BGK, Taylor-Green vortex u0 = 0.05, tau = 0.55.
A step is one TimeLoop::advance_one (one fused pull-stream + collide launch).
`value` is whole-job MLUPS (all ranks) with the state resident in HBM; the
lattice (2 x 1.27 GB FP32) is larger than L2 (126 MB), so no L2 flush is
needed between steps.  `e2e` runs the same job through the C ABI from host
memory: the Taylor-Green fields (rho, u per cell) uploaded and turned into
the equilibrium state, K steps, the fields read back.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp32|fp16] [--n 256]

N > 1 (torchrun, one process per GPU): weak scaling over x slabs -- rank r
holds slab r (256^3) of the periodic (N 256) x 256 x 256 box and exchanges
its two ghost x planes with the neighbouring slabs before every step
(rank contexts over NCCL, octlb_gpu_create_part); timed as the max over
ranks of the device time.
"""
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

HBM_FALLBACK_GBS = 6650.0


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def committed_traffic(kernel_key):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary
    (profiles/ncu_traffic.txt lines: '<key> <bytes_per_launch>', each one
    256^3 launch captured on its own), or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel_key:
                try:
                    return float(parts[1])
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled around the timed region.

    Sampling starts before the region (the first sample is awaited, up to 5 s)
    and continues until one sample after it has arrived, so a region shorter
    than the sampling interval is still bracketed by the samples on either
    side.  summary() reports the samples that arrived during the region, or
    else the last one before and the first one after it (`bracketing`), or an
    `error` string when nvidia-smi gave none."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index, interval_ms=50):
        self.index = index
        self.interval_ms = interval_ms
        self.proc = None
        self.samples = []          # (arrival time, line)
        self.error = None
        self.t0 = self.t1 = None
        self._cv = threading.Condition()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval_ms)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        except Exception as e:  # no nvidia-smi
            self.error = f"nvidia-smi could not start: {e}"
            return self
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        with self._cv:
            self._cv.wait_for(lambda: self.samples or self.proc.poll() is not None, timeout=5.0)
        if not self.samples:
            self.error = "nvidia-smi gave no sample within 5 s"
        return self

    def _read(self):
        for line in self.proc.stdout:
            with self._cv:
                self.samples.append((time.perf_counter(), line.strip()))
                self._cv.notify_all()

    def start(self):
        self.t0 = time.perf_counter()

    def stop(self):
        self.t1 = time.perf_counter()

    def __exit__(self, *a):
        if self.t1 is None:
            self.stop()
        if self.proc:
            with self._cv:
                self._cv.wait_for(lambda: any(t > self.t1 for t, _ in self.samples) or self.proc.poll() is not None,
                                  timeout=2.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _parse(self, line):
        p = [x.strip() for x in line.split(",")]
        if len(p) < 7:
            return None
        try:
            sm, mx = float(p[0]), float(p[1])
        except ValueError:
            return None
        reasons = {nm for k, nm in enumerate(self.NAMES) if p[3 + k].lower().startswith("active")}
        return sm, mx, reasons

    def summary(self):
        parsed = [(t, self._parse(ln)) for t, ln in self.samples]
        parsed = [(t, v) for t, v in parsed if v is not None]
        if not parsed:
            return {"error": self.error or f"no parsable nvidia-smi sample ({len(self.samples)} lines)"}
        t0 = self.t0 if self.t0 is not None else parsed[0][0]
        t1 = self.t1 if self.t1 is not None else parsed[-1][0]
        inside = [v for t, v in parsed if t0 <= t <= t1]
        how = "during"
        if not inside:
            before = [v for t, v in parsed if t < t0][-1:]
            after = [v for t, v in parsed if t > t1][:1]
            inside = before + after
            how = "bracketing"
        sm = [v[0] for v in inside]
        reasons = sorted(set().union(*[v[2] for v in inside]))
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": inside[-1][1], "reasons": reasons,
                "samples": len(inside), "sampling": how, "region_ms": (t1 - t0) * 1e3}


def dist_setup(args):
    """Host plumbing of N > 1 (barriers, the max over ranks, the NCCL id):
    a gloo process group with a short timeout."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def slab_comm(ob, pg, world, rank):
    """The NCCL transport of the rank contexts (None on one GPU): rank 0 makes
    the id, the gloo group carries it to the others."""
    if pg is None:
        return None
    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")  # one node: the ranks meet on the loopback
    os.environ.setdefault("OCTLB_COMM_TIMEOUT_S", "120")
    obj = [ob.Comm.nccl_unique_id() if rank == 0 else None]
    pg.broadcast_object_list(obj, src=0)
    return ob.Comm.nccl(obj[0], world, rank)


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_reference_mlups(n, steps_budget_s=12.0, threads=None):
    """The reference's own BlockLattice<double> collide / fill_periodic_halo /
    stream (oracle/_ref; the C restatement when it is absent) on the host
    cores: `threads` independent periodic z-slabs covering the n^3 box."""
    from oracle import oracle
    import ctypes
    threads = threads or os.cpu_count() or 1
    L = oracle.load("ref")
    kind = "reference"
    if L is None:
        L = oracle.load("orc")
        kind = "port"
    slabs = max(1, min(threads, n // 4))
    nzs = n // slabs
    blocks = [oracle.Block(L, n, n, nzs) for _ in range(slabs)]
    for b in blocks:
        b.initialize(1.0, (0.01, 0.0, 0.0))
    omega = 1.0 / 0.55
    # calibrate: one step on one slab
    t0 = time.perf_counter()
    blocks[0].run_periodic(omega, 1)
    t_one = time.perf_counter() - t0
    per_step_par = t_one * slabs / min(threads, slabs)
    steps = max(1, int(steps_budget_s / max(per_step_par, 1e-6)))
    ths = [threading.Thread(target=b.run_periodic, args=(omega, steps)) for b in blocks]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    sec = time.perf_counter() - t0
    mlups = n * n * nzs * slabs * steps / sec / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": min(threads, slabs), "kind": kind,
            "sample": f"{steps} steps of {n}^3 as {slabs} periodic {n}x{n}x{nzs} slabs, FP64, "
                      f"{min(threads, slabs)} threads ({sec:.1f} s)"}


class CpuSlabs:
    """The reference's BlockLattice<double> collide / fill_periodic_halo /
    stream (oracle/_ref; the C restatement when it is absent) on `slabs`
    independent periodic n x n x nz slabs, one host thread each, allocated
    once."""

    def __init__(self, n, nz, slabs):
        from oracle import oracle
        L = oracle.load("ref")
        self.kind = "reference"
        if L is None:
            L = oracle.load("orc")
            self.kind = "port"
        self.n, self.nz, self.slabs = n, nz, slabs
        self.blocks = [oracle.Block(L, n, n, nz) for _ in range(slabs)]
        for b in self.blocks:
            b.initialize(1.0, (0.01, 0.0, 0.0))
        self.omega = 1.0 / 0.55

    def step(self):
        """One step of every slab in parallel; seconds."""
        ths = [threading.Thread(target=b.run_periodic, args=(self.omega, 1)) for b in self.blocks]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        return time.perf_counter() - t0

    def cells(self):
        return self.n * self.n * self.nz * self.slabs


def run_reference_arm(args, world, rank, pg):
    """The reference's CPU path on the host cores, each step one step of a
    bounded sample of the n^3 box: as many periodic n x n x nz slabs as
    threads (n^3 when one step of the whole box fits the per-step budget;
    thinner slabs otherwise), so the K + W steps end within about 150 s."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = args.n
    slabs = max(1, min(threads, n // 4))
    nz_full = n // slabs
    per = min(args.ref_seconds, 150.0 / max(1, args.steps + args.warmup))
    probe = CpuSlabs(n, nz_full, slabs)
    probe.step()
    t_full = probe.step()
    nz = nz_full if t_full <= per else max(1, int(nz_full * per / t_full))
    ref = probe if nz == nz_full else CpuSlabs(n, nz, slabs)
    del probe
    for _ in range(args.warmup):
        ref.step()
    vals = [ref.cells() / ref.step() / 1e6 for _ in range(args.steps)]
    v = statistics.median(vals)
    sample = (f"one step per timed step of {slabs} periodic {n}x{n}x{nz} slabs "
              f"({ref.cells() / n ** 3:.3f} of the {n}^3 box), FP64, {slabs} threads")
    out = {"metric": "MLUPS", "value": v, "unit": "MLUPS", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"tgv_periodic_{args.n}^3", "cells": args.n ** 3, "tau": 0.55, "u0": 0.05},
           "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": slabs, "kind": ref.kind, "sample": sample},
           "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def accuracy_vs_fp64(ob, cases, n, steps, fields_fp32, threads=None):
    """Errors of the headline workload against FP64 runs of the reference's
    algorithm (each result states its error against an FP64 run):

    * the 256^3 box after `steps` steps (the e2e run's fields for FP32, a
      separate run for FP16) against the oracle's C restatement of the
      reference BlockLattice<double> collide / fill_periodic_halo / stream
      (pinned to the reference build at 1e-13), run on the host threads;
    * the same physics at 64^3 over 1,000 steps: the kinetic-energy history
      (every 10 steps) and the final fields on a 16^3 lattice of cells against
      the reference's own BlockLattice<double> run
      (tests/golden/tgv64_reference.npz)."""
    from oracle import oracle
    orc = oracle.load("orc")
    rho0, u0 = cases.tgv_fields(n, n, n, 0.05)
    init = ob.feq(rho0, u0)
    blk = oracle.Block(orc, n)
    blk.set_core(init)
    del init
    t0 = time.perf_counter()
    blk.run_periodic_mt(1.0 / 0.55, steps, threads)
    cpu_s = time.perf_counter() - t0
    rho_r, u_r = blk.fields()
    del blk
    out = {"tgv256": {"steps": steps, "reference": "C restatement of BlockLattice<double>, FP64",
                      "host_seconds": cpu_s}}

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    for name, prec in (("fp32", ob.FP32), ("fp16", ob.FP16_SHIFTED)):
        if name == "fp32" and fields_fp32 is not None:
            rho_g, u_g = fields_fp32
        else:
            lat = ob.GpuLattice(mesh, 1.0 / 0.55, precision=prec)
            lat.set_equilibrium(rho0.reshape(-1), u0.reshape(-1, 3))
            lat.advance(steps)
            rho_g, u_g = lat.get_fields()
            lat.close()
        out["tgv256"][name] = {"rel_err_rho_max": rel(np.asarray(rho_g).reshape(rho_r.shape), rho_r),
                               "rel_err_u_max": rel(np.asarray(u_g).reshape(u_r.shape), u_r)}
    del rho_r, u_r
    g = np.load(os.path.join(ROOT, "tests", "golden", "tgv64_reference.npz"))
    m, every, total = int(g["n"]), int(g["every"]), int(g["steps"])
    mesh64, init64, info64 = cases.tgv_periodic(m, u0=float(g["u0"]), tau=float(g["tau"]))
    out["tgv64_1000"] = {"reference": "BlockLattice<double> (oracle/_ref), FP64"}
    lat_ke = {}
    for name, prec in (("fp32", ob.FP32), ("fp16", ob.FP16_SHIFTED)):
        lat = ob.GpuLattice(mesh64, info64["omega"], precision=prec, init_pops=init64)
        ke = []
        for k in range(total // every + 1):
            if k:
                lat.advance(every)
            rho, u = lat.get_fields()
            ke.append(0.5 * float(np.sum(rho * np.sum(u * u, axis=-1))))
        lat.close()
        sl = (0, slice(2, None, 4), slice(2, None, 4), slice(2, None, 4))
        ke = np.array(ke)
        lat_ke[name] = ke
        out["tgv64_1000"][name] = {
            "ke_rel_err_max": float(np.max(np.abs(ke - g["ke"]) / g["ke"])),
            "ke_decay": float(ke[-1] / ke[0]), "ke_decay_reference": float(g["ke"][-1] / g["ke"][0]),
            "rel_err_u_sampled": rel(u[sl], g["sample_u"]), "rel_err_rho_sampled": rel(rho[sl], g["sample_rho"])}
    return out


def aa_measurements(ob, cases, torch, n, steps, warmup, peak):
    """The same periodic box in the one-buffer AA stream order (in-place
    steps alternating between a neighbour pull / push-back and a step on the
    cell's own slots; bitwise equal results, tests/test_gpu_tgv.py): MLUPS,
    the fraction of the measured copy peak at the same algorithmic bytes per
    update, and the device bytes of the population state (half the AB
    order's)."""
    out = {}
    for pn, prec in (("fp32", ob.FP32), ("fp16", ob.FP16_SHIFTED)):
        mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
        lat = ob.GpuLattice(mesh, info["omega"], precision=prec, init_pops=init, stream_order=ob.ORDER_AA)
        st = torch.cuda.Stream()
        lat.set_stream(st.cuda_stream)
        lat.advance(warmup + (warmup % 2))  # an even count: the natural layout
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lat.advance(steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        _, lups = lat.step_stats()
        bpl = 152 if pn == "fp32" else 76
        out[pn] = {"mlups": lups / ms / 1e3, "ms_per_step": ms, "bytes_per_lu": bpl,
                   "frac": bpl * lups / (ms * 1e-3) / 1e9 / peak,
                   "state_bytes": n ** 3 * 19 * (4 if pn == "fp32" else 2)}
        lat.close()
        del lat
        torch.cuda.empty_cache()
    return out


def cavity3d_gate(ob, cases, torch):
    """The reference's cavity3d example and its accuracy gate
    (tests/integration/test_cavity3d_serial.cpp:56-82): one 31^3 block,
    tau = 0.509, lid 0.1, InterpolatedVelocity walls, ConstRhoBGK, 5,269
    steps; the centerline u / u_lid against OpenLB's values (relative L2,
    gate 0.02) and against the reference TimeLoop's FP64 profile
    (tests/golden/cavity3d_centerline.json), with the steps' MLUPS (CUDA
    events; a small, launch-bound case)."""
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "tests", "golden", "cavity3d_centerline.json")) as f:
        g = json.load(f)
    mesh, init, info = cases.cavity3d(g["resolution"], g["tau"], g["phys_length"], g["phys_velocity"],
                                      g["phys_viscosity"])
    out = {"steps": g["steps"], "cells": mesh.n ** 3, "gate": 0.02,
           "reference_fp64_l2_vs_openlb": g["reference_fp64_l2"]}
    for pn, prec in (("fp32", ob.FP32), ("fp16", ob.FP16_SHIFTED)):
        lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, info["types"]), info["omega"], precision=prec, init_pops=init)
        lat.set_const_rho(True)
        lat.set_fd_boundary(info["types"], info["u_wall"])
        st = torch.cuda.Stream()
        lat.set_stream(st.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lat.advance(g["steps"])
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / g["steps"]
        _, u = lat.get_fields()
        lat.close()
        prof = cases.cavity3d_centerline(u[0][..., 0], info, g["y_over_h"])
        out[pn] = {"l2_vs_openlb": cases.relative_l2(prof, g["openlb_u_over_lid"]),
                   "max_dev_vs_fp64_profile": float(np.max(np.abs(prof - np.array(g["reference_fp64_u_over_lid"])))),
                   "ms_per_step": ms, "mlups": mesh.n ** 3 / ms / 1e3}
    return out


def forest_measurements(ob, cases, torch, peak):
    """The forest configurations beside the headline line: MLUPS of the
    two-level AMR cavity (64^3 + band under the lid) and of the three-level
    cylinder (256x64x64, D = 16, Re = 100) in FP32 and FP16-shifted storage
    (an advance_one = a step; CUDA events on the context's stream), the FP16 /
    FP32 ratio, the cylinder's time-averaged drag over its last 5,000 finest
    steps against the FP64 run of the reference TimeLoop
    (tests/golden/long_c3_cylinder.npz), and the adjoint's cost on its own
    configuration (forward + reverse sweep vs the forward alone, steady state)
    with its gradients against FP64 finite differences
    (tests/golden/adjoint_c5.npz)."""
    here = os.path.dirname(os.path.abspath(__file__))
    out = {}
    cfgs = {
        "amr_cavity_64": (lambda: cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8),
                          ob.STREAM_ROTATE, False),
        "cylinder_256x64x64": (lambda: cases.cylinder_forest(), ob.STREAM_LINKS, True),
        # the same channel at twice the resolution per axis (D = 32, 8x the
        # cells): how the FP16 / FP32 ratio grows once bytes dominate the
        # per-launch latency
        "cylinder_512x128x128": (lambda: cases.cylinder_forest(length=512, height=128, diameter=32.0,
                                                               center=(128.0, 64.0)), ob.STREAM_LINKS, True),
        # the 256x64x64 channel on 16^3 blocks: an eighth of the blocks, fewer
        # shell cells per block, a finest level that covers more of the box
        "cylinder_256x64x64_n16": (lambda: cases.cylinder_forest(n=16), ob.STREAM_LINKS, True),
        # single-level 128^3 cavity (the reference's cavity3d collision),
        # ConstRhoBGK; BGK on the same mesh beside it
        "const_rho_cavity_128": (lambda: cases.cavity_forest(cells=128, n=8, lid=0.05, tau=0.56),
                                 ob.STREAM_ROTATE, False),
    }
    for name, (fn, mode, drag) in cfgs.items():
        mesh, init, info = fn()
        r = {}
        const_rho = name.startswith("const_rho")
        for pn, prec in (("fp32", ob.FP32), ("fp16", ob.FP16_SHIFTED)) + ((("bgk_fp32", ob.FP32),) if const_rho else ()):
            lat = ob.GpuLattice(mesh, info["omega"], precision=prec, stream_mode=mode, drag=drag, init_pops=init)
            if const_rho and pn != "bgk_fp32":
                lat.set_const_rho(True)
            st = torch.cuda.Stream()
            lat.set_stream(st.cuda_stream)
            lat.advance(5)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            K = 100
            e0.record(st)
            lat.advance(K)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / K
            launches, lups = lat.step_stats()
            bpl = 76 if pn == "fp16" else 152
            # both population buffers of every block core (halo pages aside):
            # below the 126 MB L2 the step's bytes need not reach HBM at all
            cells = int(mesh.n_blocks) * int(mesh.n) ** 3
            r[pn] = {"mlups": lups / ms / 1e3, "ms_per_step": ms, "launches_per_step": int(launches),
                     "hbm_frac": bpl * lups / (ms * 1e-3) / 1e9 / peak,
                     "lattice_mb": 2 * cells * 19 * (2 if pn == "fp16" else 4) / 1e6}
            if name == "cylinder_256x64x64":
                g = np.load(os.path.join(here, "tests", "golden", "long_c3_cylinder.npz"))["force"]
                lat.close()
                lat = ob.GpuLattice(mesh, info["omega"], precision=prec, stream_mode=mode, drag=True, init_pops=init)
                steps = len(g)
                last = len(g) // 4
                lat.advance(steps - last)
                lat.force_reset()
                lat.advance(last)
                fs, nsteps = lat.force_sum()
                ref = g[steps - last:, 0].mean()
                r[pn]["drag_rel_err_vs_fp64"] = float(abs(fs[0] / nsteps - ref) / abs(ref))
            lat.close()
        r["fp16_speedup"] = r["fp16"]["mlups"] / r["fp32"]["mlups"]
        if const_rho:
            r["const_rho_over_bgk_fp32"] = r["fp32"]["mlups"] / r["bgk_fp32"]["mlups"]
        out[name] = r
    # adjoint
    case, directions = cases.adjoint_channel, cases.adjoint_directions
    g = np.load(os.path.join(here, "tests", "golden", "adjoint_c5.npz"))
    steps, window = int(g["steps"]), int(g["window"])
    mesh, init, info = case()
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32, stream_mode=ob.STREAM_LINKS, drag=True,
                        init_pops=init)
    lat.advance(3)
    lat.synchronize()
    t_fwd = float("inf")
    for _ in range(3):  # best of three
        t0 = time.perf_counter()
        lat.advance(steps)
        lat.synchronize()
        t_fwd = min(t_fwd, time.perf_counter() - t0)
    lat.close()
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32, stream_mode=ob.STREAM_LINKS, drag=True,
                        init_pops=init)
    # the first call (from the initial state) gives the checked gradients and
    # captures the sweep's graphs; the next ones, from the forward's final
    # state, reuse them and are timed (the same work; best of three)
    J, du, dtau, gF = lat.adjoint(steps, window, 16)
    lat.synchronize()
    t_adj = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        lat.adjoint(steps, window, 16)
        lat.synchronize()
        t_adj = min(t_adj, time.perf_counter() - t0)
    lat.close()
    d = directions(mesh)
    gdir = np.array([np.sum(gF * d[k]) for k in range(len(d))])
    out["adjoint_channel_128x32x32"] = {
        "advance_one_calls": steps, "window": window, "checkpoint_interval": 16,
        "forward_s": t_fwd, "forward_plus_adjoint_s": t_adj,
        "adjoint_cost_ratio": (t_adj - t_fwd) / t_fwd,
        "rel_err_vs_fp64_fd": {"u_max": float(abs(du - g["dJ_du"]) / abs(g["dJ_du"])),
                               "tau": float(abs(dtau - g["dJ_dtau"]) / abs(g["dJ_dtau"])),
                               "body_force_dirs_max": float(np.max(np.abs(gdir - g["dJ_dir"]) / np.abs(g["dJ_dir"])))},
    }
    tpath = os.path.join(here, "tests", "golden", "adjoint_c5_tlm.npz")
    if os.path.exists(tpath):  # exact FP64 derivatives of the reference (tangent-linear)
        t = np.load(tpath)
        out["adjoint_channel_128x32x32"]["rel_err_vs_fp64_tangent_linear"] = {
            "u_max": float(abs(du - t["dJ_du"]) / abs(t["dJ_du"])),
            "tau": float(abs(dtau - t["dJ_dtau"]) / abs(t["dJ_dtau"])),
            "body_force_dirs_max": float(np.max(np.abs(gdir - t["dJ_dir"]) / np.abs(t["dJ_dir"])))}
    return out


def run_single_case(args, ob, cases, torch):
    """One forest case alone (for launch lists and ncu captures): --warmup
    then --steps advance_one calls, or one adjoint sweep over --steps calls."""
    prec = ob.FP32 if args.precision == "fp32" else ob.FP16_SHIFTED
    if args.case == "adjoint":
        mesh, init, info = cases.adjoint_channel()
        lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32, stream_mode=ob.STREAM_LINKS, drag=True,
                            init_pops=init)
        t0 = time.perf_counter()
        J = lat.adjoint(args.steps, max(1, args.steps // 4), 16, force_grad=False)[0]
        print(json.dumps({"case": "adjoint", "steps": args.steps, "seconds": time.perf_counter() - t0, "J": J}))
        return
    const_rho = False
    if args.case == "amr_cavity_64":
        mesh, init, info = cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8)
        mode, drag = ob.STREAM_ROTATE, False
    elif args.case == "const_rho_cavity_128":
        mesh, init, info = cases.cavity_forest(cells=128, n=8, lid=0.05, tau=0.56)
        mode, drag, const_rho = ob.STREAM_ROTATE, False, True
    elif args.case == "cylinder_512":
        mesh, init, info = cases.cylinder_forest(length=512, height=128, diameter=32.0, center=(128.0, 64.0))
        mode, drag = ob.STREAM_LINKS, True
    else:
        mesh, init, info = cases.cylinder_forest()
        mode, drag = ob.STREAM_LINKS, True
    lat = ob.GpuLattice(mesh, info["omega"], precision=prec, stream_mode=mode, drag=drag, init_pops=init)
    if const_rho:
        lat.set_const_rho(True)
    st = torch.cuda.Stream()
    lat.set_stream(st.cuda_stream)
    lat.advance(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    lat.advance(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches, lups = lat.step_stats()
    print(json.dumps({"case": args.case, "storage": args.precision, "steps": args.steps, "ms_per_step": ms,
                      "mlups": lups / ms / 1e3, "launches_per_step": launches}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-forest", action="store_true", help="skip the forest / adjoint measurements")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the errors against the FP64 runs")
    ap.add_argument("--no-aa", action="store_true", help="skip the one-buffer (AA order) measurement")
    ap.add_argument("--case", default="tgv", choices=["tgv", "amr_cavity_64", "cylinder", "cylinder_512", "adjoint",
                                                      "const_rho_cavity_128"],
                    help="tgv: the headline line; otherwise run only that case for --steps advance_one "
                         "calls (or one adjoint sweep of --steps calls) and print its timing (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local, pg = dist_setup(args)

    if args.impl == "reference":
        run_reference_arm(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    import octlb_b200 as ob
    from octlb_b200 import cases
    if args.case != "tgv":
        run_single_case(args, ob, cases, torch)
        if pg is not None:
            pg.destroy_process_group()
        return

    n = args.n
    results = {}
    comm = slab_comm(ob, pg, world, rank)
    part = None if comm is None else (rank, np.zeros(1, np.int32), comm)
    for prec_name in (["fp32", "fp16"] if args.precision == "fp32" else ["fp16", "fp32"]):
        prec = ob.FP32 if prec_name == "fp32" else ob.FP16_SHIFTED
        mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
        lat = ob.GpuLattice(mesh, info["omega"], precision=prec, init_pops=init, part=part)
        # A dedicated (non-default) stream shared by the context and the events.
        stream = torch.cuda.Stream()
        lat.set_stream(stream.cuda_stream)
        launches, lups = lat.step_stats()
        lat.advance(args.warmup)
        torch.cuda.synchronize()
        barrier(pg)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as cs:
            cs.start()
            e0.record(stream)
            lat.advance(args.steps)
            e1.record(stream)
            lat.synchronize()  # bounded under NCCL
            torch.cuda.synchronize()
            cs.stop()
        barrier(pg)
        ms = e0.elapsed_time(e1)
        ms_max = max_over_ranks(pg, ms)
        ms_step = ms_max / args.steps
        mlups = world * lups * args.steps / (ms_max * 1e-3) / 1e6
        bytes_per_lu = 152 if prec == ob.FP32 else 76
        results[prec_name] = {"mlups": mlups, "ms_step": ms_step, "launches": launches,
                              "bytes_per_lu": bytes_per_lu, "clocks": cs.summary(), "lups": lups}
        # e2e: the same job through the C ABI from host memory: the
        # Taylor-Green fields (rho, u per cell, FP64, pinned) uploaded and
        # turned into the equilibrium state, K steps, rho / u read back
        if prec_name == args.precision:
            rho0, u0 = cases.tgv_fields(n, n, n, 0.05)
            rho_in = torch.from_numpy(np.ascontiguousarray(rho0.reshape(-1))).pin_memory().numpy()
            u_in = torch.from_numpy(np.ascontiguousarray(u0.reshape(-1))).pin_memory().numpy()
            del rho0, u0
            rho_host = torch.empty(n ** 3, dtype=torch.float64).pin_memory().numpy()
            u_host = torch.empty(3 * n ** 3, dtype=torch.float64).pin_memory().numpy()
            e2e_steps = args.steps
            # untimed warm-up of the same calls (first-use costs of the
            # staging buffers and pinned pages)
            lat.set_equilibrium(rho_in, u_in)
            lat.advance(args.warmup)
            lat.get_fields(rho_host, u_host)
            torch.cuda.synchronize()
            barrier(pg)
            t0 = time.perf_counter()
            lat.set_equilibrium(rho_in, u_in)
            lat.advance(e2e_steps)
            rho, u = lat.get_fields(rho_host, u_host)
            t1 = time.perf_counter()
            e2e_s = max_over_ranks(pg, t1 - t0)
            results["e2e"] = {"value": world * lups * e2e_steps / e2e_s / 1e6, "unit": "MLUPS",
                              "h2d_bytes_per_step": int((rho_in.nbytes + u_in.nbytes) / e2e_steps),
                              "d2h_bytes_per_step": int((rho.nbytes + u.nbytes) / e2e_steps),
                              "steps": e2e_steps, "seconds": e2e_s}
            if e2e_steps <= 20 and prec_name == "fp32":
                results["e2e_fields"] = (rho.copy(), u.copy())
        lat.close()
        del lat
        torch.cuda.empty_cache()

    main_r = results[args.precision]
    peak, peak_kind = measured_peak()
    # algorithmic bytes of one launch (per GPU) / average launch time
    achieved = main_r["bytes_per_lu"] * main_r["lups"] / (main_r["ms_step"] * 1e-3) / 1e9
    key = f"k_step_periodic_{args.precision}_{n}"
    traffic = committed_traffic(key)
    out = {
        "metric": "MLUPS", "value": main_r["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main_r["ms_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"tgv_periodic_{n}^3" + (f" per rank, x slabs of ({world}x{n})x{n}x{n}" if world > 1 else ""),
                   "cells": n ** 3 * world, "tau": 0.55, "u0": 0.05,
                   "storage": args.precision, "parallelism": f"xslab{world}" if world > 1 else "single",
                   "l2": "lattice 2x{:.2f} GB > L2, no flush".format(n ** 3 * 19 * (4 if args.precision == 'fp32' else 2) / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "bytes_per_lu": main_r["bytes_per_lu"], "peak_kind": peak_kind},
        "gpu_launches": int(main_r["launches"] * args.steps),
        "clocks": main_r["clocks"],
        "e2e": {k: v for k, v in results["e2e"].items() if k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step")},
        "fp16_shifted": {"mlups": results["fp16"]["mlups"], "ms_per_step": results["fp16"]["ms_step"],
                         "bytes_per_lu": 76, "speedup_vs_fp32": results["fp16"]["mlups"] / results["fp32"]["mlups"]},
    }
    if rank == 0 and world == 1 and not args.no_accuracy:
        m = min(args.steps, 20)
        out["accuracy_vs_fp64"] = accuracy_vs_fp64(ob, cases, n, m,
                                                   results.get("e2e_fields") if m == args.steps else None)
    if rank == 0 and world == 1 and not args.no_aa:
        out["aa_one_buffer"] = aa_measurements(ob, cases, torch, n, args.steps, args.warmup, peak)
    if rank == 0 and world == 1 and not args.no_forest:
        out["forest"] = forest_measurements(ob, cases, torch, peak)
        out["cavity3d_gate"] = cavity3d_gate(ob, cases, torch)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_reference_mlups(n, steps_budget_s=args.ref_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if comm is not None:
        barrier(pg)
        comm.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
