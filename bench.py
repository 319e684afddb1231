#!/usr/bin/env python
"""Benchmark of the CGFD3D elastic time loop on B200.

Metric: Gcell-stage updates/s = ni*nj*nk (physical points incl. PML, ghosts excluded)
x 4 RK stages x steps / time. One "step" is one time step (4 RK stages) of the plain FP32
isotropic path on the 480x480x240 workload (50 m, CFS-PML 20, layered + 5% von Karman
medium, one Ricker moment source fc=4 Hz, 400 surface stations), with every input resident
in HBM. The wavefield (4 x 9 x 58 M floats) is far larger than L2, so no flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]

Under torchrun each rank runs an independent replica on its own GPU (no collective on the
data path); rank 0 prints one JSON line. --impl reference times the CPU restatement of the
reference's time loop (the reference has no CPU solver of its own) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gpu-cgfd3d-elastic_b200"))

import numpy as np  # noqa: E402

METRIC = "Gcell-stage updates/s"
UNIT = "Gcell-stage/s"
# algorithmic bytes per cell-stage of the fused RK4 stage (FP32): 36 wavefield accesses
# (stage 0: 9 reads + 18 writes; stages 1-2: 27 + 18; stage 3: 18 + 9; averaged) plus the
# coefficients read once per stage (iso 12, VTI 15, aniso 31).
BYTES_PER_CELL_STAGE = {"iso": 36 * 4 + 12 * 4, "vti": 36 * 4 + 15 * 4, "aniso": 36 * 4 + 31 * 4}

WORKLOADS = {
    # name: (ni, nj, nk, dh, nsteps, npml, nsta_x, nsta_y, fc, perturb_std)
    "480x480x240": (480, 480, 240, 50.0, 3000, 20, 20, 20, 4.0, 0.05),
    "100x100x60": (100, 100, 60, 100.0, 500, 12, 5, 5, 2.0, 0.0),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="480x480x240", choices=sorted(WORKLOADS))
    ap.add_argument("--grid", type=int, nargs=3, default=None, help="override ni nj nk (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--zchunk", type=int, default=0, help="fixed z chunk (skips the autotuner)")
    ap.add_argument("--tile-shape", type=int, default=-1, help="fixed bulk tile shape 0/1 (with --zchunk: no autotuner)")
    ap.add_argument("--no-autotune", action="store_true", help="default tile shape and z chunk")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched / mixed-precision section")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving section")
    ap.add_argument("--no-media", action="store_true", help="skip the VTI / aniso section")
    # profiling case (no JSON line): K steps of direct launches on the chosen grid, for ncu
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many directly launched steps of the profiling case and exit")
    ap.add_argument("--pml-faces", default="x1,x2,y1,y2,z1",
                    help="profiling case: CFS-PML faces (comma list of x1,x2,y1,y2,z1, or none)")
    ap.add_argument("--pml-layers", type=int, default=0, help="profiling case: layers per face (0: workload's)")
    ap.add_argument("--shots", type=int, default=1, help="profiling case: shots of a batched problem")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "u16coef", "fp16wave", "fp64"],
                    help="profiling case: storage precision")
    ap.add_argument("--medium", default="iso", choices=["iso", "ac"],
                    help="profiling case: elastic iso or acoustic medium (the same layers' vp and rho)")
    return ap.parse_args()


def profile_run(args):
    """Profiling case for ncu: the workload (or --grid) with the chosen CFS-PML faces and width,
    shots and precision, `--profile-steps` steps launched directly (one launch per kernel, no
    graph). Prints the face points and the kernels' cell counts."""
    import dataclasses
    from cgfd_b200 import synth, Simulation, CGFD_PREC_FP32, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE, CGFD_PREC_FP64
    p = build_problem(args)
    nl = args.pml_layers or WORKLOADS[args.workload][5]
    face = dict(p.pml[0][0], num_layers=nl)
    names = [f for f in args.pml_faces.split(",") if f and f != "none"]
    slots = {"x1": (0, 0), "x2": (0, 1), "y1": (1, 0), "y2": (1, 1), "z1": (2, 0)}
    p.pml = [[None, None], [None, None], [None, None]]
    for f in names:
        a, sd = slots[f]
        p.pml[a][sd] = face
    p.precision = {"fp32": CGFD_PREC_FP32, "u16coef": CGFD_PREC_U16_COEF, "fp16wave": CGFD_PREC_FP16_WAVE,
                   "fp64": CGFD_PREC_FP64}[args.precision]
    if args.shots > 1:
        rng = np.random.default_rng(78)
        mk = synth.ac_sources if args.medium == "ac" else synth.dc_sources
        shots = [mk(p.coord, p.ni, p.nj, 1, rng, depth_range=(1000.0, 3000.0), fc_range=(2.0, 5.0),
                    stf_length=p.nt_total * p.dt) for _ in range(args.shots)]
        sim = Simulation(p, shots=shots)
    else:
        sim = Simulation(p)
    sim.set_graph_mode(0)
    sim.run(args.profile_steps)
    # per-kernel CUDA-event times of 8 more steps (not for use under ncu)
    sim.set_timing(True)
    sim.timing(reset=True)
    sim.run(8)
    sim.synchronize()
    bulk_ms, bulk_n = sim.timing(reset=True)["bulk"]
    sim.set_timing(False)
    pts = 0
    for f in names:
        n = [p.ni, p.nj, p.nk]
        n[slots[f][0]] = nl + 1
        pts += n[0] * n[1] * n[2]
    bulk = p.ni * p.nj * (p.nk if args.medium == "ac" or not p.free_top else p.nk - 4)
    print(f"profile case {p.ni}x{p.nj}x{p.nk} medium={args.medium} faces={names or 'none'} layers={nl} "
          f"shots={args.shots} precision={args.precision}: {args.profile_steps} steps, face points {pts}, "
          f"bulk cells {bulk}; event-timed bulk stage {bulk_ms / max(bulk_n, 1):.4f} ms", flush=True)
    sim.close()
    return 0


def max_over_ranks(x, dist, device):
    """Max of a per-rank float over all ranks (timings: the slowest rank sets the job time).
    Every rank must call it at the same point; device is the tensor device of the backend
    ("cuda:<n>" for nccl, "cpu" for gloo)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, cells, steps, ms):
    """Whole-job Gcell-stage/s: every rank advances its own replica of `cells` for `steps`
    steps (4 RK stages each) within the max-over-ranks time `ms`."""
    return world * cells * 4 * steps / (ms * 1e-3) / 1e9


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def build_problem(args, device=0, nk_override=None):
    from cgfd_b200 import synth
    ni, nj, nk, dh, nsteps, npml, sx, sy, fc, pert = WORKLOADS[args.workload]
    if args.grid:
        ni, nj, nk = args.grid
    if nk_override:
        nk = nk_override
    p = synth.make_problem(ni, nj, nk, dh, nsteps, dt=None, medium=getattr(args, "medium", "iso"), npml=npml,
                           nsrc=1, sta_grid=(sx, sy),
                           fc=fc, seed=2024, perturb_std=pert, corr=1000.0, hurst=0.3,
                           src_depth=(2000.0, 2000.0), center_src=True)
    p.device = device
    return p


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload, cells_per_launch, shape, zchunk):
    """DRAM bytes per bulk-kernel launch (one RK stage) from the committed ncu summary, scaled
    by cells: the capture of the same tile shape with the nearest z chunk (the tile choice it
    was taken with is returned beside it); (None, None) when that shape has no capture."""
    path = os.path.join(ROOT, "profiles", "k_stage_bulk_iso.md")
    try:
        vals = {}
        with open(path) as f:
            for ln in f:
                if ":" in ln and ln.strip().startswith("- "):
                    k, v = ln.strip()[2:].split(":", 1)
                    vals[k.strip()] = v.strip().split()[0]
        pre = f"dram_bytes_per_launch_shape{shape}_zchunk"
        caps = {int(k[len(pre):]): float(v) for k, v in vals.items() if k.startswith(pre)}
        z = min(caps, key=lambda c: abs(c - zchunk))
        return caps[z] * cells_per_launch / float(vals["cells_per_launch"]), f"tile shape {shape}, z chunk {z}"
    except Exception:
        return None, None


def _time_steps(sim, steps, warm=8):
    """ms per step of `steps` graph-replayed steps after `warm` (>= 8 captures every graph)."""
    import torch
    st = torch.cuda.ExternalStream(sim.stream)
    sim.enqueue(warm)
    sim.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.enqueue(steps)
    e1.record(st)
    e1.synchronize()
    sim.synchronize()
    return e0.elapsed_time(e1) / steps


def batched_mixed(local, steps=16):
    """Batched sources and storage precision on the 256x256x128 batch workload (50 m, CFS-PML
    20, layered + 5% von Karman iso medium, 32 random double-couple sources at 1-6 km depth,
    fc 2-5 Hz, 200 surface stations): source x time steps per second of the plain FP32 path
    (one source per simulation) against batches of S shots in FP32, in 16-bit fixed-point
    coefficients and in the mixed mode (16-bit coefficients + FP16 RK stage levels), each with
    its seismogram error against the FP64 build of the same kernels. Every problem is autotuned
    (tile shape, z chunk and, for batches, the shot group) before it is timed."""
    import dataclasses
    from cgfd_b200 import synth, Simulation, CGFD_PREC_FP32, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE
    ni, nj, nk, nsteps = 256, 256, 128, 1500
    p = synth.make_problem(ni, nj, nk, 50.0, nsteps, dt=None, medium="iso", npml=20, nsrc=0, sta_grid=(20, 10),
                           fc=3.0, seed=77, perturb_std=0.05, corr=1000.0, hurst=0.3)
    p.device = local
    rng = np.random.default_rng(78)
    shots = [synth.dc_sources(p.coord, ni, nj, 1, rng, depth_range=(1000.0, 6000.0), fc_range=(2.0, 5.0),
                              stf_length=p.nt_total * p.dt) for _ in range(32)]
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import rel_l2
    from cgfd_b200 import CGFD_PREC_FP64
    out = {"workload": f"{ni}x{nj}x{nk}", "sources": 32, "stations": 200, "steps_timed": steps,
           "unit": "source-steps/s"}
    nacc = 400  # steps of the accuracy comparison (arrivals reach the stations)
    # the FP64 build of the kernels on shot 0: the reference of every error below
    s64 = Simulation(dataclasses.replace(p, src=shots[0], precision=CGFD_PREC_FP64))
    s64.run(nacc)
    ref = s64.seismograms()[:, :, :nacc]
    s64.close()
    one = Simulation(dataclasses.replace(p, src=shots[0]))
    one.autotune(4)
    plain_tuned = {"tile_shape": one.tile_shape, "zchunk": one.zchunk}
    plain_ms = _time_steps(one, steps)
    one.run(nacc - one.step)
    plain_err = rel_l2(one.seismograms()[:, :, :nacc], ref)
    one.close()
    out["plain_fp32"] = {"source_steps_per_s": 1e3 / plain_ms, "ms_per_step": plain_ms,
                         "seismo_rel_l2_vs_fp64": plain_err, "seismo_steps_compared": nacc,
                         "autotuned": plain_tuned}
    for name, prec in (("batched_fp32", CGFD_PREC_FP32), ("batched_u16coef", CGFD_PREC_U16_COEF),
                       ("batched_mixed", CGFD_PREC_FP16_WAVE)):
        for nshot in (8, 32):
            q = dataclasses.replace(p, precision=prec)
            b = Simulation(q, shots=shots[:nshot])
            b.autotune(2)
            ms = _time_steps(b, steps)
            rec = {"shots": nshot, "ms_per_step": ms, "source_steps_per_s": nshot * 1e3 / ms,
                   "vs_plain": nshot * plain_ms / ms, "device_gb": b.device_bytes() / 1e9,
                   "autotuned": {"tile_shape": b.tile_shape, "zchunk": b.zchunk, "shot_group": b.shot_group}}
            if nshot == 8:
                b.run(nacc - b.step)
                rec["seismo_rel_l2_vs_fp64"] = rel_l2(b.seismograms()[0][:, :, :nacc], ref)
                rec["seismo_steps_compared"] = nacc
            b.close()
            out[f"{name}_{nshot}"] = rec
    out["note"] = ("seismo_rel_l2_vs_fp64: gather relative L2 of shot 0 after 400 steps against the FP64 build of "
                   "the same kernels (CGFD_PREC_FP64) on the same GPU.")
    return out


def media_bench(local, steps=2000, media=("vti", "aniso", "ac", "vis")):
    """The anisotropic precision workload at its full size: 320x320x160 (50 m, CFS-PML 20, free
    surface), layered Thomsen VTI and Bond-rotated tilted-TI 21-Cij media, one double-couple
    source (fc 3 Hz) at 2 km, 100 surface stations, 2000 steps; and the same grid with a layered
    acoustic medium (pressure and force source; FP32 only, its 16-bit modes are not built). The FP64 build of the kernels
    runs first; then every storage-precision mode runs the same 2000 steps (graph-replayed, timed
    with CUDA events: Gcell-stage/s) and reports its seismogram error against the FP64 build
    (relative L2 of the gather, largest per-station relative L2 with the tests' 1e-3 floor,
    relative error of the peak amplitude). FP32 and 16-bit fixed-point coefficients also report
    the bulk stage's algorithmic bytes (36 wavefield + NCOEF coefficient accesses per
    cell-stage; acoustic: 16 wavefield + 11 coefficient accesses over every plane) per event-timed
    duration against the measured HBM peak. Each mode's problem is autotuned (tile shape, z chunk)
    before it runs. Last, the same grid with a visco-elastic medium (3 GMB mechanisms, FP32):
    Gcell-stage/s and the event-timed stage (both passes) against its 593 B per cell-stage.
    `media` picks the legs."""
    import torch
    from cgfd_b200 import (synth, Simulation, CGFD_PREC_FP32, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE,
                           CGFD_PREC_FP16_COEF, CGFD_PREC_BF16_COEF, CGFD_PREC_FP64)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import rel_l2, per_station_rel_l2
    ni, nj, nk = 320, 320, 160
    peak, _ = measured_peak()
    out = {"workload": f"{ni}x{nj}x{nk}", "steps": steps, "reference": "FP64 build of the same kernels (GPU)"}
    modes = (("fp32", CGFD_PREC_FP32, 4), ("u16coef", CGFD_PREC_U16_COEF, 2), ("mixed_fp16wave", CGFD_PREC_FP16_WAVE, 2),
             ("fp16coef", CGFD_PREC_FP16_COEF, 2), ("bf16coef", CGFD_PREC_BF16_COEF, 2))
    for med, ncoef in (("vti", 15), ("aniso", 31), ("ac", 11)):  # visco-elastic after the loop
        if med not in media:
            continue
        nf, nplanes = (4, nk) if med == "ac" else (9, nk - 4)  # fields; planes of the bulk kernel
        p = synth.make_problem(ni, nj, nk, 50.0, steps, dt=None, medium=med, npml=20, nsrc=1, sta_grid=(10, 10),
                               fc=3.0, seed=31, src_depth=(2000.0, 2000.0), center_src=True)
        p.device = local
        p.precision = CGFD_PREC_FP64
        sim = Simulation(p)
        t = time.perf_counter()
        sim.run(steps)
        t64 = time.perf_counter() - t
        ref = sim.seismograms()[:, :, :steps]
        sim.close()
        pk = float(np.abs(ref).max())
        out[f"{med}_fp64"] = {"value": ni * nj * nk * 4 * steps / t64 / 1e9, "unit": UNIT, "wall_s": t64}
        for name, prec, cbytes in modes[:1] if med == "ac" else modes:
            p.precision = prec
            sim = Simulation(p)
            sim.autotune(4)  # tile shape and z chunk for this medium and storage mode
            tuned = {"tile_shape": sim.tile_shape, "zchunk": sim.zchunk}
            st = torch.cuda.ExternalStream(sim.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            sim.enqueue(steps)
            e1.record(st)
            e1.synchronize()
            sim.synchronize()
            ms = e0.elapsed_time(e1) / steps
            s = sim.seismograms()[:, :, :steps]
            rec = {"value": ni * nj * nk * 4 / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
                   "gather_rel_l2_vs_fp64": rel_l2(s, ref), "station_rel_l2_vs_fp64": per_station_rel_l2(s, ref),
                   "peak_rel_err_vs_fp64": abs(float(np.abs(s).max()) - pk) / pk, "autotuned": tuned}
            if name in ("fp32", "u16coef"):
                sim.set_timing(True)
                sim.timing(reset=True)
                sim.enqueue(8)
                sim.synchronize()
                bulk_ms, bulk_n = sim.timing(reset=True)["bulk"]
                sim.set_timing(False)
                bpc = 4 * nf * 4 + ncoef * cbytes
                achieved = bpc * ni * nj * nplanes / (bulk_ms / bulk_n * 1e-3) / 1e9
                rec.update({"bulk_ms_per_stage": bulk_ms / bulk_n, "bytes_per_cell_stage": bpc,
                            "roofline_frac": achieved / peak})
            sim.close()
            out[f"{med}_{name}"] = rec
    # visco-elastic (GMB, 3 mechanisms; FP32 only, no FP64 build): the iso layers with Q, the
    # same source and stations; the stage time covers the iso kernels in their right-hand-side
    # mode and the attenuation pass. Bytes per cell-stage of this two-pass form, averaged over
    # the 4 stages: the iso pass 30 floats (9 stage-input fields, 12 coefficients, 9 RHS) and the
    # attenuation pass 118.25 (RHS, wave levels, 2 moduli, 6 weights and 18 memory variables per
    # level touched: 98 / 143 / 143 / 89 floats at stages 0-3) = 593 B.
    if "vis" not in media:
        return out
    p = synth.make_problem(ni, nj, nk, 50.0, steps, dt=None, medium="vis", npml=20, nsrc=1, sta_grid=(10, 10),
                           fc=3.0, seed=31, src_depth=(2000.0, 2000.0), center_src=True)
    p.device = local
    sim = Simulation(p)
    sim.autotune(4)
    st = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.enqueue(steps)
    e1.record(st)
    e1.synchronize()
    sim.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sim.set_timing(True)
    sim.timing(reset=True)
    sim.enqueue(8)
    sim.synchronize()
    bulk_ms, _ = sim.timing(reset=True)["bulk"]  # both passes of the 32 stages
    sim.set_timing(False)
    s = sim.seismograms()[:, :, :steps]
    zc = sim.zchunk
    sim.close()
    bpc = 593.0
    stage_ms = bulk_ms / 32
    achieved = bpc * ni * nj * nk / (stage_ms * 1e-3) / 1e9
    out["vis_fp32"] = {"value": ni * nj * nk * 4 / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
                       "nmaxwell": 3, "stage_ms": stage_ms, "bytes_per_cell_stage": bpc,
                       "roofline_frac": achieved / peak, "finite": bool(np.isfinite(s).all()), "zchunk": zc}
    return out


def serving_bench(local, nreq=40, nmodels=8, mean_gap_s=2.5, seed=11):
    """The serving loop on a stream shaped like the serving workload: `nmodels` seeded models
    with grid sizes drawn uniformly between 64^3 and 320x320x160 (x, y in [64, 320], z in
    [64, 160]) and media 50% iso / 30% VTI / 20% 21-Cij aniso (each with its own topography and
    medium, 100 m, CFS-PML 10, free surface, 16 surface stations); `nreq` requests with Poisson
    arrivals (mean gap `mean_gap_s`), each on a random model with 1-8 random double-couple
    sources and 500-2000 steps (drawn in steps of 500, so that same-grid requests can batch).
    The full workload's 500 requests would hold the GPU for about ten minutes; the stream keeps
    its size, media and step distributions at `nreq` requests. Reports p50 / p99 latency (submit
    -> seismograms ready), completed cell-stages/s and the largest device memory held."""
    import dataclasses
    from cgfd_b200 import synth, Server
    rng = np.random.default_rng(seed)
    kinds = rng.choice(["iso", "vti", "aniso"], size=nmodels, p=[0.5, 0.3, 0.2])
    models = []
    for n in range(nmodels):
        ni, nj = (int(v) for v in rng.integers(8, 41, 2) * 8)
        nk = int(rng.integers(8, 21) * 8)
        m = synth.make_problem(ni, nj, nk, 100.0, 500, dt=None, medium=str(kinds[n]), npml=10, nsrc=0,
                               sta_grid=(4, 4), fc=2.0, seed=300 + n)
        m.device = local
        models.append(m)
    reqs = []
    for r in range(nreq):
        m = models[int(rng.integers(nmodels))]
        steps = int(rng.integers(1, 5)) * 500
        src = synth.dc_sources(m.coord, m.ni, m.nj, int(rng.integers(1, 9)), rng, depth_range=(1500.0, 4000.0),
                               fc_range=(1.5, 2.5), stf_length=(steps + 1) * m.dt)
        reqs.append(dataclasses.replace(m, src=src, nt_total=steps + 1))
    gaps = rng.exponential(mean_gap_s, nreq)
    work = sum(q.ni * q.nj * q.nk * 4.0 * q.nt_total for q in reqs)
    with Server(device=local, max_active=4, max_batch=8, steps_per_slice=100) as srv:
        t0 = time.perf_counter()
        ids = []
        for q, g in zip(reqs, gaps):
            time.sleep(float(g))
            ids.append(srv.submit(q))
        for i in ids:
            if srv.wait(i, timeout=1800) is None:
                raise RuntimeError("serving request timed out")
        wall = time.perf_counter() - t0
        st = srv.stats()
    return {"requests": nreq, "models": [f"{m.medium_type}:{m.ni}x{m.nj}x{m.nk}" for m in models],
            "steps": "500-2000 (multiples of 500)", "sources": "1-8",
            "arrivals": f"Poisson, mean gap {mean_gap_s * 1e3:.0f} ms", "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "mean_ms": st["mean_ms"], "completed": st["completed"], "failed": st["failed"], "batches": st["batches"],
            "cell_stages_per_s": st["cell_stages_per_s"], "source_steps_per_s": st["source_steps_per_s"],
            "wall_s": wall, "offered_gcell_stages": work / 1e9, "hbm_peak_gb": st["hbm_peak"] / 1e9,
            "hbm_budget_gb": st["hbm_budget"] / 1e9}


def cpu_baseline(args, threads, p=None, steps=3):
    """The oracle (FP32 CPU restatement, OpenMP on all host cores) on the full workload grid:
    one warm-up time step, then `steps` timed time steps (each a full 4-stage step of every
    cell, PML, free surface, source and stations), i.e. the same sample as each step of the
    --impl reference arm."""
    from oracle.oracle import Oracle
    if p is None:
        p = build_problem(args)
    o = Oracle(p)
    o.run(1)  # warm-up
    t = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t
    o.close()
    cells = p.ni * p.nj * p.nk * 4 * steps
    return {"value": cells / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} full time steps (4 RK stages each) of the {p.ni}x{p.nj}x{p.nk} workload grid after "
                      f"1 warm-up step, {dt:.1f} s; the same per-step sample as --impl reference"}


def reference_gpu_kernels(p, steps):
    """The reference's own GPU solver code (oracle/_ref/ref_harness: its unmodified per-stage
    kernels, RK-combine launches and per-station sampling, built for sm_100a) timed on the same
    grid and step count on this B200; None when the harness was not built."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import tempfile
    from golden import ref_io
    if not os.path.exists(ref_io.HARNESS):
        return None
    with tempfile.TemporaryDirectory() as d:
        r = ref_io.run(p, d, steps, timeout=1800)
    rate = r["cell_stages"] / (r["loop_ms"] * 1e-3) / 1e9
    return {"value": rate, "unit": UNIT, "steps": steps, "ms_per_step": r["loop_ms"] / steps,
            "grid": [p.ni, p.nj, p.nk],
            "note": "reference time loop (sv_curv_col_el_iso_onestage + wav_update + io_recv_keep per step) on the "
                    "same B200, same grid, medium, PML, source and stations; device-synchronised loop time"}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's time loop on host cores (the
    reference has no CPU solver of its own), on the full workload grid: W warm-up time steps,
    then K timed full time steps. If K + W full steps would take more than about four minutes
    on this host, each step is a bounded z-slab sample of the workload instead (reported)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    from oracle.oracle import Oracle
    p = build_problem(args)
    o = Oracle(p)
    t = time.perf_counter()
    o.run(1)  # probe step (also the first warm-up step)
    t_step = time.perf_counter() - t
    same = (args.steps + args.warmup) * t_step <= 240.0
    if not same:
        o.close()
        nk_s = max(8, min(p.nk, int(p.nk * 240.0 / ((args.steps + args.warmup) * t_step))))
        p = build_problem(args, nk_override=nk_s)
        o = Oracle(p)
        o.run(1)
    for _ in range(max(0, args.warmup - 1)):
        o.run(1)
    t = time.perf_counter()
    for _ in range(args.steps):
        o.run(1)
    el = time.perf_counter() - t
    o.close()
    cells = p.ni * p.nj * p.nk * 4 * args.steps
    v = cells / el / 1e9
    sample = (f"each step = one full time step (4 RK stages) of the {p.ni}x{p.nj}x{p.nk} workload grid by the oracle"
              if same else f"each step = one time step of a {p.ni}x{p.nj}x{p.nk} z-slab of the workload (full grid "
                           f"would exceed the time bound: {t_step:.1f} s per step)")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"{WORKLOADS[args.workload][0]}x{WORKLOADS[args.workload][1]}x"
                                  f"{WORKLOADS[args.workload][2]}", "sample_grid": [p.ni, p.nj, p.nk],
                      "medium": "elastic_iso", "same_grid_as_b200_arm": same},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.medium != "iso" and args.profile_steps <= 0:
        raise SystemExit("--medium applies to the profiling case (--profile-steps); the bench line is the iso workload")
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_steps > 0:
        return profile_run(args)
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from cgfd_b200 import Simulation

    p = build_problem(args, device=local)
    cells = p.ni * p.nj * p.nk
    nbulk = p.nk - 4
    sim = Simulation(p)
    tuned = None
    if args.tile_shape >= 0:
        sim.set_tile_shape(args.tile_shape)
    if args.zchunk:
        sim.set_zchunk(args.zchunk)
    elif not args.no_autotune:
        # cgfd_autotune: both tile shapes x the z-chunk candidates timed on this problem (8 steps
        # each), before the warm-up; the state is reset to step 0 afterwards
        t = time.perf_counter()
        sim.autotune(8)
        tuned = {"tile_shape": sim.tile_shape, "zchunk": sim.zchunk, "tuning_s": time.perf_counter() - t}
    shape_used, zchunk_used = sim.tile_shape, sim.zchunk
    st = torch.cuda.ExternalStream(sim.stream)
    # warm-up: W steps, at least 8 so that the CUDA graph of every step of the 8-step
    # operator-pair cycle is captured before the timed region
    sim.enqueue(max(args.warmup, 8))
    sim.synchronize()
    sim.timing(reset=True)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    # timed region: K graph-replayed steps (the production path; no per-kernel events)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.enqueue(args.steps)
    e1.record(st)
    e1.synchronize()
    sim.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = sim.timing(reset=True)["launches"]
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    value = job_value(world, cells, args.steps, ms)

    # kernel breakdown: further steps launched directly with CUDA events around every kernel
    # on the launching stream (the surface slab then runs after the bulk tiles instead of
    # beside them); the roofline uses the bulk stage's mean duration from here
    ksteps = max(8, min(args.steps, 24))
    sim.set_timing(True)
    sim.timing(reset=True)
    e0.record(st)
    sim.enqueue(ksteps)
    e1.record(st)
    e1.synchronize()
    sim.synchronize()
    ms_k = e0.elapsed_time(e1)
    tim = sim.timing(reset=True)
    sim.set_timing(False)

    # roofline of the dominant kernel (bulk stage): algorithmic bytes per launch / duration
    bulk_ms, bulk_n = tim["bulk"]
    bpc = BYTES_PER_CELL_STAGE["iso"]
    bulk_cells = p.ni * p.nj * nbulk
    alg = bpc * bulk_cells
    achieved = alg / (bulk_ms / bulk_n * 1e-3) / 1e9 if bulk_n else None
    peak, peak_kind = measured_peak()
    traffic, traffic_capture = ncu_traffic(args.workload, bulk_cells, shape_used, zchunk_used)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "traffic": traffic, "traffic_capture": traffic_capture,
            "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback",
            "kernel": "k_stage_bulk_tma<iso> (interior-tile and PML-tile launches of one RK stage)",
            "bytes_per_cell_stage": bpc, "cells_per_launch": bulk_cells,
            "kernel_ms": {k: (v[0] / v[1] if v[1] else None) for k, v in tim.items() if k != "launches"},
            "kernel_share": {k: (v[0] / ms_k if ms_k else None) for k, v in tim.items()
                             if k in ("bulk", "surface", "source", "recv")},
            "breakdown_steps": ksteps}
    sim.close()
    del sim

    e2e = None
    if not args.no_e2e:
        # public API end to end: host arrays -> create (H2D + setup) -> K steps -> seismograms D2H
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t = time.perf_counter()
        s2 = Simulation(p)
        s2.enqueue(args.steps)
        seis = s2.seismograms()
        s2.synchronize()
        t_e2e = time.perf_counter() - t
        s2.close()
        t_e2e = max_over_ranks(t_e2e, dist, f"cuda:{local}")
        fld = (p.ni + 6) * (p.nj + 6) * (p.nk + 6) * 4
        h2d = 13 * fld
        e2e = {"value": world * cells * 4 * args.steps / t_e2e / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": seis.nbytes / args.steps,
               "note": "cgfd_problem_create from host arrays (metric 10 + medium 3 fields) + K steps + "
                       "seismogram read-back, wall clock"}

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            batched = batched_mixed(local)
        except Exception as ex:  # report, do not fail the headline measurement
            batched = {"error": str(ex)}

    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        try:
            serving = serving_bench(local)
        except Exception as ex:  # report, do not fail the headline measurement
            serving = {"error": str(ex)}

    # after serving: the large anisotropic models would otherwise sit in host memory while the
    # serving loop's requests are built and uploaded
    media = None
    if rank == 0 and world == 1 and not args.no_media:
        try:
            media = media_bench(local)
        except Exception as ex:  # report, do not fail the headline measurement
            media = {"error": str(ex)}

    cpu = None
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        try:
            cpu = cpu_baseline(args, threads, p)
        except Exception as ex:  # report, do not fail the GPU measurement
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "port", "sample": f"failed: {ex}"}
        try:
            ref_gpu = reference_gpu_kernels(p, args.steps)
        except Exception as ex:  # report, do not fail the GPU measurement
            ref_gpu = {"error": str(ex)}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": f"{p.ni}x{p.nj}x{p.nk}", "medium": "elastic_iso", "dh_m": 50.0,
                          "pml_layers": 20, "free_surface": "timg", "sources": 1, "stations": 400,
                          "dt": p.dt, "precision": "fp32", "parallelism": f"replicas x{world}",
                          "l2": f"inputs larger than L2 (wavefield 4 levels x 9 x {(p.ni + 6) * (p.nj + 6) * (p.nk + 6) / 1e6:.1f}M floats)",
                          "autotuned": tuned},
               "roofline": roof, "cpu_baseline": cpu, "reference_gpu_kernels": ref_gpu, "e2e": e2e,
               "gpu_launches": launches,
               "clocks": clocks, "batched_mixed": batched, "media": media, "serving": serving}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
