"""Long-run precision study: seismogram errors of every storage-precision mode against the FP64
oracle (the CPU restatement instantiated in double, same inputs) on VTI and 21-Cij aniso media.

The GPU test suite checks the modes over 240 steps on 56x52x40 grids; this study runs them long
enough for phase errors to accumulate (default 2000 steps, the step count of the anisotropic
precision workload) on the largest grid whose FP64 oracle run stays practical on a CPU
(128x128x64, 50 m, CFS-PML 10, free surface, one double-couple source at 1.5 km, 16 surface
stations; the full 320x320x160 workload would take the oracle days).

Two stages, because the oracle runs on the host and the modes on a GPU:

    python tests/precision_study.py oracle --cache DIR     # CPU: FP64 oracle seismograms
    python tests/precision_study.py gpu --cache DIR        # GPU: every mode, error table
    python tests/precision_study.py fp16sol --steps 1500   # GPU: FP16 solution-level bound

`oracle --cache tests/golden` made the committed fixtures tests/golden/fp64_long_{vti,aniso}.npz
that tests/test_gpu_precision_long.py checks the FP32, fixed-point and mixed modes against.

Errors per mode (against FP64): relative L2 of the whole gather, largest per-station relative
L2 (denominator floored at 1e-3 of the strongest station, as in the tests) and relative error
of the peak amplitude.
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "gpu-cgfd3d-elastic_b200"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

MEDIA = ("vti", "aniso")


def problem(medium, ni, nj, nk, nsteps):
    from cgfd_b200 import synth
    return synth.make_problem(ni, nj, nk, 50.0, nsteps, dt=None, medium=medium, npml=10, nsrc=1, sta_grid=(4, 4),
                              fc=4.0, seed=41, src_depth=(1500.0, 1500.0), center_src=True)


def stage_oracle(args):
    from oracle.oracle import Oracle
    os.makedirs(args.cache, exist_ok=True)
    for med in MEDIA:
        p = problem(med, args.ni, args.nj, args.nk, args.steps)
        t = time.perf_counter()
        o = Oracle(p, fp64=True)
        o.run()
        s = o.seismograms()
        np.savez_compressed(os.path.join(args.cache, f"fp64_long_{med}.npz"), seis=s, dt=p.dt, steps=args.steps,
                            shape=np.array([args.ni, args.nj, args.nk]))
        print(f"{med}: FP64 oracle {time.perf_counter() - t:.0f} s, {s.shape[0]} stations", flush=True)


def stage_gpu(args):
    from cgfd_b200 import (Simulation, CGFD_PREC_FP32, CGFD_PREC_BF16_COEF, CGFD_PREC_FP16_COEF,
                           CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE)
    from helpers import rel_l2, per_station_rel_l2
    modes = {"fp32": CGFD_PREC_FP32, "bf16_coef": CGFD_PREC_BF16_COEF, "fp16_coef": CGFD_PREC_FP16_COEF,
             "u16_coef": CGFD_PREC_U16_COEF, "fp16_wave": CGFD_PREC_FP16_WAVE}
    out = {"grid": f"{args.ni}x{args.nj}x{args.nk}", "steps": args.steps}
    for med in MEDIA:
        z = np.load(os.path.join(args.cache, f"fp64_long_{med}.npz"))
        if int(z["steps"]) != args.steps or list(z["shape"]) != [args.ni, args.nj, args.nk]:
            raise SystemExit(f"cache for {med} was made for another configuration")
        ref = z["seis"]
        peak = float(np.abs(ref).max())
        p = problem(med, args.ni, args.nj, args.nk, args.steps)
        for name, prec in modes.items():
            p.precision = prec
            sim = Simulation(p)
            sim.run()
            s = sim.seismograms()
            sim.close()
            out[f"{med}_{name}"] = {"gather_rel_l2": rel_l2(s, ref), "station_rel_l2": per_station_rel_l2(s, ref),
                                    "peak_rel_err": abs(float(np.abs(s).max()) - peak) / peak}
            e = out[f"{med}_{name}"]
            print(f"{med:6s} {name:10s} gather {e['gather_rel_l2']:.2e}  station {e['station_rel_l2']:.2e}  "
                  f"peak {e['peak_rel_err']:.2e}", flush=True)
    print(json.dumps(out))


def round_fp16_scaled(w):
    """FP16 storage of a wavefield with one power-of-two scale per group (velocity, stress),
    max |w| mapped into [2^12, 2^13) as the FP16 stage levels do: the value read back."""
    out = np.empty_like(w)
    for sl in (slice(0, 3), slice(3, 9)):
        m = float(np.abs(w[sl]).max())
        if m == 0.0:
            out[sl] = w[sl]
            continue
        e = int(np.floor(np.log2(m))) - 12
        sc = 2.0 ** e
        out[sl] = (w[sl].astype(np.float64) / sc).astype(np.float16).astype(np.float64) * sc
    return out.astype(np.float32)


def stage_fp16sol(args):
    """Lower bound of the error of FP16 solution levels: the FP64 build of the kernels, its
    solution level w_pre rounded to scaled FP16 after every time step (through
    cgfd_get_wavefield / cgfd_set_wavefield), against the same FP64 run without rounding. A
    real FP16-solution mode rounds at least this often (every RK stage's accumulator too), so
    an error above the bar here rules it out."""
    from cgfd_b200 import Simulation, CGFD_PREC_FP64
    from helpers import rel_l2, per_station_rel_l2
    out = {"grid": f"{args.ni}x{args.nj}x{args.nk}", "steps": args.steps}
    for med in MEDIA:
        p = problem(med, args.ni, args.nj, args.nk, args.steps)
        p.precision = CGFD_PREC_FP64
        ref = Simulation(p)
        ref.run(args.steps)
        r = ref.seismograms()[:, :, :args.steps]
        ref.close()
        sim = Simulation(p)
        for it in range(args.steps):
            sim.run(1)
            sim.set_wavefield(round_fp16_scaled(sim.wavefield()))
        s = sim.seismograms()[:, :, :args.steps]
        sim.close()
        e = {"gather_rel_l2": rel_l2(s, r), "station_rel_l2": per_station_rel_l2(s, r)}
        out[med] = e
        print(f"{med:6s} FP16 solution level (per-step rounding) gather {e['gather_rel_l2']:.2e}  "
              f"station {e['station_rel_l2']:.2e}", flush=True)
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["oracle", "gpu", "fp16sol"])
    ap.add_argument("--cache", default=None, help="directory of the FP64 oracle seismograms (oracle, gpu)")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--grid", type=int, nargs=3, default=(128, 128, 64))
    args = ap.parse_args()
    args.ni, args.nj, args.nk = args.grid
    {"oracle": stage_oracle, "gpu": stage_gpu, "fp16sol": stage_fp16sol}[args.stage](args)


if __name__ == "__main__":
    main()
