"""Times the reference's own GPU solver code (oracle/_ref/ref_harness, built unmodified from
the reference sources for sm_100a) on the benchmark workload, on the same B200:

    python oracle/ref_timing.py [--steps N] [--grid ni nj nk]

Prints one JSON line with Gcell-stage/s of the reference's time loop (its per-stage kernels,
RK combine launches and per-station sampling), for comparison with bench.py's number.
Test/measurement infrastructure: it runs the reference, not the product.
"""
import argparse
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, os.path.join(ROOT, "gpu-cgfd3d-elastic_b200"), os.path.join(ROOT, "tests")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--grid", type=int, nargs=3, default=None)
    a = ap.parse_args()
    import bench
    from golden import ref_io
    ns = argparse.Namespace(workload="480x480x240", grid=a.grid)
    p = bench.build_problem(ns)
    with tempfile.TemporaryDirectory() as d:
        r = ref_io.run(p, d, a.steps, timeout=3000)
    rate = r["cell_stages"] / (r["loop_ms"] * 1e-3) / 1e9
    print(json.dumps({"impl": "reference_gpu_kernels", "grid": [p.ni, p.nj, p.nk], "steps": a.steps,
                      "loop_ms": r["loop_ms"], "ms_per_step": r["loop_ms"] / a.steps,
                      "value": rate, "unit": "Gcell-stage/s", "stations": int(r["seismo"].shape[0])}))


if __name__ == "__main__":
    main()
