"""Generates tests/golden/ref_<case>.npz by running the reference's own solver code
(oracle/_ref/ref_harness, built by `make -f oracle/Makefile.ref`) on a B200.

    python tests/golden/make_ref_golden.py <out_dir> [case ...]   (default: every case)

The fixtures hold the reference-computed metrics, seismograms, final wavefield and free-surface
peak ground motion (PG_calcu_gpu) of small seeded problems (tests/golden/cases.py); tests/test_cpu_golden.py checks the oracle against
them without a GPU.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "gpu-cgfd3d-elastic_b200"), os.path.join(ROOT, "tests")]

from golden.cases import GOLDEN_CASES, golden_problem  # noqa: E402
from golden import ref_io  # noqa: E402


def main(out_dir, names=None):
    os.makedirs(out_dir, exist_ok=True)
    for name in names or list(GOLDEN_CASES):
        p, nsteps = golden_problem(name)
        with tempfile.TemporaryDirectory() as d:
            r = ref_io.run(p, d, nsteps)
        sl = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))
        extra = {"pg": r["pg"]} if r["pg"] is not None else {}
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), metric=r["metric"], seismo=r["seismo"],
                            wave=r["wave"][sl], nsteps=nsteps, **extra)
        print(name, "stations", r["seismo"].shape[0], "max|seis|", float(np.abs(r["seismo"]).max()))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE, sys.argv[2:])
