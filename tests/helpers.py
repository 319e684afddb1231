"""Shared builders for the parity tests (small seeded problems)."""
import numpy as np

from cgfd_b200 import synth
from oracle.oracle import metric_fp32


def small_problem(medium="iso", ni=40, nj=36, nk=30, nsteps=40, npml=6, free_top=1, nsrc=1, seed=0, dt=None,
                  sta_grid=(3, 3), dh=100.0):
    return synth.make_problem(ni, nj, nk, dh, nsteps, dt=dt, medium=medium, npml=npml, nsrc=nsrc,
                              sta_grid=sta_grid, seed=seed, metric_fn=metric_fp32, free_top=free_top,
                              src_depth=(800.0, 1200.0), center_src=(nsrc == 1))


def random_wavefield(p, seed=0, smooth=True):
    """A seeded wavefield with zero ghosts; smooth variant = sum of a few plane waves."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = p.nk + 6, p.nj + 6, p.ni + 6
    w = np.zeros((9, nz, ny, nx), np.float32)
    if smooth:
        k, j, i = np.meshgrid(np.arange(p.nk), np.arange(p.nj), np.arange(p.ni), indexing="ij")
        for c in range(9):
            acc = np.zeros(k.shape)
            for _ in range(4):
                kv = rng.uniform(-0.6, 0.6, 3)
                acc += rng.standard_normal() * np.cos(kv[0] * i + kv[1] * j + kv[2] * k + rng.uniform(0, 6.3))
            w[c, 3:-3, 3:-3, 3:-3] = acc * (1e-2 if c < 3 else 1e5)
    else:
        w[:3, 3:-3, 3:-3, 3:-3] = rng.standard_normal((3, p.nk, p.nj, p.ni)) * 1e-2
        w[3:, 3:-3, 3:-3, 3:-3] = rng.standard_normal((6, p.nk, p.nj, p.ni)) * 1e5
    return w


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def per_station_rel_l2(s, ref, floor=1e-3):
    """max over stations of the relative L2 of the 9-component seismogram. The denominator
    is floored at `floor` x the largest station norm so that a station the wave has not
    reached yet (signal at rounding level) does not turn rounding noise into a large ratio."""
    s = np.asarray(s, np.float64)
    ref = np.asarray(ref, np.float64)
    norms = [np.linalg.norm(ref[n]) for n in range(ref.shape[0])]
    if not norms:
        return 0.0
    top = max(norms)
    return max(float(np.linalg.norm(s[n] - ref[n]) / max(norms[n], floor * top, 1e-300)) for n in range(ref.shape[0]))
