"""Storage-precision modes against the FP64 oracle (the CPU restatement instantiated in
double, same inputs).

Every mode computes in FP32; they differ in what HBM holds:
  CGFD_PREC_FP32       everything FP32
  CGFD_PREC_BF16_COEF  metrics, 1/rho and moduli as BF16 (power-of-two scale per field)
  CGFD_PREC_FP16_COEF  the same in FP16
  CGFD_PREC_U16_COEF   the same as 16-bit fixed point over each field's [min, max]
  CGFD_PREC_FP16_WAVE  U16 coefficients + FP16 RK stage levels (per-step scale), FP32 solution
All 16-bit coefficients are stochastically rounded.

Each run reports its seismogram error against FP64: relative L2 of the whole gather, the
largest per-station relative L2 and the relative error of the peak amplitude.
Bars (written here, checked below):
  FP32                  per-station rel L2 <= 1e-4
  U16_COEF, FP16_WAVE   gather rel L2, per-station rel L2 and peak amplitude <= 1e-3
  FP16_COEF             gather rel L2 <= 3e-3 (11 significant bits; reported)
  BF16_COEF             gather rel L2 <= 2e-2 (8 significant bits; reported)
"""
import numpy as np
import pytest

from cgfd_b200 import (Simulation, synth, CGFD_PREC_FP32, CGFD_PREC_BF16_COEF, CGFD_PREC_FP16_COEF,
                       CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE)
from oracle.oracle import Oracle
from helpers import small_problem, random_wavefield, rel_l2, per_station_rel_l2

pytestmark = pytest.mark.gpu

MODES = {"fp32": CGFD_PREC_FP32, "bf16_coef": CGFD_PREC_BF16_COEF, "fp16_coef": CGFD_PREC_FP16_COEF,
         "u16_coef": CGFD_PREC_U16_COEF, "fp16_wave": CGFD_PREC_FP16_WAVE}
BARS = {"fp32": 1e-4, "bf16_coef": 2e-2, "fp16_coef": 3e-3, "u16_coef": 1e-3, "fp16_wave": 1e-3}

_fp64_cache = {}


def _problem(medium):
    return small_problem(medium, ni=56, nj=52, nk=40, nsteps=240, npml=8, sta_grid=(4, 4), seed=7)


def _fp64(medium):
    if medium not in _fp64_cache:
        o = Oracle(_problem(medium), fp64=True)
        o.run()
        _fp64_cache[medium] = o.seismograms()
    return _fp64_cache[medium]


def seismo_errors(s, ref):
    peak = float(np.abs(ref).max())
    return {"gather_rel_l2": rel_l2(s, ref), "station_rel_l2": per_station_rel_l2(s, ref),
            "peak_rel_err": abs(float(np.abs(s).max()) - peak) / peak}


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
@pytest.mark.parametrize("mode", list(MODES))
def test_precision_vs_fp64(medium, mode):
    p = _problem(medium)
    p.precision = MODES[mode]
    sim = Simulation(p)
    sim.run()
    s = sim.seismograms()
    ref = _fp64(medium)
    assert np.isfinite(s).all()
    e = seismo_errors(s, ref)
    print(f"\n{medium} {mode}: gather rel L2 {e['gather_rel_l2']:.2e}  station rel L2 "
          f"{e['station_rel_l2']:.2e}  peak {e['peak_rel_err']:.2e}  device bytes {sim.device_bytes()}")
    bar = BARS[mode]
    if mode == "fp32":
        assert e["station_rel_l2"] <= bar
    elif mode in ("bf16_coef", "fp16_coef"):
        assert e["gather_rel_l2"] <= bar
    else:
        assert e["gather_rel_l2"] <= bar and e["station_rel_l2"] <= bar and e["peak_rel_err"] <= bar


def test_precision_storage_sizes():
    """16-bit coefficients halve the coefficient array; FP16 stage levels halve two of the four
    wavefield levels."""
    p = _problem("iso")
    sizes = {}
    for mode, v in MODES.items():
        p.precision = v
        sizes[mode] = Simulation(p).device_bytes()
    assert sizes["bf16_coef"] == sizes["fp16_coef"] == sizes["u16_coef"] < sizes["fp32"]
    assert sizes["fp16_wave"] < sizes["u16_coef"]


def test_fp16_wave_batched_vs_fp64():
    """The batched mixed-precision form: 3 shots in one FP16_WAVE batch, each bitwise equal to
    its solo FP16_WAVE run and within the bar of its own FP64 oracle run."""
    p = small_problem("iso", ni=48, nj=44, nk=36, nsteps=200, npml=6, nsrc=0, sta_grid=(3, 3), seed=3)
    rng = np.random.default_rng(21)
    shots = [synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(700.0, 1500.0), fc_range=(2.5, 4.0),
                              stf_length=p.nt_total * p.dt) for _ in range(3)]
    p.precision = CGFD_PREC_FP16_WAVE
    b = Simulation(p, shots=shots)
    b.run()
    bs = b.seismograms()
    for n, s in enumerate(shots):
        p.src = s
        p.precision = CGFD_PREC_FP16_WAVE
        solo = Simulation(p)  # per-shot FP16 scales: a shot rounds as it does alone
        solo.run()
        assert np.array_equal(solo.seismograms(), bs[n])
        p.precision = CGFD_PREC_FP32
        o = Oracle(p, fp64=True)
        o.run()
        e = seismo_errors(bs[n], o.seismograms())
        assert e["gather_rel_l2"] <= 1e-3 and e["station_rel_l2"] <= 1e-3, (n, e)


@pytest.mark.parametrize("it0", [0, 3])
def test_fp16_wave_follows_host_wavefield(it0):
    """The FP16 stage scale follows a wavefield the host loads (set_step + set_wavefield):
    stresses of 1e5-1e6 Pa would overflow unscaled FP16. 12 steps against FP32 from the
    same state."""
    p = small_problem("vti", nsteps=20, nsrc=0, sta_grid=None)
    w0 = random_wavefield(p, seed=5) * np.float32(10.0)
    out = {}
    for mode in ("fp16_wave", "fp32"):
        p.precision = MODES[mode]
        sim = Simulation(p)
        sim.set_step(it0)
        sim.set_wavefield(w0)
        sim.run(12)
        out[mode] = sim.wavefield()
    assert np.isfinite(out["fp16_wave"]).all()
    assert rel_l2(out["fp16_wave"], out["fp32"]) <= 1e-3
