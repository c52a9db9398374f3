"""Precision study (symmetric two-stream electron beams): GPU FP32 against the FP64 oracle.

tests/golden/two_stream_energy.json holds the field-energy history of the
FP64 and FP32 oracle runs (tests/golden/make_two_stream.py).  The GPU split path
(with plain and with compensated current sums) and the plain path start from the
same seeded particles and run the same 2000 steps.
Reported (printed with -s): the linear growth rate of the field energy and the
relative field-energy error against FP64 over time.  The instability amplifies
rounding differences exponentially, so after saturation the runs decorrelate;
the assertions bound the linear phase tightly and the late phase statistically.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
FIXTURE = os.path.join(ROOT, "tests", "golden", "two_stream_energy.json")
# the same plasma on a 512 x 512 crop (make_two_stream.py 512), when generated
FIXTURE_512 = os.path.join(ROOT, "tests", "golden", "two_stream_energy_512.json")


def _run_gpu(path, fixture=FIXTURE):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_two_stream as mts
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    with open(fixture) as f:
        study = json.load(f)["study"]
    mts.STUDY.update(study)
    p, bs = mts.beams(study)
    p.compensated = path == "split_compensated"
    with Sim(Config(p, Setup(study["steps"]), Output(False, False, 1, 1, 1, 1)),
             path="plain" if path == "plain" else "split") as sim:
        for a in bs:
            sim.add_species(-1.0, 1.0, study["vth"], a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                            a["psa"])
        sim.prepare()
        hist = []
        for _ in range(0, study["steps"], study["every"]):
            sim.step(study["every"])
            d = sim.diag()
            hist.append(d[0])
    return np.array(hist), study


def _growth_rate(e, every, dt):
    """Fit d ln(E_field)/dt over the window where the FP64 energy grows exponentially."""
    t = (np.arange(len(e)) + 1) * every * dt
    le = np.log(e)
    return t, le


def _fixtures():
    return [FIXTURE] + ([FIXTURE_512] if os.path.exists(FIXTURE_512) else [])


@pytest.mark.parametrize("fixture", _fixtures(), ids=lambda f: os.path.basename(f))
@pytest.mark.parametrize("path", ["split", "split_compensated", "plain"])
def test_two_stream_energy_vs_fp64(fixture, path):
    with open(fixture) as f:
        ref = json.load(f)
    e_gpu, study = _run_gpu(path, fixture)
    e64 = np.array(ref["fp64"]["E"])
    e32 = np.array(ref["fp32"]["E"])
    assert len(e_gpu) == len(e64)
    every, dt = study["every"], study["dt"]
    t = (np.arange(len(e64)) + 1) * every * dt
    # exponential phase of the FP64 history: from its minimum before the peak to
    # half the peak, first quarter skipped (noise floor)
    peak = int(np.argmax(e64))
    start = int(np.argmin(e64[:peak + 1]))
    end = start + int(np.flatnonzero(e64[start:] > 0.5 * e64[peak])[0])
    win = np.arange(start + (end - start) // 4, end + 1)
    assert len(win) >= 5, "no exponential phase in the FP64 history"
    g64 = np.polyfit(t[win], np.log(e64[win]), 1)[0] / 2   # field amplitude growth rate
    ggp = np.polyfit(t[win], np.log(e_gpu[win]), 1)[0] / 2
    g32 = np.polyfit(t[win], np.log(e32[win]), 1)[0] / 2
    rel = np.abs(e_gpu - e64) / e64
    rel32 = np.abs(e32 - e64) / e64
    lin_end = win[-1]
    path = f"{path} {study['size_x']}x{study['size_y']}"
    print(f"\n[{path}] growth rate (1/omega_pe): fp64 {g64:.5f}  gpu fp32 {ggp:.5f}  oracle fp32 {g32:.5f}")
    print(f"[{path}] rel. field-energy error vs fp64: end of linear phase (step {(lin_end + 1) * every}) "
          f"{rel[lin_end]:.2e} (oracle fp32 {rel32[lin_end]:.2e}); step {len(e64) * every}: {rel[-1]:.2e} "
          f"(oracle fp32 {rel32[-1]:.2e}); median over run {np.median(rel):.2e} (oracle fp32 {np.median(rel32):.2e})")
    assert abs(ggp - g64) < 0.01 * abs(g64)
    assert rel[lin_end] < 1e-3
    # saturated, decorrelated phase: statistical agreement of the energy level
    late = slice(len(e64) * 3 // 4, None)
    assert abs(np.mean(e_gpu[late]) - np.mean(e64[late])) < 0.2 * np.mean(e64[late])
