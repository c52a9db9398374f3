"""Field-energy histories of the two-stream precision study, FP64 and FP32 oracle.

The two-stream precision workload (symmetric two-stream electron beams, +-0.2c along x,
thermal spread 0.01c, 32 particles per cell per beam, immobile neutralizing ions
left out: a uniform background only touches k = 0, which the solver ignores) on
a crop small enough for the CPU oracle: 128 x 128 cells, 2000 steps, c = 3.0,
dt = 0.1, 4 filter passes, dens = 64 (both beams: omega_pe = 1).  (At c = 4.5,
dt = 0.1 the reference algorithm itself is numerically unstable for this plasma.)  The oracle is
the CPU restatement of the reference (oracle/); FP64 is the reference's dprec
build, FP32 its default build.  The seeded initial arrays come from
spectral_rs_b200.init, so the GPU test starts from the same particles.

Writes tests/golden/two_stream_energy.json.  Run: python tests/golden/make_two_stream.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

STUDY = dict(size_x=128, size_y=128, delta=0, dt=0.1, c=3.0, dens=64, gamma_inj=1.0206207261596576, n_pass=4,
             periodic_x=True, ppc=32, vth=0.01, steps=2000, every=10, seed=33)
OUT = "two_stream_energy.json"


def beams(study):
    from spectral_rs_b200.config import Params
    from spectral_rs_b200.init import positions, draws, velocities
    p = Params(size_x=study["size_x"], size_y=study["size_y"], delta=0, dt=study["dt"], c=study["c"],
               dens=study["dens"], gamma_inj=study["gamma_inj"], n_pass=study["n_pass"], periodic_x=True)
    out = []
    for k, sign in enumerate((1.0, -1.0)):
        rng = np.random.default_rng([study["seed"], k])
        ix, iy, dx, dy = positions(p.size_x, p.size_y, 0, study["ppc"], 0, p.size_x, True, rng)
        nrm, uni = draws(len(ix), rng)
        px, py, pz, psa = velocities(nrm, uni, p.c, study["vth"], study["gamma_inj"], sign)
        out.append(dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa))
    return p, out


def field_energy(get):
    e = sum(float(np.sum(get(n)[1:-1, 1:-1].astype(np.float64) ** 2)) for n in ("Ex", "Ey", "Ez")) / 2
    b = sum(float(np.sum(get(n)[1:-1, 1:-1].astype(np.float64) ** 2)) for n in ("Bx", "By", "Bz")) / 2
    return e, b


def run_oracle(dtype):
    from oracle import oracle as orc
    p, bs = beams(STUDY)
    o = orc.OracleSim.from_params(p, dtype=dtype)
    for a in bs:
        o.add_species(-1.0, 1.0, STUDY["vth"], a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                      a["psa"])
    o.prepare()
    hist = []
    for t in range(0, STUDY["steps"], STUDY["every"]):
        o.step(STUDY["every"])
        hist.append(field_energy(o.spatial))
    return hist


def main():
    # optional: a larger crop, e.g. `python tests/golden/make_two_stream.py 512`
    # writes two_stream_energy_512.json (the same plasma on 512 x 512 cells)
    global OUT
    if len(sys.argv) > 1:
        n = int(sys.argv[1])
        STUDY.update(size_x=n, size_y=n)
        OUT = f"two_stream_energy_{n}.json"
    t0 = time.time()
    out = {"study": STUDY}
    for name, dt in (("fp64", np.float64), ("fp32", np.float32)):
        h = run_oracle(dt)
        out[name] = {"E": [x[0] for x in h], "B": [x[1] for x in h]}
        print(name, "done", round(time.time() - t0, 1), "s", flush=True)
    with open(os.path.join(HERE, OUT), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
