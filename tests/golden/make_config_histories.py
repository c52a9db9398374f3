"""Field-energy histories of two benchmark configurations, FP64 and FP32 oracle.

  shock   the plain-method unmagnetized shock at its own size: 512 x 64 cells,
          delta = 8, reflecting wall on the right (the reference's geometry,
          src/prtls.rs:153) and its mirror image on the left, ions (mass ratio
          16) and electrons, 16 particles per cell per species, thermal spread
          0.1c, drift 0.1c toward the right wall (gamma 1.0050378), 4 filter
          passes, 1000 steps.
  weibel  the Weibel filamentation configuration on a 1024 x 256 sub-run:
          counter-streaming electron-positron beams along x at +-0.5c (gamma
          1.1547005), thermal spread 0.05c, 16 particles per cell per beam per
          species (4 species), 8 filter passes, 250 steps (linear growth of the
          magnetic energy from step ~50, saturation by step ~200).

Both use c = 3.0, dt = 0.1 (Courant number 0.3) and random positions in the
cell.  The oracle is the CPU restatement of the reference (oracle/); FP64 is
the reference's dprec build, FP32 its default build.  The seeded initial arrays
come from spectral_rs_b200.init (`species_of`), so the GPU tests start from the
same particles.

Writes tests/golden/config_histories.json.  Run: python tests/golden/make_config_histories.py
"""
import json
import os
import sys
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

GAMMA_SHOCK = 1.0050378  # drift 0.1c
GAMMA_WEIBEL = 1.1547005  # +-0.5c

CONFIGS = {
    "shock": dict(size_x=512, size_y=64, delta=8, dt=0.1, c=3.0, dens=16, gamma_inj=GAMMA_SHOCK, n_pass=4,
                  periodic_x=False, left_wall=True, steps=1000, every=10, seed=1001,
                  # (charge, mass, vth, ppc, drift gamma, drift sign)
                  species=[(1.0, 16.0, 0.1, 16, GAMMA_SHOCK, 1.0), (-1.0, 1.0, 0.1, 16, GAMMA_SHOCK, 1.0)]),
    "weibel": dict(size_x=1024, size_y=256, delta=0, dt=0.1, c=3.0, dens=32, gamma_inj=GAMMA_WEIBEL, n_pass=8,
                   periodic_x=True, left_wall=False, steps=250, every=5, seed=1002,
                   species=[(-1.0, 1.0, 0.05, 16, GAMMA_WEIBEL, 1.0), (-1.0, 1.0, 0.05, 16, GAMMA_WEIBEL, -1.0),
                            (1.0, 1.0, 0.05, 16, GAMMA_WEIBEL, 1.0), (1.0, 1.0, 0.05, 16, GAMMA_WEIBEL, -1.0)]),
}


def params_of(cfg):
    from spectral_rs_b200.config import Params
    return Params(size_x=cfg["size_x"], size_y=cfg["size_y"], delta=cfg["delta"], dt=cfg["dt"], c=cfg["c"],
                  dens=cfg["dens"], gamma_inj=cfg["gamma_inj"], n_pass=cfg["n_pass"], periodic_x=cfg["periodic_x"],
                  left_wall=cfg["left_wall"])


def species_of(cfg):
    """[(charge, mass, vth, arrays)] of the configuration, in the reference's order."""
    from spectral_rs_b200.init import positions, draws, velocities
    out = []
    for k, (q, m, vth, ppc, gamma, sign) in enumerate(cfg["species"]):
        rng = np.random.default_rng([cfg["seed"], k])
        ix, iy, dx, dy = positions(cfg["size_x"], cfg["size_y"], cfg["delta"], ppc, None, None, True, rng)
        nrm, uni = draws(len(ix), rng)
        px, py, pz, psa = velocities(nrm, uni, cfg["c"], vth, gamma, sign)
        out.append((q, m, vth, dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)))
    return out


def field_energy(get):
    e = sum(float(np.sum(get(n)[1:-1, 1:-1].astype(np.float64) ** 2)) for n in ("Ex", "Ey", "Ez")) / 2
    b = sum(float(np.sum(get(n)[1:-1, 1:-1].astype(np.float64) ** 2)) for n in ("Bx", "By", "Bz")) / 2
    return e, b


def run_oracle(name, dtype_name):
    from oracle import oracle as orc
    cfg = CONFIGS[name]
    o = orc.OracleSim.from_params(params_of(cfg), dtype=np.float64 if dtype_name == "fp64" else np.float32)
    for q, m, vth, a in species_of(cfg):
        o.add_species(q, m, vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
    o.prepare()
    hist = []
    for _ in range(0, cfg["steps"], cfg["every"]):
        o.step(cfg["every"])
        hist.append(field_energy(o.spatial))
    return name, dtype_name, {"E": [h[0] for h in hist], "B": [h[1] for h in hist]}


def main():
    t0 = time.time()
    out = {name: {"config": cfg} for name, cfg in CONFIGS.items()}
    jobs = [(n, d) for n in CONFIGS for d in ("fp64", "fp32")]
    threads = max(1, (os.cpu_count() or 4) // len(jobs))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    # spawned workers: no fork of a process that may hold threads
    import multiprocessing as mp
    with ProcessPoolExecutor(len(jobs), mp_context=mp.get_context("spawn")) as ex:
        for name, dname, h in ex.map(run_oracle, *zip(*jobs)):
            out[name][dname] = h
            print(name, dname, "done", round(time.time() - t0, 1), "s", flush=True)
    with open(os.path.join(HERE, "config_histories.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
