"""save_output (src/save/mod.rs:8-80): the reference's .npy output layout.

output/dat_{t/output_interval:05}/
  x.npy, y.npy   species 0, every stride-th particle, x = ix + dx (ghost offset included)
  u.npy          px / c
  gam.npy        Lorentz factor
  flds/{Jx,Jy,Jz,Ex,Ey,Ez,Bx,By,Bz,Dens}.npy   1-D, interior cells, row-major
All arrays are the reference's `Float` (float32).  Rho (dsty) is not saved.
"""
import os

import numpy as np

SAVED_FIELDS = ("Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Dens")


def save_output(t, sim, out_dir="output"):
    cfg = sim.config.output
    if t % cfg.output_interval != 0:
        return None
    prefix = os.path.join(out_dir, f"dat_{t // cfg.output_interval:05d}")
    os.makedirs(os.path.join(prefix, "flds"), exist_ok=True)
    st = sim.prtls[0].state(stride=cfg.stride)
    f = np.float32
    np.save(os.path.join(prefix, "x.npy"), (st["ix"].astype(f) + st["dx"]).astype(f))
    np.save(os.path.join(prefix, "y.npy"), (st["iy"].astype(f) + st["dy"]).astype(f))
    np.save(os.path.join(prefix, "u.npy"), (st["px"] / f(sim.c)).astype(f))
    np.save(os.path.join(prefix, "gam.npy"), st["psa"])
    for name in SAVED_FIELDS:
        np.save(os.path.join(prefix, "flds", f"{name}.npy"), sim.flds.spatial(name, with_ghosts=False).reshape(-1))
    return prefix
