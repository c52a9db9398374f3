"""Batched ensemble (spx_batch_*): uneven simulations stepped together must
match the same simulations stepped one by one through spx_step."""
import numpy as np
import pytest

from conftest import test_params

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    from spectral_rs_b200.config import Config, Setup, Output
    return Config(test_params(**kw), Setup(10), Output(False, False, 1, 1, 1, 1))


def _arrays(p, ppc, vth, gamma, seed):
    from spectral_rs_b200.init import positions, draws, velocities
    rng = np.random.default_rng(seed)
    ix, iy, dx, dy = positions(p.size_x, p.size_y, p.delta, ppc, None, None, True, rng)
    nrm, uni = draws(len(ix), rng)
    px, py, pz, psa = velocities(nrm, uni, p.c, vth, gamma, 1.0)
    return dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)


def _member(kind, size_x, size_y, dens, n_pass):
    if kind == "periodic":
        return _cfg(size_x=size_x, size_y=size_y, delta=0, c=3.0, dt=0.1, dens=dens, periodic_x=True, n_pass=n_pass)
    return _cfg(size_x=size_x, size_y=size_y, delta=6, c=3.0, dt=0.1, dens=dens, periodic_x=False, left_wall=True,
                n_pass=n_pass)


# mixed boundaries run the batch kernel's generic form, uniform ones its periodic / wall forms
@pytest.mark.parametrize("kinds", [("periodic", "wall", "periodic"), ("periodic",) * 3, ("wall",) * 3])
def test_batch_matches_single_simulations(kinds):
    _batch_vs_singles([_member(kinds[0], 64, 32, 8, 4), _member(kinds[1], 128, 64, 4, 2),
                       _member(kinds[2], 32, 32, 16, 4)])


def test_batch_members_sharing_a_grid():
    """The field phase runs once per group of members with one grid and pass count
    (blockIdx.z = member): members of a group differ in density (the per-member
    constants of the tables) and boundaries, pass counts split groups, and a pass count
    beyond the fused filter (or none) takes the member-by-member fallback."""
    _batch_vs_singles([_member("periodic", 64, 32, 8, 4), _member("wall", 64, 32, 4, 4),
                       _member("periodic", 64, 32, 16, 4), _member("periodic", 64, 32, 8, 2),
                       _member("periodic", 32, 32, 8, 0), _member("wall", 32, 32, 4, 17),
                       _member("periodic", 32, 32, 8, 4)])


def _batch_vs_singles(cfgs):
    from spectral_rs_b200 import Sim, Batch
    species = []
    for k, cfg in enumerate(cfgs):
        p = cfg.params
        species.append([(1.0, 16.0, 0.1, _arrays(p, p.dens, 0.1, 1.02, 10 * k + 1)),
                        (-1.0, 1.0, 0.1, _arrays(p, p.dens, 0.1, 1.02, 10 * k + 2))])
    singles = []
    for cfg, sp in zip(cfgs, species):
        s = Sim(cfg)
        for q, m, v, a in sp:
            s.add_species(q, m, v, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
        s.prepare()
        s.step(12)
        singles.append(s)
    with Batch(cfgs) as b:
        for sim, sp in zip(b.sims, species):
            for q, m, v, a in sp:
                sim.add_species(q, m, v, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
        b.prepare()
        b.step(5)
        b.set_timing(True)
        b.step(2)  # uncaptured, timed steps in between captured ones
        b.set_timing(False)
        b.step(5)
        assert b.timing()[1] > 0
        for ghosts in (True, False):  # the batched read-back equals each member's own
            for name in ("Ex", "Jy", "Dens"):
                for x, bs in zip(b.get_field(name, with_ghosts=ghosts), b.sims):
                    assert np.array_equal(x, bs.flds.spatial(name, with_ghosts=ghosts)), (name, ghosts)
        for s, bs in zip(singles, b.sims):
            for name in ("Ex", "Ey", "Bz", "Jx", "Dens"):  # interior cells (raw ghost deposits in Dens)
                x, y = bs.flds.spatial(name)[1:-1, 1:-1], s.flds.spatial(name)[1:-1, 1:-1]
                assert np.max(np.abs(x - y)) <= 2e-4 * max(float(np.max(np.abs(y))), 1e-30), name
            for k in range(2):
                x, y = bs.prtls[k].state(), s.prtls[k].state()
                assert np.mean((x["ix"] != y["ix"]) | (x["iy"] != y["iy"])) < 1e-3
                assert np.max(np.abs(x["px"] - y["px"])) < 1e-3 * np.max(np.abs(y["px"]))
    for s in singles:
        s.close()


def test_batch_rejects_separate_steps():
    from spectral_rs_b200 import Batch, _lib
    cfgs = [_cfg(size_x=32, size_y=32, delta=0, c=4.5, dt=0.1, dens=4, periodic_x=True)] * 2
    with Batch(cfgs) as b:
        for k, sim in enumerate(b.sims):
            a = _arrays(sim.config.params, 4, 0.1, 1.0, k)
            sim.add_species(-1.0, 1.0, 0.1, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
        b.prepare()
        b.sims[0].move_and_deposit(b.sims[0].prtls[0])  # steps one simulation alone
        with pytest.raises(_lib.SpxError):
            b.step(1)
