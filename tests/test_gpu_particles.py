"""GPU particle kernels against the CPU oracle (FP32 reference path and FP64 dprec path).

Bit-exact on identical inputs: cell indices (ix, iy), offsets (dx, dy), momenta
and Lorentz factors after boris_push and after move_and_deposit (the particle
TU is built with -fmad=false, IEEE div/sqrt, exactly like the reference's
Rust arithmetic).  Deposited J / rho / dens differ only by summation order:
compared with a relative tolerance.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from conftest import test_params

pytestmark = pytest.mark.gpu

DEP_RTOL = 4e-6  # summation-order tolerance on deposited moments (relative to max |field|)


def _cfg(**kw):
    from spectral_rs_b200.config import Config, Setup, Output
    return Config(test_params(**kw), Setup(10), Output(False, False, 1, 1, 1, 1))


def _species(p, ppc, vth, gamma, sign, seed, random_positions=True, x0=None, x1=None):
    from spectral_rs_b200.init import positions, draws, velocities
    rng = np.random.default_rng(seed)
    ix, iy, dx, dy = positions(p.size_x, p.size_y, p.delta, ppc, x0, x1, random_positions, rng)
    nrm, uni = draws(len(ix), rng)
    px, py, pz, psa = velocities(nrm, uni, p.c, vth, gamma, sign)
    return dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)


def _pair(cfg, specs, dtype=np.float32, path=None):
    from spectral_rs_b200 import Sim
    sim = Sim(cfg, path=path)
    o = orc.OracleSim.from_params(cfg.params, dtype=dtype)
    for (q, m, vth, a) in specs:
        sim.add_species(q, m, vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
        o.add_species(q, m, vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
    return sim, o


def _random_fields(sim, o, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    for name in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        f = (rng.standard_normal((sim.size_y + 2, sim.size_x + 2)) * scale).astype(np.float32)
        sim.flds.set_spatial(name, f)
        o.set_spatial(name, f.astype(o.dtype))


def _assert_state_equal(g, r, keys=("ix", "iy", "dx", "dy", "px", "py", "pz", "psa")):
    for k in keys:
        assert np.array_equal(g[k], r[k].astype(g[k].dtype)), (k, np.flatnonzero(g[k] != r[k])[:5])


def _assert_moments_close(sim, o, names=("Jx", "Jy", "Jz", "Rho", "Dens"), rtol=DEP_RTOL):
    dens = np.max(np.abs(o.spatial("Dens")))
    for name in names:
        g, r = sim.flds.spatial(name), o.spatial(name).astype(np.float64)
        # charge of +-1 species cancels: measure its error against the number density
        scale = max(np.max(np.abs(r)), dens if name == "Rho" else 0.0, 1e-30)
        err = np.max(np.abs(g - r)) / scale
        assert err < rtol, (name, err)


TILES = [(0, 0), (16, 16), (16, 8)]  # the library's choice (8x8), the 16x16 and 16x8 instantiations


@pytest.mark.parametrize("tile", TILES)
@pytest.mark.parametrize("periodic", [True, False])
def test_boris_push_bit_exact(periodic, tile):
    cfg = _cfg(size_x=64, size_y=32, delta=6, c=4.5, dt=0.1, dens=8, periodic_x=periodic, left_wall=not periodic,
               tile_x=tile[0], tile_y=tile[1])
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 1)),
             (-1.0, 1.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 2))]
    sim, o = _pair(cfg, specs)
    _random_fields(sim, o, 3)
    for s in range(2):
        sim.prtls[s].boris_push()
        o.boris_push(s)
        _assert_state_equal(sim.prtls[s].state(), o.state(s))
    sim.close()


@pytest.mark.parametrize("tile", TILES)
@pytest.mark.parametrize("periodic", [True, False])
def test_move_and_deposit_bit_exact(periodic, tile):
    cfg = _cfg(size_x=64, size_y=32, delta=6, c=4.5, dt=0.1, dens=8, periodic_x=periodic, left_wall=not periodic,
               tile_x=tile[0], tile_y=tile[1])
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 11)),
             (-1.0, 1.0, 0.3, _species(p, 8, 0.3, 1.2, 1.0, 12))]
    sim, o = _pair(cfg, specs)
    for s in range(2):
        sim.move_and_deposit(sim.prtls[s])
        o.move_and_deposit(s)
        _assert_state_equal(sim.prtls[s].state(), o.state(s))
    _assert_moments_close(sim, o)
    for name in ("Jx", "Jy", "Jz", "Rho", "Dens"):
        sim.flds.deposit_ghosts(name)
    o.fold_sources()
    _assert_moments_close(sim, o)
    sim.close()


def _uneven_species(p, seed, vth, gamma):
    """Clustered occupancy: every eleventh cell holds 40 particles, the others 0-2, so a warp's
    cells hold very different counts and its balanced rounds hand the excess of the full
    cells to the lanes of the empty ones (helper rounds)."""
    from spectral_rs_b200.init import draws, velocities
    rng = np.random.default_rng(seed)
    ix, iy = [], []
    for y in range(1, p.size_y + 1):
        for x in range(p.delta + 1, p.size_x - p.delta + 1):
            n = 40 if (7 * x + 3 * y) % 11 == 0 else int(rng.integers(0, 3))
            ix += [x] * n
            iy += [y] * n
    ix, iy = np.array(ix, dtype=np.uint64), np.array(iy, dtype=np.uint64)
    n = len(ix)
    dx = (rng.random(n, dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    dy = (rng.random(n, dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    nrm, uni = draws(n, rng)
    px, py, pz, psa = velocities(nrm, uni, p.c, vth, gamma, 1.0)
    return dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)


@pytest.mark.parametrize("tile", [(8, 8), (16, 16), (16, 8)])
@pytest.mark.parametrize("periodic", [True, False])
def test_uneven_cells_bit_exact(periodic, tile):
    """Cells with very different counts (excess particles moved in helper rounds): particle
    state bit-exact and deposits within tolerance over three push + move cycles."""
    cfg = _cfg(size_x=64, size_y=32, delta=6, c=4.5, dt=0.1, dens=8, periodic_x=periodic, left_wall=not periodic,
               tile_x=tile[0], tile_y=tile[1])
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _uneven_species(p, 21, 0.1, 1.0050378)),
             (-1.0, 1.0, 0.3, _uneven_species(p, 22, 0.3, 1.2))]
    sim, o = _pair(cfg, specs)
    _random_fields(sim, o, 23)
    for cycle in range(3):
        for s in range(2):
            sim.prtls[s].boris_push()
            o.boris_push(s)
            _assert_state_equal(sim.prtls[s].state(), o.state(s))
        sim.zero_sources()
        o.zero_sources()
        for s in range(2):
            sim.move_and_deposit(sim.prtls[s])
            o.move_and_deposit(s)
            _assert_state_equal(sim.prtls[s].state(), o.state(s))
        _assert_moments_close(sim, o)
    sim.close()


def test_wall_reflection_bit_exact():
    # fast particles driven into the reflecting wall (src/prtls.rs:153-188), several moves
    cfg = _cfg(size_x=32, size_y=16, delta=4, c=4.5, dt=0.1, dens=4, periodic_x=False)
    p = cfg.params
    a = _species(p, 4, 0.05, 3.0, 1.0, 21, x0=20, x1=28)
    sim, o = _pair(cfg, [(-1.0, 1.0, 0.05, a)])
    for _ in range(12):
        sim.move_and_deposit(sim.prtls[0])
        o.move_and_deposit(0)
    g = sim.prtls[0].state()
    _assert_state_equal(g, o.state(0))
    assert np.max(g["ix"]) <= p.size_x + 1 - p.delta + 1
    sim.close()


def test_wall_assertion_like_the_reference():
    """Without the optional left wall, a particle reaching ix <= delta trips the
    reference's assertion (src/prtls.rs:163-170): an error status on both sides."""
    from spectral_rs_b200 import _lib
    cfg = _cfg(size_x=32, size_y=16, delta=4, c=4.5, dt=0.1, dens=4, periodic_x=False)
    p = cfg.params
    a = _species(p, 4, 0.3, 1.0, 1.0, 23, x0=4, x1=8)  # hot plasma next to the left edge
    sim, o = _pair(cfg, [(-1.0, 1.0, 0.3, a)])
    with pytest.raises(_lib.SpxError) as ei:
        for _ in range(10):
            sim.move_and_deposit(sim.prtls[0])
    assert ei.value.code == 4  # SPX_ERR_WALL
    with pytest.raises(RuntimeError):
        for _ in range(10):
            o.move_and_deposit(0)
    sim.close()


def test_add_species_rejects_cells_outside_the_grid():
    """Prtl cell indices outside 1..size (the reference would index out of bounds):
    SPX_ERR_BOUNDS naming the first offending particle; the context stays usable."""
    from spectral_rs_b200 import _lib, Sim
    cfg = _cfg(size_x=32, size_y=16, delta=0, c=3.0, dt=0.1, dens=4, periodic_x=True)
    p = cfg.params
    a = _species(p, 4, 0.05, 1.0, 1.0, 29)
    bad = dict(a)
    bad["ix"] = a["ix"].copy()
    bad["ix"][[100, 7]] = [p.size_x + 1, 0]
    sim = Sim(cfg)
    with pytest.raises(_lib.SpxError) as ei:
        sim.add_species(-1.0, 1.0, 0.05, bad["ix"], bad["iy"], bad["dx"], bad["dy"], bad["px"], bad["py"],
                        bad["pz"], bad["psa"])
    assert ei.value.code == 3 and "particle 7 " in str(ei.value)  # SPX_ERR_BOUNDS
    sim.add_species(-1.0, 1.0, 0.05, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
    sim.prepare()
    sim.step(2)
    sim.close()


def test_compensated_currents_track_fp64():
    """compensated = true: Kahan sums of J per owner cell, compensation carried through the
    tile flush.  Particle state is untouched (bit-exact with the FP32 oracle); J moves closer
    to the FP64 deposit than the plain FP32 sums (512 particles per cell)."""
    errs = {}
    for comp in (False, True):
        cfg = _cfg(size_x=16, size_y=16, delta=0, c=3.0, dt=0.1, dens=512, periodic_x=True, compensated=comp)
        p = cfg.params
        a = _species(p, 512, 0.2, 1.0, 1.0, 31)
        sim, o = _pair(cfg, [(-1.0, 1.0, 0.2, a)])
        o64 = orc.OracleSim.from_params(p, dtype=np.float64)
        o64.add_species(-1.0, 1.0, 0.2, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
        sim.move_and_deposit(sim.prtls[0])
        o.move_and_deposit(0)
        o64.move_and_deposit(0)
        _assert_state_equal(sim.prtls[0].state(), o.state(0))
        errs[comp] = max(np.max(np.abs(sim.flds.spatial(n) - o64.spatial(n))) / np.max(np.abs(o64.spatial(n)))
                         for n in ("Jx", "Jy", "Jz"))
        sim.close()
    print(f"\nrelative J error vs FP64: FP32 sums {errs[False]:.2e}, compensated {errs[True]:.2e}")
    assert errs[True] < 0.5 * errs[False]


@pytest.mark.parametrize("grid", [(64, 32), (512, 256)])
@pytest.mark.parametrize("tile", TILES)
@pytest.mark.parametrize("periodic", [True, False])
def test_fused_step_equals_per_phase_sequence(periodic, tile, grid):
    """spx_step (push of step t fused with move+deposit of t+1, CUDA graphs) must
    equal the reference's sequence of per-phase calls on the same device.  The
    64x32 grid is small enough for the fused kernel to take one CTA per (tile,
    species); the 512x256 grid runs both species in every CTA."""
    from spectral_rs_b200 import Sim
    cfg = _cfg(size_x=grid[0], size_y=grid[1], delta=0 if periodic else 6, c=3.0, dt=0.1, dens=8,
               periodic_x=periodic, left_wall=not periodic, n_pass=2, tile_x=tile[0], tile_y=tile[1])
    p = cfg.params
    sp = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0, 1.0, 31)), (-1.0, 1.0, 0.1, _species(p, 8, 0.1, 1.0, 1.0, 32))]
    fused = Sim(cfg)
    phased = Sim(cfg)
    for (q, m, v, a) in sp:
        for s in (fused, phased):
            s.add_species(q, m, v, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
    fused.prepare()
    phased.prepare()
    fused.step(5)
    for _ in range(5):
        phased.zero_sources()
        for pr in phased.prtls:
            phased.move_and_deposit(pr)
        for name in ("Jx", "Jy", "Jz", "Rho", "Dens"):
            phased.flds.deposit_ghosts(name)
        phased.flds.update()
        for pr in phased.prtls:
            pr.boris_push()
    # deposits are summed in a different order on every run, so after the first
    # field solve the two agree to rounding, not bit for bit
    for s in range(2):
        a, b = fused.prtls[s].state(), phased.prtls[s].state()
        assert np.mean((a["ix"] != b["ix"]) | (a["iy"] != b["iy"])) < 1e-3
        assert np.max(np.abs(a["px"] - b["px"])) < 1e-4 * np.max(np.abs(b["px"]))
    for name in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        a, b = fused.flds.spatial(name), phased.flds.spatial(name)
        assert np.max(np.abs(a - b)) <= 1e-4 * max(np.max(np.abs(b)), 1e-30), name
    fused.close()
    phased.close()


@pytest.mark.parametrize("periodic,steps", [(True, 20), (False, 20)])
def test_run_vs_oracle(periodic, steps):
    """The full loop (src/lib.rs:130-200) against the FP32 and FP64 oracles."""
    from spectral_rs_b200 import Sim
    cfg = _cfg(size_x=64, size_y=32, delta=0 if periodic else 6, c=3.0, dt=0.1, dens=8, periodic_x=periodic,
               left_wall=not periodic, n_pass=4)
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 41, random_positions=True)),
             (-1.0, 1.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 42, random_positions=True))]
    sim, o32 = _pair(cfg, specs, np.float32)
    _, o64 = None, orc.OracleSim.from_params(p, dtype=np.float64)
    for (q, m, v, a) in specs:
        o64.add_species(q, m, v, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
    sim.prepare()
    o32.prepare()
    o64.prepare()
    sim.step(steps)
    o32.step(steps)
    o64.step(steps)
    for name in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Dens"):
        # interior cells (Dens's ghost frame holds raw, unfolded deposits, which a particle on
        # the periodic edge splits differently for an ulp of difference in its position)
        g, r = sim.flds.spatial(name)[1:-1, 1:-1].astype(np.float64), o64.spatial(name)[1:-1, 1:-1]
        r32 = o32.spatial(name)[1:-1, 1:-1].astype(np.float64)
        scale = max(np.max(np.abs(r)), 1e-30)
        err_gpu, err_ref = np.max(np.abs(g - r)) / scale, np.max(np.abs(r32 - r)) / scale
        # GPU FP32 error against FP64 within a small factor of the reference FP32 path's own error
        assert err_gpu < max(10 * err_ref, 1e-5), (name, err_gpu, err_ref)
    for s in range(2):
        g, r = sim.prtls[s].state(), o32.state(s)
        mism = np.mean((g["ix"] != r["ix"]) | (g["iy"] != r["iy"]))
        assert mism < 1e-3, mism
        assert np.max(np.abs(g["px"] - r["px"])) < 1e-3 * max(np.max(np.abs(r["px"])), 1e-30)
    sim.close()


def test_plain_path_vs_oracle():
    """The plain FP32 baseline (global positions, unfused, atomics) stays within tolerance."""
    cfg = _cfg(size_x=64, size_y=32, delta=0, c=4.5, dt=0.1, dens=8, periodic_x=True, n_pass=4)
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0, 1.0, 51)), (-1.0, 1.0, 0.1, _species(p, 8, 0.1, 1.0, 1.0, 52))]
    sim, o = _pair(cfg, specs, np.float64, path="plain")
    sim.prepare()
    o.prepare()
    sim.step(10)
    o.step(10)
    for name in ("Ex", "Ey", "Bz", "Jx", "Dens"):
        g, r = sim.flds.spatial(name)[1:-1, 1:-1], o.spatial(name)[1:-1, 1:-1]  # interior (see above)
        assert np.max(np.abs(g - r)) / max(np.max(np.abs(r)), 1e-30) < 1e-3, name
    for s in range(2):
        g, r = sim.prtls[s].state(), o.state(s)
        x_g = g["ix"].astype(np.float64) + g["dx"]
        x_r = r["ix"].astype(np.float64) + r["dx"]
        assert np.max(np.abs(x_g - x_r)) < 1e-2
    sim.close()


def test_slot_overflow_and_repack():
    """Slot capacity equal to the initial occupancy: every arrival overflows into
    the fallback list, which must give the same particles; spx_step then repacks."""
    cfg = _cfg(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, dens=4, periodic_x=True, n_pass=2, slot_capacity=-4)
    p = cfg.params
    a = _species(p, 4, 0.2, 1.0, 1.0, 61, random_positions=False)
    sim, o = _pair(cfg, [(-1.0, 1.0, 0.2, a)])
    for _ in range(6):
        sim.move_and_deposit(sim.prtls[0])
        o.move_and_deposit(0)
        _assert_state_equal(sim.prtls[0].state(), o.state(0))
    _assert_moments_close(sim, o)
    sim.prepare()
    o.prepare()
    sim.step(4)
    o.step(4)
    g, r = sim.prtls[0].state(), o.state(0)
    assert np.mean((g["ix"] != r["ix"]) | (g["iy"] != r["iy"])) < 1e-3
    assert len(g["ix"]) == len(a["ix"])
    sim.close()


def test_diag_counts_and_charge():
    cfg = _cfg(size_x=64, size_y=32, delta=0, c=4.5, dt=0.1, dens=8, periodic_x=True)
    p = cfg.params
    a = _species(p, 8, 0.1, 1.0, 1.0, 71)
    b = _species(p, 8, 0.1, 1.0, 1.0, 72)
    sim, o = _pair(cfg, [(1.0, 1.0, 0.1, a), (-1.0, 1.0, 0.1, b)])
    sim.prepare()
    d = sim.diag()
    assert d[4] == len(a["ix"]) + len(b["ix"])
    # kinetic energy, FP64 sum of m (gamma - 1) c^2
    o.prepare()
    ke = sum(np.sum((o.state(s)["psa"].astype(np.float64) - 1.0)) for s in range(2)) * 4.5 ** 2
    assert abs(d[2] - ke) <= 1e-6 * ke
    # net deposited charge of a neutral plasma after the fold is ~0
    assert abs(d[3]) < 1e-2 * len(a["ix"])
    sim.close()


def test_device_init_statistics():
    from spectral_rs_b200 import Sim
    cfg = _cfg(size_x=64, size_y=32, delta=0, c=4.5, dt=0.1, dens=16, periodic_x=True)
    with Sim(cfg) as sim:
        pr = sim.init_species(-1.0, 1.0, 0.1, 16, 0, 64, gamma_drift=0.0, random_positions=True, seed=5)
        st = pr.state()
        assert len(st["ix"]) == 64 * 32 * 16
        assert np.all((st["dx"] >= -0.5) & (st["dx"] < 0.5))
        assert abs(np.std(st["px"]) / (0.1 * 4.5) - 1) < 0.02
        assert abs(np.mean(st["py"])) < 0.01
        # every cell holds exactly ppc particles, in reference order
        assert np.all(np.bincount((st["iy"] - 1) * 64 + (st["ix"] - 1)) == 16)


def test_run_writes_the_reference_output_layout(tmp_path):
    """run() with write_output: output/dat_NNNNN/{x,y,u,gam}.npy (species 0, every stride-th
    particle) and flds/*.npy (interior, 1-D) at every output_interval (src/save/mod.rs:8-80).
    The t = 0 dump follows the pre-loop move: positions bit-exact with the oracle, sources
    within the deposit tolerance."""
    import os
    from spectral_rs_b200 import run
    from spectral_rs_b200.config import Config, Setup, Output
    from spectral_rs_b200.init import species_arrays
    from spectral_rs_b200.save import SAVED_FIELDS
    p = test_params(size_x=64, size_y=32, delta=0, c=3.0, dt=0.1, dens=8, periodic_x=True, n_pass=4,
                    random_positions=True, seed=5, mass_ratio=16.0, vth=0.1, gamma_inj=1.0050378)
    cfg = Config(p, Setup(10), Output(False, True, 1, 5, 3, 1))
    out = str(tmp_path / "output")
    run(cfg, out_dir=out)
    assert sorted(os.listdir(out)) == ["dat_00000", "dat_00001", "dat_00002"]
    o = orc.OracleSim.from_params(p, dtype=np.float32)
    for k, spec in enumerate(cfg.species_list()):
        a = species_arrays(p, spec, seed_offset=k)
        o.add_species(spec.charge, spec.mass, spec.vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                      a["psa"])
    o.prepare()
    r = o.state(0)
    d0 = os.path.join(out, "dat_00000")
    x = np.load(os.path.join(d0, "x.npy"))
    assert x.dtype == np.float32 and len(x) == (len(r["ix"]) + 2) // 3
    assert np.array_equal(x, (r["ix"].astype(np.float32) + r["dx"])[::3])
    assert np.array_equal(np.load(os.path.join(d0, "y.npy")), (r["iy"].astype(np.float32) + r["dy"])[::3])
    assert np.array_equal(np.load(os.path.join(d0, "u.npy")), (r["px"] / np.float32(p.c))[::3])
    assert np.array_equal(np.load(os.path.join(d0, "gam.npy")), r["psa"][::3])
    for name in SAVED_FIELDS:
        f = np.load(os.path.join(d0, "flds", f"{name}.npy"))
        assert f.shape == (p.size_x * p.size_y,) and f.dtype == np.float32
        ref = o.spatial(name).reshape(p.size_y + 2, p.size_x + 2)[1:-1, 1:-1].reshape(-1)
        assert np.max(np.abs(f - ref)) <= DEP_RTOL * max(float(np.max(np.abs(ref))), 1e-30) + 1e-30, name
    for d in ("dat_00001", "dat_00002"):
        assert len(np.load(os.path.join(out, d, "gam.npy"))) == len(x)


@pytest.mark.parametrize("path", ["split", "plain"])
def test_tags_round_trip_through_fused_steps(path):
    """Prtl::tag / Prtl::track (src/prtls.rs:21-22) survive fused steps (particles change
    cells and slots), and spx_get_tracked gathers the tracking output of save_output
    (src/save/mod.rs:94-96) for exactly the tracked particles, in the reference's order."""
    cfg = _cfg(size_x=64, size_y=32, delta=6, c=3.0, dt=0.1, dens=8, periodic_x=False, left_wall=True, n_pass=4)
    p = cfg.params
    specs = [(1.0, 16.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 71)),
             (-1.0, 1.0, 0.1, _species(p, 8, 0.1, 1.0050378, 1.0, 72))]
    sim, _ = _pair(cfg, specs, path=path)
    pr = sim.prtls[1]
    n = len(pr)
    # defaults: tag = index (src/prtls.rs:213), particle 40 tracked (src/prtls.rs:79)
    t0, k0 = pr.tags()
    assert np.array_equal(t0, np.arange(n, dtype=np.uint64)) and np.flatnonzero(k0).tolist() == [40]
    rng = np.random.default_rng(5)
    tags = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    track = rng.random(n) < 0.01
    pr.set_tags(tags, track)
    sim.prepare()
    sim.step(7)
    t, k = pr.tags()
    assert np.array_equal(t, tags) and np.array_equal(k, track)
    ts, ks = pr.tags(stride=5)
    assert np.array_equal(ts, tags[::5]) and np.array_equal(ks, track[::5])
    x, y, g = pr.tracked()
    st = pr.state()
    f = np.float32
    c = f(p.c)
    sel = np.flatnonzero(track)
    assert len(x) == len(sel)
    assert np.array_equal(x, ((st["ix"][sel].astype(f) + st["dx"][sel]) / c).astype(f))
    assert np.array_equal(y, ((st["iy"][sel].astype(f) + st["dy"][sel]) / c).astype(f))
    assert np.array_equal(g, st["psa"][sel])
    # the first species keeps its defaults
    x0, _, _ = sim.prtls[0].tracked()
    st0 = sim.prtls[0].state()
    assert len(x0) == 1 and x0[0] == ((f(st0["ix"][40]) + st0["dx"][40]) / c).astype(f)
    sim.close()
