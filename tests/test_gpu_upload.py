"""spx_add_species uploads the caller's arrays in chunks of 2^22 particles
through a two-buffer device ring: species of several chunks (the last one
ragged), in shuffled order, must come back exactly as they went in, and the
bounds and Lorentz-factor checks must name particles of any chunk."""
import numpy as np
import pytest

from conftest import test_params

pytestmark = pytest.mark.gpu

CHUNK = 1 << 22


def _cfg(**kw):
    from spectral_rs_b200.config import Config, Setup, Output
    return Config(test_params(**kw), Setup(10), Output(False, False, 1, 1, 1, 1))


def _shuffled_species(p, ppc, seed):
    """A thermal species of 2 full chunks and a ragged third, in random order."""
    from spectral_rs_b200.init import positions, draws, velocities
    rng = np.random.default_rng(seed)
    ix, iy, dx, dy = positions(p.size_x, p.size_y, p.delta, ppc, None, None, True, rng)
    nrm, uni = draws(len(ix), rng)
    px, py, pz, psa = velocities(nrm, uni, p.c, 0.1, 1.0, 1.0)
    perm = rng.permutation(len(ix))
    return {k: v[perm] for k, v in dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa).items()}


def _add(sim, a):
    return sim.add_species(-1.0, 1.0, 0.1, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])


CFG = dict(size_x=512, size_y=256, delta=0, c=3.0, dt=0.1, dens=66, periodic_x=True)


def test_chunked_upload_round_trip():
    from spectral_rs_b200 import Sim
    cfg = _cfg(**CFG)
    a = _shuffled_species(cfg.params, 66, 3)
    n = len(a["ix"])
    assert 2 * CHUNK < n < 3 * CHUNK
    with Sim(cfg) as sim:
        pr = _add(sim, a)
        g = pr.state()
        for k in ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa"):
            assert np.array_equal(g[k], a[k].astype(g[k].dtype)), k
        sim.prepare()
        sim.step(1)  # the slots the upload filled are the ones the kernels walk


def test_chunked_upload_plain_path():
    """The plain path stores global positions x = ix + dx (FP32) in the caller's order."""
    from spectral_rs_b200 import Sim
    cfg = _cfg(**CFG)
    a = _shuffled_species(cfg.params, 66, 4)
    f = np.float32
    with Sim(cfg, path="plain") as sim:
        g = _add(sim, a).state()
    for c, d in (("ix", "dx"), ("iy", "dy")):
        x = (a[c].astype(f) + a[d]).astype(f)
        cx = np.floor((x + f(0.5)).astype(f))
        assert np.array_equal(g[c], cx.astype(np.uint64)), c
        assert np.array_equal(g[d], (x - cx).astype(f)), d
    for k in ("px", "py", "pz"):
        assert np.array_equal(g[k], a[k]), k


@pytest.mark.parametrize("where", ["first", "last"])
def test_chunked_upload_checks_every_chunk(where):
    from spectral_rs_b200 import _lib, Sim
    cfg = _cfg(**CFG)
    a = _shuffled_species(cfg.params, 66, 5)
    n = len(a["ix"])
    i_bad = 11 if where == "first" else n - 3
    with Sim(cfg) as sim:
        bad = dict(a, iy=a["iy"].copy())
        bad["iy"][i_bad] = cfg.params.size_y + 1
        with pytest.raises(_lib.SpxError) as ei:
            _add(sim, bad)
        assert ei.value.code == 3 and f"particle {i_bad} " in str(ei.value)  # SPX_ERR_BOUNDS
        bad = dict(a, psa=a["psa"].copy())
        bad["psa"][i_bad] = bad["psa"][i_bad] * np.float32(1.5)
        with pytest.raises(_lib.SpxError) as ei:
            _add(sim, bad)
        assert ei.value.code == 7  # SPX_ERR_GAMMA
        assert _add(sim, a).sid == 0  # neither failure added a species; the context stays usable
        sim.prepare()
        sim.step(1)


def test_upload_scratch_grows_and_reads_page_locked_arrays():
    """A small species, then a large one from page-locked host memory (the
    context's upload scratch grows between them), then a small one again."""
    import torch
    from spectral_rs_b200 import Sim
    cfg = _cfg(**CFG)
    big = _shuffled_species(cfg.params, 66, 6)
    pinned = {}
    for k, v in big.items():
        t = torch.empty(len(v), dtype=torch.int64 if v.dtype == np.uint64 else torch.float32, pin_memory=True)
        t.numpy().view(v.dtype)[:] = v
        pinned[k] = t.numpy().view(v.dtype)
    small = {k: v[:1000].copy() for k, v in big.items()}
    with Sim(cfg) as sim:
        prs = [_add(sim, small), _add(sim, pinned), _add(sim, small)]
        for pr, a in zip(prs, (small, big, small)):
            g = pr.state()
            for k in ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa"):
                assert np.array_equal(g[k], a[k].astype(g[k].dtype)), k


def test_device_init_in_chunks_matches_a_single_chunk():
    """spx_init_species generates a species chunk by chunk (particle i depends only
    on i and the seed): the first rows of a 3-chunk species equal the whole of a
    one-chunk species on a grid of fewer rows, every cell holds ppc particles, and
    the plain path holds the same particles."""
    from spectral_rs_b200 import Sim
    big_cfg = _cfg(**CFG)
    small_cfg = _cfg(**dict(CFG, size_y=8))
    args = (-1.0, 1.0, 0.1, 66, 0, 512)
    kw = dict(gamma_drift=1.2, sign_x=1.0, random_positions=True, seed=9)
    with Sim(big_cfg) as sim:
        big = sim.init_species(*args, **kw).state()
        sim.prepare()
        sim.step(1)
    assert 2 * CHUNK < len(big["ix"]) < 3 * CHUNK
    with Sim(small_cfg) as sim:
        small = sim.init_species(*args, **kw).state()
    n = len(small["ix"])
    for k in ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa"):
        assert np.array_equal(big[k][:n], small[k]), k
    assert np.all(np.bincount((big["iy"] - 1) * 512 + (big["ix"] - 1)) == 66)
    with Sim(big_cfg, path="plain") as sim:
        plain = sim.init_species(*args, **kw).state()
    for k in ("px", "py", "pz"):
        assert np.array_equal(plain[k], big[k]), k
    f = np.float32
    for c, d in (("ix", "dx"), ("iy", "dy")):
        x = (big[c].astype(f) + big[d]).astype(f)
        cx = np.floor((x + f(0.5)).astype(f))
        assert np.array_equal(plain[c], cx.astype(np.uint64)), c
        assert np.array_equal(plain[d], (x - cx).astype(f)), d


def test_device_init_partial_columns_against_a_wall():
    """Columns [x0, x1) of a wall grid (with the mirrored left wall): the slot
    capacity comes from ppc before any particle exists; the species runs a few
    steps against the wall."""
    from spectral_rs_b200 import Sim
    cfg = _cfg(size_x=512, size_y=64, delta=8, c=3.0, dt=0.1, dens=16, periodic_x=False, left_wall=True)
    with Sim(cfg) as sim:
        pr = sim.init_species(-1.0, 1.0, 0.1, 16, 8, 504, gamma_drift=1.1, sign_x=1.0, seed=3)
        st = pr.state()
        counts = np.bincount((st["iy"] - 1) * 512 + (st["ix"] - 1), minlength=512 * 64).reshape(64, 512)
        assert np.all(counts[:, 8:504] == 16) and counts[:, :8].sum() == 0 and counts[:, 504:].sum() == 0
        sim.prepare()
        sim.step(5)
        assert len(pr.state()["ix"]) == 64 * 496 * 16
