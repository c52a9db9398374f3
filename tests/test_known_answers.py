"""Known-answer tests of the hot path's physics.

The reference pins none of update_position, apply_bc, deposit_current,
calc_density, boris_push or Flds::update with tests, so these properties pin
the oracle (CPU, FP64 and FP32) and, under the gpu marker, the CUDA path:
  - seeded host init equals the oracle's restatement of src/prtls.rs:222-250 bit for bit
  - uniform E: linear momentum growth; uniform Bz: Boris gyration angle 2 atan(alpha B / gamma)
  - deposition: number density sums to the particle count, charge to sum(q)
  - reflecting walls only flip signs: |p| is conserved exactly
  - vacuum light wave: E^{n+1} + E^{n-1} = (2 - (c dt k)^2) E^n, i.e. sin(w dt/2) = c dt k / 2
  - the spectral correction leaves i k.E = rho at every non-Nyquist k
"""
import numpy as np
import pytest

from oracle import oracle as orc
from conftest import test_params


def _species(p, ppc, vth, gamma, sign, seed, x0=None, x1=None, random_positions=True):
    from spectral_rs_b200.init import positions, draws, velocities
    rng = np.random.default_rng(seed)
    ix, iy, dx, dy = positions(p.size_x, p.size_y, p.delta, ppc, x0, x1, random_positions, rng)
    nrm, uni = draws(len(ix), rng)
    px, py, pz, psa = velocities(nrm, uni, p.c, vth, gamma, sign)
    return dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)


def _add(o, q, m, vth, a):
    o.add_species(q, m, vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])


def _uniform(o, p, name, value):
    o.set_spatial(name, np.full((p.size_y + 2, p.size_x + 2), value, dtype=o.dtype))


@pytest.mark.parametrize("gamma,sign", [(1.0, 1.0), (1.0050378, 1.0), (1.0206, -1.0), (10.0, 1.0)])
def test_init_velocities_numpy_matches_oracle(gamma, sign):
    from spectral_rs_b200.init import draws, velocities
    rng = np.random.default_rng(3)
    nrm, uni = draws(20000, rng)
    a = velocities(nrm, uni, 4.5, 0.1, gamma, sign)
    b = orc.init_velocities(nrm, uni, 4.5, 0.1, gamma, sign)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_uniform_E_linear_momentum():
    p = test_params(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, periodic_x=True)
    o = orc.OracleSim.from_params(p, dtype=np.float64)
    a = _species(p, 2, 0.0, 1.0, 1.0, 5)
    _add(o, -1.0, 1.0, 0.0, a)
    E0 = 0.3
    _uniform(o, p, "Ex", E0)
    p0 = o.state(0)["px"].copy()
    beta = (-1.0 / 1.0) * 0.5 * p.dt
    for _ in range(50):
        o.boris_push(0)
    np.testing.assert_allclose(o.state(0)["px"], p0 + 50 * 2 * beta * E0, rtol=1e-12, atol=1e-12)


def test_uniform_Bz_gyration():
    p = test_params(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, periodic_x=True)
    o = orc.OracleSim.from_params(p, dtype=np.float64)
    a = _species(p, 2, 0.3, 1.0, 1.0, 6)
    a["pz"][:] = 0.0
    a["psa"] = np.sqrt(1 + (a["px"].astype(np.float64) ** 2 + a["py"].astype(np.float64) ** 2) / p.c ** 2)
    _add(o, 1.0, 1.0, 0.3, a)
    B0 = 0.7
    _uniform(o, p, "Bz", B0)
    s0 = o.state(0)
    alpha = 1.0 * 0.5 * p.dt / p.c
    nsteps = 40
    for _ in range(nsteps):
        o.boris_push(0)
    s1 = o.state(0)
    np.testing.assert_allclose(np.hypot(s1["px"], s1["py"]), np.hypot(s0["px"], s0["py"]), rtol=1e-13)
    theta = 2 * np.arctan(alpha * B0 / s0["psa"])  # Boris rotation per step
    ang = np.angle((s1["px"] + 1j * s1["py"]) / (s0["px"] + 1j * s0["py"]))
    expect = np.angle(np.exp(-1j * nsteps * theta))  # positive charge, Bz > 0: clockwise
    np.testing.assert_allclose(np.angle(np.exp(1j * (ang - expect))), 0, atol=1e-10)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_deposit_sums(dtype):
    p = test_params(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, periodic_x=True)
    o = orc.OracleSim.from_params(p, dtype=dtype)
    a, b = _species(p, 8, 0.2, 1.0, 1.0, 8), _species(p, 4, 0.2, 1.0, 1.0, 9)
    _add(o, 1.0, 16.0, 0.2, a)
    _add(o, -1.0, 1.0, 0.2, b)
    o.move_and_deposit(0)
    o.move_and_deposit(1)
    o.fold_sources()
    n = len(a["ix"]) + len(b["ix"])
    dens = o.spatial("Dens")[1:-1, 1:-1].astype(np.float64).sum()
    rho = o.spatial("Rho")[1:-1, 1:-1].astype(np.float64).sum()
    tol = 1e-9 if dtype == np.float64 else 2e-5
    assert abs(dens - n) < tol * n
    assert abs(rho - (len(a["ix"]) - len(b["ix"]))) < tol * n


def test_walls_conserve_momentum_magnitude():
    p = test_params(size_x=32, size_y=16, delta=4, c=4.5, dt=0.1, periodic_x=False, left_wall=True)
    o = orc.OracleSim.from_params(p, dtype=np.float32)
    a = _species(p, 4, 0.4, 1.0, 1.0, 10)
    _add(o, -1.0, 1.0, 0.4, a)
    p0 = np.sort(np.abs(a["px"]))
    for _ in range(60):
        o.move_and_deposit(0)
    s = o.state(0)
    assert np.array_equal(np.sort(np.abs(s["px"])), p0)
    assert s["ix"].min() >= p.delta and s["ix"].max() <= p.size_x + 2 - p.delta


def _light_wave(sim, p, m, steps):
    """Ey = cos(k x) in vacuum, advanced by Flds::update; `sim` is the oracle or a GPU Sim."""
    x = np.arange(p.size_x + 2) - 1
    k = 2 * np.pi * m / p.size_x
    ey = np.tile(np.cos(k * x), (p.size_y + 2, 1))
    gpu = hasattr(sim, "flds")
    if gpu:
        sim.flds.set_spatial("Ey", ey.astype(np.float32))
    else:
        sim.set_spatial("Ey", ey)
    hist = []
    for _ in range(steps):
        if gpu:
            sim.flds.update()
            f = sim.flds.spatial("Ey")
        else:
            sim.fields_update()
            f = sim.spatial("Ey")
        hist.append(f[1:-1, 1:-1].astype(np.float64))
    return k, hist


@pytest.mark.parametrize("m", [1, 5, 12])
def test_vacuum_light_wave_dispersion(m):
    p = test_params(size_x=64, size_y=8, delta=0, c=4.5, dt=0.1, n_pass=0, periodic_x=True)
    o = orc.OracleSim.from_params(p, dtype=np.float64)
    k, h = _light_wave(o, p, m, 12)
    a = p.c * p.dt * k
    for n in range(1, len(h) - 1):
        np.testing.assert_allclose(h[n + 1] + h[n - 1], (2 - a * a) * h[n], atol=1e-11)


def _gauss_check(e_x, e_y, dsty, p):
    nx, ny = p.size_x, p.size_y
    kx, ky, _ = orc.wave_numbers(nx, ny)
    kx, ky = kx.reshape(ny, nx), ky.reshape(ny, nx)
    Ex, Ey = np.fft.fft2(e_x), np.fft.fft2(e_y)
    rho = np.fft.fft2(dsty) / p.dens
    res = kx * Ex + ky * Ey + 1j * rho
    mask = np.ones((ny, nx), bool)
    mask[0, 0] = False
    mask[:, nx // 2] = False
    mask[ny // 2, :] = False
    return np.max(np.abs(res[mask])) / np.max(np.abs(rho[mask]))


def test_divergence_correction_gauss_law():
    p = test_params(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, dens=4, n_pass=0, periodic_x=True)
    o = orc.OracleSim.from_params(p, dtype=np.float64)
    rng = np.random.default_rng(12)
    shape = (p.size_y + 2, p.size_x + 2)
    for name in ("Ex", "Ey", "Rho"):
        o.set_spatial(name, rng.standard_normal(shape))
    rho_in = o.spatial("Rho")[1:-1, 1:-1].copy()
    o.fields_update()
    assert _gauss_check(o.spatial("Ex")[1:-1, 1:-1], o.spatial("Ey")[1:-1, 1:-1], rho_in, p) < 1e-12


# ------------------------------------------------------------------ the same properties on the GPU
@pytest.mark.gpu
def test_gpu_divergence_correction_gauss_law():
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    p = test_params(size_x=32, size_y=16, delta=0, c=4.5, dt=0.1, dens=4, n_pass=0, periodic_x=True)
    rng = np.random.default_rng(12)
    shape = (p.size_y + 2, p.size_x + 2)
    with Sim(Config(p, Setup(1), Output(False, False, 1, 1, 1, 1))) as sim:
        for name in ("Ex", "Ey", "Rho"):
            sim.flds.set_spatial(name, rng.standard_normal(shape).astype(np.float32))
        rho_in = sim.flds.spatial("Rho")[1:-1, 1:-1].astype(np.float64)
        sim.flds.update()
        e_x = sim.flds.spatial("Ex")[1:-1, 1:-1].astype(np.float64)
        e_y = sim.flds.spatial("Ey")[1:-1, 1:-1].astype(np.float64)
        assert _gauss_check(e_x, e_y, rho_in, p) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("m", [1, 5, 12])
def test_gpu_vacuum_light_wave_dispersion(m):
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    p = test_params(size_x=64, size_y=8, delta=0, c=4.5, dt=0.1, n_pass=0, periodic_x=True)
    with Sim(Config(p, Setup(1), Output(False, False, 1, 1, 1, 1))) as sim:
        k, h = _light_wave(sim, p, m, 12)
    a = p.c * p.dt * k
    for n in range(1, len(h) - 1):
        np.testing.assert_allclose(h[n + 1] + h[n - 1], (2 - a * a) * h[n], atol=2e-5)


@pytest.mark.gpu
def test_gpu_deposit_sums():
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    p = test_params(size_x=64, size_y=32, delta=0, c=4.5, dt=0.1, periodic_x=True)
    a, b = _species(p, 8, 0.2, 1.0, 1.0, 8), _species(p, 4, 0.2, 1.0, 1.0, 9)
    with Sim(Config(p, Setup(1), Output(False, False, 1, 1, 1, 1))) as sim:
        for q, m, x in ((1.0, 16.0, a), (-1.0, 1.0, b)):
            sim.add_species(q, m, 0.2, x["ix"], x["iy"], x["dx"], x["dy"], x["px"], x["py"], x["pz"], x["psa"])
        sim.prepare()
        n = len(a["ix"]) + len(b["ix"])
        dens = sim.flds.spatial("Dens")[1:-1, 1:-1].astype(np.float64).sum()
        rho = sim.flds.spatial("Rho")[1:-1, 1:-1].astype(np.float64).sum()
        assert abs(dens - n) < 2e-5 * n
        assert abs(rho - (len(a["ix"]) - len(b["ix"]))) < 2e-5 * n


def _thermal_energy_growth(c, steps):
    """E-field energy after `steps` of a 32 x 32 thermal e-p plasma (FP64 oracle)."""
    from spectral_rs_b200.config import Params, SpeciesSpec
    from spectral_rs_b200.init import species_arrays
    p = Params(size_x=32, size_y=32, delta=0, dt=0.1, c=c, dens=16, gamma_inj=1.0, n_pass=4, periodic_x=True,
               random_positions=True, seed=3)
    o = orc.OracleSim.from_params(p, dtype=np.float64)
    for k, (q, m) in enumerate(((1.0, 64.0), (-1.0, 1.0))):
        a = species_arrays(p, SpeciesSpec(charge=q, mass=m, vth=0.05, ppc=16, drift_gamma=0.0, x0=0, x1=32),
                           seed_offset=k)
        _add(o, q, m, 0.05, a)
    o.prepare()
    o.step(10)
    e0 = sum(float(np.sum(o.spatial(n)[1:-1, 1:-1] ** 2)) for n in ("Ex", "Ey", "Ez"))
    o.step(steps)
    e1 = sum(float(np.sum(o.spatial(n)[1:-1, 1:-1] ** 2)) for n in ("Ex", "Ey", "Ez"))
    return e1 / e0


def test_courant_stability_boundary():
    """The reference algorithm is stable at c dt = 0.3 (its own config.toml: c = 3,
    dt = 0.1) and blows up at c dt = 0.45 (c = 4.5, dt = 0.1): with omega_pe dt =
    0.1 the highest resolved k of the leapfrog solver leaves the stable region.
    The benchmark workloads therefore use c = 3, dt = 0.1."""
    assert _thermal_energy_growth(3.0, 150) < 10.0
    assert _thermal_energy_growth(4.5, 150) > 1e6


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_periodic_edge_representation(dtype):
    """One particle at rest on the periodic y edge, stored as (iy = 1, dy = -0.5) or as
    (iy = ny, dy = the largest value below 0.5): the same place to within one ulp.  The
    fold (field.rs:260-373) makes the interior deposits equal, but the ghost rows keep
    their raw deposits (the reference never clears them) and the first filter pass
    (field.rs:376-426) reads them as neighbours, so the filtered sources and the next E
    differ by O(1/ppc) at the edge rows.  A 1-ulp difference in a particle's position that
    moves it across the periodic edge therefore changes the reference's own fields near
    that edge at the 1e-3 level of a 64-per-cell plasma; parity tests of long runs bound
    the field error by its RMS and by a max-norm that allows for this."""
    p = test_params(size_x=16, size_y=8, delta=0, c=3.0, dt=0.1, dens=1, periodic_x=True)
    below = np.nextafter(dtype(0.5), dtype(0.0))
    res = []
    for iy, dy in ((1, dtype(-0.5)), (p.size_y, below)):
        o = orc.OracleSim.from_params(p, dtype=dtype)
        z = np.zeros(1, dtype=dtype)
        o.add_species(-1.0, 1.0, 0.0, np.array([5], np.uint64), np.array([iy], np.uint64), z, np.array([dy], dtype),
                      z, z, z, np.ones(1, dtype))
        o.move_and_deposit(0)
        o.fold_sources()
        dens, rho = o.spatial("Dens").astype(np.float64), o.spatial("Rho").astype(np.float64)
        o.fields_update()
        res.append((dens, rho, o.spatial("Ey").astype(np.float64)))
    (d0, r0, e0), (d1, r1, e1) = res
    tol = 1e-12 if dtype == np.float64 else 1e-6
    assert np.max(np.abs(d0[1:-1, 1:-1] - d1[1:-1, 1:-1])) < tol       # folded interior: the same
    assert np.max(np.abs(d0[[0, -1]] - d1[[0, -1]])) > 0.3              # raw ghost rows: not (0.5 x 0.75)
    f0 = orc.field_op(p.size_x, p.size_y, 2, r0, n_pass=1, dtype=dtype).astype(np.float64)
    f1 = orc.field_op(p.size_x, p.size_y, 2, r1, n_pass=1, dtype=dtype).astype(np.float64)
    assert np.max(np.abs(f0[1:-1, 1:-1] - f1[1:-1, 1:-1])) > 0.02      # one filter pass sees the ghosts
    assert np.max(np.abs(e0 - e1)) > 1e-3 * np.max(np.abs(e0))         # and so does E
