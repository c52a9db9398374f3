"""The CPU oracle against every known-answer vector of the reference's own tests.

Mirrors the reference's unit tests (same names), with its tolerance E_TOL
(src/lib.rs:28-32: 1e-4 for f32, 1e-13 for f64).  Two of the reference's
comparisons are one-sided (src/flds/fft_2d.rs:904-905, 949-950); here every
comparison is two-sided.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from conftest import cplx

E_TOL = {np.float32: 1e-4, np.float64: 1e-13}
DTYPES = [np.float32, np.float64]


@pytest.mark.parametrize("dt", DTYPES)
def test_copy_to_spectral(golden, dt):  # src/flds/field.rs:486-570
    g = golden["copy_to_spectral"]
    out = orc.copy_to_spectral(24, 12, np.array(g["input"]), dtype=dt)
    exp = np.array(g["expected"], dtype=dt)
    assert np.array_equal(out.real, exp)
    assert np.all(out.imag == 0)


@pytest.mark.parametrize("dt", DTYPES)
def test_copy_to_spatial(golden, dt):  # src/flds/field.rs:572-655
    g = golden["copy_to_spatial"]
    out = orc.copy_to_spatial(24, 12, np.array(g["input"]).astype(dt), dtype=dt)
    assert np.array_equal(out, np.array(g["expected"], dtype=dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_ghost_deposit(golden, dt):  # src/flds/field.rs:656-723
    g = golden["ghost_deposit"]
    out = orc.field_op(24, 12, 0, np.array(g["input"]), dtype=dt)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL[dt]


@pytest.mark.parametrize("dt", DTYPES)
def test_ghosts_update(golden, dt):  # src/flds/field.rs:725-795: deposit_ghosts then update_ghosts
    g = golden["ghosts_update"]
    a = orc.field_op(24, 12, 0, np.array(g["input"]), dtype=dt)
    out = orc.field_op(24, 12, 1, a, dtype=dt)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL[dt]


@pytest.mark.parametrize("dt", DTYPES)
def test_binomial_filter(golden, dt):  # src/flds/field.rs:797-1543, 4 passes
    g = golden["binomial_filter"]
    out = orc.field_op(24, 12, 2, np.array(g["input"]), n_pass=g["n_pass"], dtype=dt)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL[dt]


@pytest.mark.parametrize("dt", DTYPES)
def test_forward_fft(golden, dt):  # src/flds/fft_2d.rs:478-547
    g = golden["forward_fft"]
    out = orc.fft1d(cplx(g["input"]), dtype=dt)
    exp = cplx(g["expected"])
    assert np.max(np.abs(out.real - exp.real)) < E_TOL[dt]
    assert np.max(np.abs(out.imag - exp.imag)) < E_TOL[dt]


@pytest.mark.parametrize("dt", DTYPES)
def test_fft_1d_roundtrip(golden, dt):  # src/flds/fft_2d.rs:549-600 (unnormalized inverse)
    x = cplx(golden["fft_1d_roundtrip"]["input"])
    y = orc.fft1d(orc.fft1d(x, dtype=dt), inverse=True, dtype=dt)
    n = len(x)
    assert np.max(np.abs(y.real - x.real * n)) < E_TOL[dt] * n
    assert np.max(np.abs(y.imag - x.imag * n)) < E_TOL[dt] * n


@pytest.mark.parametrize("dt", DTYPES)
def test_forward_fft2d(golden, dt):  # src/flds/fft_2d.rs:601-907, two-sided here
    x = cplx(golden["fft2d_input"]).reshape(12, 24)
    exp = cplx(golden["forward_fft2d"]["expected"]).reshape(12, 24)
    out = orc.fft2d(x, dtype=dt)
    tol = E_TOL[dt] * (10 if dt == np.float32 else 1)  # |X| ~ 150: f32 rounding ~1.5e-5 * log2 N
    assert np.max(np.abs(out.real - exp.real)) < tol
    assert np.max(np.abs(out.imag - exp.imag)) < tol


@pytest.mark.parametrize("dt", DTYPES)
def test_fft_2d_roundtrip(golden, dt):  # src/flds/fft_2d.rs:929-952, normalized inverse, two-sided
    x = cplx(golden["fft2d_input"]).reshape(12, 24)
    y = orc.fft2d(orc.fft2d(x, dtype=dt), inverse=True, dtype=dt)
    assert np.max(np.abs(y - x)) < E_TOL[dt]
    assert not np.array_equal(orc.fft2d(x, dtype=dt), x.astype(y.dtype))


def test_transpose_convention(golden):  # src/flds/fft_2d.rs:909-927: the row-major (ky, kx) layout
    x = cplx(golden["fft2d_input"]).reshape(12, 24)
    np.testing.assert_allclose(orc.fft2d(x), np.fft.fft2(x), atol=1e-12)


@pytest.mark.parametrize("dt", DTYPES)
def test_wave_nums_init(golden, dt):  # src/flds/wave_num.rs:49-943
    kx, ky, kn = orc.wave_numbers(24, 12, dtype=dt)
    g = golden["wave_nums_init"]
    # the reference compares against values made in double precision
    tol = 1e-4 if dt == np.float32 else 1e-13
    for a, k in ((kx, "k_x"), (ky, "k_y"), (kn, "k_norm")):
        e = np.array(g[k])
        assert np.max(np.abs(a - e)) < tol * max(1.0, np.max(np.abs(e))), k


def test_sim_init(golden):  # src/lib.rs:495-500
    ts = golden["test_sim"]
    s = orc.OracleSim(ts["size_x"], ts["size_y"], ts["delta"], ts["dt"], ts["c"], ts["dens"], ts["gamma_inj"],
                      ts["n_pass"], False)
    assert (s.size_x, s.size_y) == (24, 12)


@pytest.mark.parametrize("dt", DTYPES)
def test_flds_init(dt):  # src/flds/mod.rs:316-340: every field zero, (ny+2) x (nx+2)
    s = orc.OracleSim(24, 12, 5, 0.1, 3.0, 2, 5.0, 4, False, dtype=dt)
    for name in orc.FIELD_IDS:
        f = s.spatial(name)
        assert f.shape == (14, 26)
        assert not f.any()
    for comp in range(3):
        assert s.b_wrk(comp).shape == (12, 24) and not s.b_wrk(comp).any()
