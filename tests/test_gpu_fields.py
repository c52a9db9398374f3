"""GPU field solver against the CPU oracle and the reference's golden vectors."""
import numpy as np
import pytest

from oracle import oracle as orc
from conftest import cplx

pytestmark = pytest.mark.gpu

E_TOL = 1e-4  # src/lib.rs:32 (f32)


def _lib():
    from spectral_rs_b200 import _lib
    return _lib


def test_gpu_ghost_deposit(golden):  # src/flds/field.rs:656-723; bit-exact with the f32 oracle
    g = golden["ghost_deposit"]
    x = np.array(g["input"], dtype=np.float32)
    out = _lib().field_op(24, 12, 0, x)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL
    assert np.array_equal(out, orc.field_op(24, 12, 0, x, dtype=np.float32))


def test_gpu_ghosts_update(golden):  # src/flds/field.rs:725-795
    g = golden["ghosts_update"]
    a = _lib().field_op(24, 12, 0, np.array(g["input"], dtype=np.float32))
    out = _lib().field_op(24, 12, 1, a)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL


def test_gpu_binomial_filter(golden):  # src/flds/field.rs:797-1543
    g = golden["binomial_filter"]
    x = np.array(g["input"], dtype=np.float32)
    out = _lib().field_op(24, 12, 2, x, n_pass=4)
    assert np.max(np.abs(out - np.array(g["expected"]))) < E_TOL
    assert np.array_equal(out, orc.field_op(24, 12, 2, x, n_pass=4, dtype=np.float32))


@pytest.mark.parametrize("nx,ny", [(32, 16), (64, 8), (512, 64)])
def test_gpu_filter_raw_ghosts_bit_exact(nx, ny):
    # first pass reads the deposited (non-periodic) ghost frame, as the reference does
    rng = np.random.default_rng(7)
    x = rng.standard_normal((ny + 2) * (nx + 2)).astype(np.float32)
    for npass in (1, 2, 3):
        assert np.array_equal(_lib().field_op(nx, ny, 2, x, n_pass=npass),
                              orc.field_op(nx, ny, 2, x, n_pass=npass, dtype=np.float32))
    assert np.array_equal(_lib().field_op(nx, ny, 0, x), orc.field_op(nx, ny, 0, x, dtype=np.float32))


@pytest.mark.parametrize("nx,ny", [(24, 12), (8, 8), (64, 16), (200, 40), (512, 64), (4096, 32), (1024, 256)])
def test_gpu_fused_filter_bit_exact(nx, ny):
    # all passes in one kernel (the Flds::update path): identical to the passes one by one,
    # the first one reading the raw ghost frame; tiles inside the grid and tiles at its edges
    rng = np.random.default_rng(nx + 13 * ny)
    x = rng.standard_normal((ny + 2) * (nx + 2)).astype(np.float32)
    for npass in (1, 2, 4, 8, 16):
        assert np.array_equal(_lib().field_op(nx, ny, 3, x, n_pass=npass),
                              orc.field_op(nx, ny, 2, x, n_pass=npass, dtype=np.float32)), npass


# every compiled transform length (2^6 .. 2^13) as rows and as columns, and the generic shorter ones
@pytest.mark.parametrize("nx,ny", [(8, 8), (16, 32), (64, 8), (512, 64), (128, 1024), (2048, 16), (8192, 8),
                                   (16, 2048), (256, 4096), (4096, 128), (1024, 512), (32, 8192), (64, 256)])
def test_gpu_fft2d_vs_numpy(nx, ny):
    rng = np.random.default_rng(nx * 7 + ny)
    x = (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))).astype(np.complex64)
    ref = np.fft.fft2(x.astype(np.complex128))
    out = _lib().fft2d(x)
    rel = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    assert rel < 2e-6 * np.log2(nx * ny)
    back = _lib().fft2d(out, inverse=True)
    assert np.max(np.abs(back - x)) < 1e-5 * np.log2(nx * ny)


def test_gpu_fft2d_golden(golden):  # the reference's 2-D vector on a power-of-two crop is not available;
    # pin the convention with the numpy-generated forward_fft2d data instead: zero-pad to 32 x 16
    x = cplx(golden["fft2d_input"]).reshape(12, 24)
    pad = np.zeros((16, 32), dtype=np.complex64)
    pad[:12, :24] = x
    np.testing.assert_allclose(_lib().fft2d(pad), np.fft.fft2(pad.astype(np.complex128)), atol=2e-4)


def _field_state(nx, ny, seed):
    """Random sources, E and B(t-1/2) consistent with real fields, as the solver sees them."""
    rng = np.random.default_rng(seed)
    W = nx + 2
    st = {}
    for name in ("Jx", "Jy", "Jz", "Rho", "Ex", "Ey", "Ez"):
        st[name] = rng.standard_normal((ny + 2, W)).astype(np.float32) * (0.1 if name[0] == "J" else 1.0)
    bw = []
    for _ in range(3):
        b = rng.standard_normal((ny, nx))
        k = np.fft.fft2(b)
        k[:, nx // 2] = 0
        k[ny // 2, :] = 0
        bw.append(k.astype(np.complex64))
    return st, bw


# includes the benchmark's row length (4096) and column lengths (1024, 2048), the 8192-point
# rows and columns, the shortest rows (8 points: a half spectrum of 4 columns) and every column
# length from 16 to 8192
@pytest.mark.parametrize("nx,ny,n_pass", [(64, 32, 4), (128, 64, 1), (512, 64, 4), (4096, 64, 4), (1024, 256, 2),
                                          (8192, 16, 8), (64, 1024, 4), (32, 2048, 8), (16, 4096, 4),
                                          (16, 8192, 4), (8, 128, 4), (256, 512, 4)])
def test_gpu_fields_update_vs_oracle(nx, ny, n_pass):
    """Flds::update on identical inputs: E, B, filtered J and B_wrk against the FP64 oracle."""
    from spectral_rs_b200 import Sim
    from conftest import test_params
    p = test_params(size_x=nx, size_y=ny, delta=4, dt=0.1, c=4.5, dens=8, n_pass=n_pass, periodic_x=True)
    from spectral_rs_b200.config import Config, Setup, Output
    cfg = Config(p, Setup(1), Output(False, False, 1, 1, 1, 1))
    st, bw = _field_state(nx, ny, seed=nx + ny)
    with Sim(cfg) as sim:
        o64 = orc.OracleSim.from_params(p, dtype=np.float64)
        o32 = orc.OracleSim.from_params(p, dtype=np.float32)
        for name, arr in st.items():
            sim.flds.set_spatial(name, arr)
            o64.set_spatial(name, arr.astype(np.float64))
            o32.set_spatial(name, arr)
        for c in range(3):
            sim.flds.set_b_wrk(c, bw[c])
            o64.set_b_wrk(c, bw[c].astype(np.complex128))
            o32.set_b_wrk(c, bw[c])
        sim.flds.update()
        o64.fields_update()
        o32.fields_update()
        for name in ("Jx", "Jy", "Jz", "Rho"):  # filtered sources: bit-exact with the f32 oracle
            assert np.array_equal(sim.flds.spatial(name), o32.spatial(name)), name
        for name in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            g, r = sim.flds.spatial(name), o64.spatial(name)
            rel = np.max(np.abs(g - r)) / max(np.max(np.abs(r)), 1e-30)
            assert rel < 1e-5, (name, rel)
            # the ghost frame is the periodic image
            assert np.array_equal(g[0, 1:-1], g[ny, 1:-1]) and np.array_equal(g[1:-1, 0], g[1:-1, nx])
        for c in range(3):
            g, r = sim.flds.b_wrk(c), o64.b_wrk(c)
            rel = np.max(np.abs(g - r)) / max(np.max(np.abs(r)), 1e-30)
            assert rel < 1e-5, ("bwrk", c, rel)


@pytest.mark.parametrize("nx,ny", [(64, 32), (8, 16), (256, 128)])
def test_gpu_bwrk_half_spectrum(nx, ny):
    """B_wrk lives on the device as the kx < nx/2 half of a Hermitian spectrum: set keeps that
    half bit for bit, get completes the rest by the conjugate mirror with column nx/2 zero, and
    after field updates the array a caller reads is still the spectrum of a real field."""
    from spectral_rs_b200 import Sim
    from conftest import test_params
    from spectral_rs_b200.config import Config, Setup, Output
    p = test_params(size_x=nx, size_y=ny, delta=4, dt=0.1, c=3.0, dens=8, n_pass=4, periodic_x=True)
    cfg = Config(p, Setup(1), Output(False, False, 1, 1, 1, 1))
    st, bw = _field_state(nx, ny, seed=7 * nx + ny)
    H = nx // 2
    with Sim(cfg) as sim:
        for c in range(3):
            sim.flds.set_b_wrk(c, bw[c])
            got = sim.flds.b_wrk(c)
            assert np.array_equal(got[:, :H], bw[c][:, :H])
            assert not np.any(got[:, H])
            mirror = np.conj(got[(-np.arange(ny)) % ny][:, (nx - np.arange(H + 1, nx))])
            assert np.array_equal(got[:, H + 1:], mirror)
        for name, arr in st.items():
            sim.flds.set_spatial(name, arr)
        for _ in range(2):
            sim.flds.update()
        for c in range(3):
            got = sim.flds.b_wrk(c).astype(np.complex128)
            assert not np.any(got[:, H]) and not np.any(got[ny // 2])
            # column kx = 0 and row ky = 0 are their own mirrors, held to FP32 rounding only
            spatial = np.fft.ifft2(got)
            assert np.max(np.abs(spatial.imag)) <= 1e-5 * max(np.max(np.abs(spatial.real)), 1e-30)
