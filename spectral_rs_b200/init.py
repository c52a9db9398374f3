"""Seeded host-side particle initialisation in the reference's order and FP32 arithmetic.

The reference places particles with ``Prtl::initialize_positions``
(src/prtls.rs:191-221, deterministic diagonal) and draws momenta in
``initialize_velocities`` (src/prtls.rs:222-261) from an *unseeded*
``thread_rng``.  This module restates both with numpy float32 operations in
the same order (numpy applies each float32 operation with one IEEE rounding),
drawing the random numbers from a seeded ``numpy.random.Generator`` so every
path (GPU split, GPU plain, CPU oracle) starts from identical arrays.
"""
import numpy as np

F = np.float32


def positions(size_x, size_y, delta, ppc, x0=None, x1=None, random_positions=False, rng=None):
    """Cell indices (with the +1 ghost offset) and offsets in the reference order:
    rows outer, columns delta..size_x-delta, then the ppc particles of a cell."""
    x0 = delta if x0 is None else x0
    x1 = size_x - delta if x1 is None else x1
    ncols = x1 - x0
    n = size_y * ncols * ppc
    i = np.arange(n, dtype=np.int64)
    k = i % ppc
    cell = i // ppc
    ix = (x0 + cell % ncols + 1).astype(np.uint64)
    iy = (cell // ncols + 1).astype(np.uint64)
    if random_positions:
        dx = (rng.random(n, dtype=np.float32) - F(0.5)).astype(F)
        dy = (rng.random(n, dtype=np.float32) - F(0.5)).astype(F)
    else:
        # src/prtls.rs:209-212: r1 = 1/(2 dens) + k/dens; dx = dy = r1 - 0.5
        r1 = F(1.0) / (F(2.0) * F(ppc))
        r1 = (r1 + k.astype(F) / F(ppc)).astype(F)
        dx = (r1 - F(0.5)).astype(F)
        dy = dx.copy()
    return ix, iy, dx, dy


def draws(n, rng):
    """The random numbers initialize_velocities consumes: 3 standard normals and
    one uniform [0,1) per particle."""
    normals = rng.standard_normal((n, 3), dtype=np.float32)
    uniforms = rng.random(n, dtype=np.float32)
    return normals, uniforms


def velocities(normals, uniforms, c, vth, gamma_inj, sign=1.0):
    """src/prtls.rs:222-250 in float32.  gamma_inj <= 1 means no drift."""
    c = F(c)
    vth = F(vth)
    csqinv = F(1.0) / (c * c)
    px = (normals[:, 0] * (vth * c)).astype(F)
    py = (normals[:, 1] * (vth * c)).astype(F)
    pz = (normals[:, 2] * (vth * c)).astype(F)
    psa = np.sqrt((F(1.0) + (px * px + py * py + pz * pz) * csqinv).astype(F)).astype(F)
    if gamma_inj > 1.0:
        g = F(gamma_inj)
        beta_inj = F(sign) * np.sqrt(F(1.0) - F(1.0) / (g * g)).astype(F)
        ux = (px / c).astype(F)
        flip = (-beta_inj * ux) > (uniforms * psa)
        ux = np.where(flip, ux * F(-1.0), ux).astype(F)
        px = (g * (ux + beta_inj * psa)).astype(F)
        px = (px * c).astype(F)
        psa = np.sqrt((F(1.0) + (px * px + py * py + pz * pz) * csqinv).astype(F)).astype(F)
    return px, py, pz, psa


def species_arrays(params, spec, seed_offset=0):
    """All arrays of one species for ``spx_add_species`` / the oracle."""
    rng = np.random.default_rng([int(params.seed), int(seed_offset)])
    ix, iy, dx, dy = positions(params.size_x, params.size_y, params.delta, spec.ppc, spec.x0, spec.x1,
                               params.random_positions, rng)
    normals, uniforms = draws(len(ix), rng)
    px, py, pz, psa = velocities(normals, uniforms, params.c, spec.vth, spec.drift_gamma, spec.drift_sign)
    return dict(ix=ix, iy=iy, dx=dx, dy=dy, px=px, py=py, pz=pz, psa=psa)
