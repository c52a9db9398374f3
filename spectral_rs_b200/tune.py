"""Layout autotuner of the split path: tile shapes and sort-bin sizes.

The fused particle kernel works on tiles of TX x TY cells, one CTA per tile and
one thread per cell (TX*TY <= 256 threads).  The best shape depends on the grid,
the particles per cell and how far particles move per step.  ``autotune_tiles``
times the whole step for each candidate on the configuration itself (or on a
crop of it with the same particles per cell and physics), keeps the fastest and
remembers it in a small JSON cache keyed by everything that affects the choice.

The particles of a cell live in sort bins: a low range of KL slots and two
arrival regions of H slots (the cell-slot layout).  KL = headroom x the fullest
cell's count (+ margin), H = the room for one step's arrivals.  Too little room
sends particles to the overflow list (a slower fallback, then a repack); too
much costs device memory and spreads a tile's slots over more pages.
``autotune_layout`` picks the tile shape first, then (headroom, H) with it, and
caches the triple; ``Sim(cfg, tile="auto")`` and ``Batch(cfgs, tile="auto")``
use it.
"""
import math
import dataclasses
import json
import os

CANDIDATES = ((16, 16), (32, 8), (16, 8), (32, 4), (8, 16), (8, 8))
HEADROOMS = (1.25, 2.0, 4.0)          # low range: x the fullest cell's count
ARRIVAL_FRACTIONS = (0.125, 0.25, 0.5)  # arrival regions: x the low range
CACHE = os.path.join(os.path.expanduser("~"), ".cache", "spectral_rs_b200", "tiles.json")
LAYOUT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "spectral_rs_b200", "layout.json")


def tile_key(params, species, crop=None):
    """Cache key: the grid (or crop), the physics and the species' particles per cell and drifts."""
    sx, sy = crop if crop else (params.size_x, params.size_y)
    sp = ";".join(f"{s.charge:g},{s.mass:g},{s.vth:g},{s.ppc},{s.drift_gamma:g}" for s in species)
    return (f"{sx}x{sy}|d{params.delta}|dt{params.dt:g}|c{params.c:g}|n{params.n_pass}|"
            f"px{int(params.periodic_x)}|lw{int(params.left_wall)}|{sp}")


def fits(shape, size_x, size_y):
    tx, ty = shape
    return tx * ty <= 256 and tx <= size_x and ty <= size_y and size_x % tx == 0 and size_y % ty == 0


def measure_step_ms(params, species, shape, steps=4, warmup=2, seed=1, headroom=None, arrival=None):
    """Mean ms per step of the split path with this tile shape (CUDA events of the library);
    headroom / arrival override the sort-bin sizes (slot_headroom, arrival_slots)."""
    from .config import Config, Setup, Output
    from .sim import Sim
    p = dataclasses.replace(params, tile_x=shape[0], tile_y=shape[1], path="split")
    if headroom is not None:
        p = dataclasses.replace(p, slot_headroom=float(headroom), arrival_slots=int(arrival))
    with Sim(Config(p, Setup(0), Output(False, False, 1, 1, 1, 1))) as sim:
        for k, s in enumerate(species):
            x0 = p.delta if s.x0 is None else s.x0
            x1 = p.size_x - p.delta if s.x1 is None else s.x1
            sim.init_species(s.charge, s.mass, s.vth, s.ppc, x0, x1, s.drift_gamma, s.drift_sign, True, seed + k)
        sim.prepare()
        sim.step(warmup)
        sim.set_timing(True)
        sim.step(steps)
        ms = float(sim.timing()[3]) / steps
        sim.set_timing(False)
    return ms


def autotune_tiles(params, species, candidates=CANDIDATES, crop=None, steps=4, cache=CACHE, measure=None):
    """Fastest tile shape (tx, ty) for this configuration.

    params: a ``config.Params``; species: list of ``config.SpeciesSpec``; crop:
    (size_x, size_y) to tune on a smaller grid with the same physics; cache: JSON
    file path or None; measure: replacement of ``measure_step_ms`` (tests).
    Returns ((tx, ty), {shape: ms}) -- the timings are empty on a cache hit.
    """
    measure = measure or measure_step_ms
    key = tile_key(params, species, crop)
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if key in table:
        return tuple(table[key]), {}
    p = dataclasses.replace(params, size_x=crop[0], size_y=crop[1]) if crop else params
    times = {}
    for shape in candidates:
        if fits(shape, p.size_x, p.size_y):
            times[tuple(shape)] = measure(p, species, tuple(shape), steps)
    if not times:
        raise ValueError("no candidate tile shape fits the grid")
    best = min(times, key=times.get)
    if cache:
        table[key] = list(best)
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, cache)
    return best, times


def arrival_slots_for(params, species, headroom, fraction):
    """H for an arrival fraction, sized on the fullest species as the library sizes KL
    (KL = max(headroom x ppc, ppc + 8 sqrt(ppc)) + 8 for a uniform start)."""
    ppc = max(s.ppc for s in species)
    kl = math.ceil(max(headroom * ppc, ppc + 8.0 * math.sqrt(ppc))) + 8
    return max(8, math.ceil(fraction * kl))


def autotune_layout(params, species, crop=None, steps=4, cache=True, tile_cache=True, measure=None,
                    headrooms=HEADROOMS, fractions=ARRIVAL_FRACTIONS):
    """Fastest (tile shape, slot headroom, arrival slots) for this configuration.

    Stage 1 is ``autotune_tiles`` (default sort bins); stage 2 times every
    (headroom, arrival fraction) pair with the chosen tile.  A pair within 1 % of
    the fastest that needs less room wins (smaller headroom, then smaller H).
    measure(p, species, shape, steps, headroom, arrival) replaces the timing (tests).
    cache / tile_cache: a JSON path, True for the module's default path (LAYOUT_CACHE,
    CACHE, read at call time), or None for no cache.
    Returns ({"tile": (tx, ty), "slot_headroom": f, "arrival_slots": h}, {(f, h): ms}).
    """
    cache = LAYOUT_CACHE if cache is True else cache
    tile_cache = CACHE if tile_cache is True else tile_cache
    key = "layout|" + tile_key(params, species, crop)
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if key in table:
        e = table[key]
        return {"tile": tuple(e["tile"]), "slot_headroom": e["slot_headroom"], "arrival_slots": e["arrival_slots"]}, {}
    tmeasure = None if measure is None else (lambda p, sp, shape, n: measure(p, sp, shape, n, None, None))
    tile, _ = autotune_tiles(params, species, crop=crop, steps=steps, cache=tile_cache, measure=tmeasure)
    measure = measure or (lambda p, sp, shape, n, f, h: measure_step_ms(p, sp, shape, n, headroom=f, arrival=h))
    p = dataclasses.replace(params, size_x=crop[0], size_y=crop[1]) if crop else params
    times = {}
    for f in headrooms:
        for fr in fractions:
            h = arrival_slots_for(p, species, f, fr)
            if (f, h) not in times:
                times[(f, h)] = measure(p, species, tile, steps, f, h)
    fastest = min(times.values())
    best = min((k for k, v in times.items() if v <= 1.01 * fastest), key=lambda k: (k[0], k[1]))
    choice = {"tile": tuple(tile), "slot_headroom": best[0], "arrival_slots": best[1]}
    if cache:
        table[key] = {"tile": list(tile), "slot_headroom": best[0], "arrival_slots": best[1]}
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, cache)
    return choice, times
