"""Host mirror of the reference's hot-path API over the C ABI.

The reference's types and call sequence (src/lib.rs, src/prtls.rs, src/flds)
map onto this module as follows:

  Sim::new (src/lib.rs:247-264)                  -> Sim(cfg)
  Prtl::new (src/prtls.rs:60-84)                 -> Sim.add_species / Prtl
  Flds::new (src/flds/mod.rs:40-65)              -> created with the Sim (device resident)
  Sim::move_and_deposit (src/lib.rs:478-489)     -> Sim.move_and_deposit(prtl)
  Field::deposit_ghosts (src/flds/field.rs:260)  -> Flds.deposit_ghosts(name)
  Flds::update (src/flds/mod.rs:87-309)          -> Flds.update(sim)
  Prtl::boris_push (src/prtls.rs:262-443)        -> Prtl.boris_push(sim, flds)
  run (src/lib.rs:119-202)                       -> run(cfg)

All state lives in device memory; getters copy back in the reference layout.
"""
import ctypes
import sys

import numpy as np

from . import _lib
from .config import Config
from .init import species_arrays


def device_index():
    """The CUDA device new contexts are created on: PyTorch's current device when the caller
    has loaded torch (one process per GPU under torchrun sets it from LOCAL_RANK), else 0.
    The library keeps its own CUDA runtime state, so the index is passed to it explicitly."""
    torch = sys.modules.get("torch")
    try:
        if torch is not None and torch.cuda.is_available():
            return int(torch.cuda.current_device())
    except Exception:
        pass
    return 0


def _layout_choice(cfg, tile):
    """(tile_x, tile_y, slot_headroom, arrival_slots) for spx_params: an explicit tile shape,
    "auto" (tile shape and sort bins from spectral_rs_b200.tune), or the config's (0 = library rule)."""
    p = cfg.params
    if tile is None:
        return p.tile_x, p.tile_y, p.slot_headroom, p.arrival_slots
    if tile == "auto":
        from .tune import autotune_layout
        crop = (min(p.size_x, 1024), min(p.size_y, 256)) if p.periodic_x else None
        c = autotune_layout(p, cfg.species_list(), crop=crop)[0]
        return c["tile"][0], c["tile"][1], c["slot_headroom"], c["arrival_slots"]
    return int(tile[0]), int(tile[1]), p.slot_headroom, p.arrival_slots


class Sim:
    """Owns one device context (``spx_ctx``)."""

    def __init__(self, cfg: Config, path=None, tile=None):
        """path: "split" / "plain" overrides the config; tile: (tx, ty), or "auto" for the
        autotuner (spectral_rs_b200.tune), or None for the config's / the library's choice."""
        self.lib = _lib.load()
        self.config = cfg
        p = cfg.params
        tx, ty, headroom, arrival = _layout_choice(cfg, tile)
        self.t = 0
        self.t_final = cfg.setup.t_final
        self.size_x, self.size_y, self.delta = p.size_x, p.size_y, p.delta
        self.dt, self.c, self.dens = p.dt, p.c, p.dens
        self.gamma_inj, self.n_pass = p.gamma_inj, p.n_pass
        self.prtl_num = p.dens * (p.size_x - 2 * p.delta) * p.size_y  # src/lib.rs:258-260
        prm = _lib.SpxParams(
            size_x=p.size_x, size_y=p.size_y, delta=p.delta, dt=p.dt, c=p.c, dens=p.dens,
            gamma_inj=p.gamma_inj, n_pass=p.n_pass, periodic_x=1 if p.periodic_x else 0,
            left_wall=1 if p.left_wall else 0,
            path=_lib.PATH_PLAIN if (path or p.path) == "plain" else _lib.PATH_SPLIT,
            tile_x=tx, tile_y=ty, slot_capacity=p.slot_capacity, device=device_index(),
            compensated=1 if p.compensated else 0, slot_headroom=headroom, arrival_slots=arrival)
        self.layout = {"tile": (tx, ty), "slot_headroom": headroom, "arrival_slots": arrival}
        self._ctx = ctypes.c_void_p()
        _lib.check(self.lib.spx_create(ctypes.byref(prm), ctypes.byref(self._ctx)))
        self.flds = Flds(self)
        self.prtls = []

    # -- lifecycle -------------------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.spx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, code):
        return _lib.check(code, self._ctx)

    # -- species ---------------------------------------------------------------------
    def add_species(self, charge, mass, vth, ix, iy, dx, dy, px, py, pz, psa=None):
        """Prtl::new with caller-supplied state (arrays in the reference's order)."""
        n = len(ix)
        arrs = [np.ascontiguousarray(ix, dtype=np.uint64), np.ascontiguousarray(iy, dtype=np.uint64)]
        arrs += [np.ascontiguousarray(a, dtype=np.float32) for a in (dx, dy, px, py, pz)]
        ps = None if psa is None else np.ascontiguousarray(psa, dtype=np.float32)
        sid = ctypes.c_int32(-1)
        self._chk(self.lib.spx_add_species(self._ctx, charge, mass, vth, n, *[_lib.ptr(a) for a in arrs],
                                           _lib.ptr(ps), ctypes.byref(sid)))
        pr = Prtl(self, sid.value, charge, mass, vth)
        self.prtls.append(pr)
        return pr

    def init_species(self, charge, mass, vth, ppc, x0, x1, gamma_drift=0.0, sign_x=1.0,
                     random_positions=True, seed=0):
        """Seeded on-device initialisation (no host arrays)."""
        sid = ctypes.c_int32(-1)
        self._chk(self.lib.spx_init_species(self._ctx, charge, mass, vth, ppc, x0, x1, gamma_drift, sign_x,
                                            1 if random_positions else 0, seed, ctypes.byref(sid)))
        pr = Prtl(self, sid.value, charge, mass, vth)
        self.prtls.append(pr)
        return pr

    def init_from_config(self):
        """The species of run() (src/lib.rs:121-126), from host arrays drawn with the config's seed."""
        for k, spec in enumerate(self.config.species_list()):
            a = species_arrays(self.config.params, spec, seed_offset=k)
            self.add_species(spec.charge, spec.mass, spec.vth, a["ix"], a["iy"], a["dx"], a["dy"],
                             a["px"], a["py"], a["pz"], a["psa"])
        return self.prtls

    # -- the hot path -------------------------------------------------------------------
    def move_and_deposit(self, prtl):
        self._chk(self.lib.spx_move_and_deposit(self._ctx, prtl.sid))

    def zero_sources(self):
        self._chk(self.lib.spx_zero_sources(self._ctx))

    def prepare(self):
        """The extra move+deposit and ghost fold before the loop (src/lib.rs:130-142)."""
        self._chk(self.lib.spx_prepare(self._ctx))

    def step(self, n=1):
        """n iterations of run()'s loop body without output (fused, graph-captured)."""
        self._chk(self.lib.spx_step(self._ctx, n))
        self.t += n

    def flush(self):
        self._chk(self.lib.spx_flush(self._ctx))

    def synchronize(self):
        self._chk(self.lib.spx_synchronize(self._ctx))

    def diag(self):
        """FP64 device diagnostics: (E energy, B energy, kinetic energy, net charge, particles)."""
        out = np.zeros(5, dtype=np.float64)
        self._chk(self.lib.spx_diag(self._ctx, _lib.ptr(out)))
        return out

    def set_timing(self, on=True):
        self._chk(self.lib.spx_set_timing(self._ctx, 1 if on else 0))

    def timing(self):
        out = np.zeros(4, dtype=np.float32)
        self._chk(self.lib.spx_get_timing(self._ctx, _lib.ptr(out)))
        return out

    def last_launch_count(self):
        return int(self.lib.spx_last_launch_count(self._ctx))

    def counters(self):
        """dict of slot-layout counters (repacks, overflow, occupancy, K, tiles, launches, device memory
        in use: total - free, every context on the device)."""
        out = np.zeros(8, dtype=np.uint64)
        self._chk(self.lib.spx_get_counters(self._ctx, _lib.ptr(out)))
        keys = ("repacks", "overflow", "max_occupancy", "slot_capacity", "tiles", "cells_per_tile",
                "launches", "device_bytes")
        return {k: int(v) for k, v in zip(keys, out)}

    def stream(self):
        """The context's cudaStream_t as an integer handle (torch.cuda.ExternalStream accepts it)."""
        return int(self.lib.spx_get_stream(self._ctx) or 0)


class Flds:
    """Device-resident fields with the reference's names (src/flds/mod.rs:15-37)."""

    NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz", "Rho", "Dens")

    def __init__(self, sim):
        self.sim = sim

    def spatial(self, name, with_ghosts=True, out=None):
        """Field `name` as a float32 (rows, cols) array, into `out` when given
        (C-contiguous float32 of that shape, e.g. a reused or page-locked buffer)."""
        s = self.sim
        shape = (s.size_y + 2, s.size_x + 2) if with_ghosts else (s.size_y, s.size_x)
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {shape}")
        s._chk(s.lib.spx_get_field(s._ctx, _lib.FIELD_IDS[name], 1 if with_ghosts else 0, _lib.ptr(out)))
        return out

    def set_spatial(self, name, arr):
        s = self.sim
        a = np.ascontiguousarray(arr, dtype=np.float32)
        assert a.size == (s.size_y + 2) * (s.size_x + 2)
        s._chk(s.lib.spx_set_field(s._ctx, _lib.FIELD_IDS[name], _lib.ptr(a)))

    def b_wrk(self, comp):
        s = self.sim
        out = np.empty((s.size_y, s.size_x), dtype=np.complex64)
        s._chk(s.lib.spx_get_bwrk(s._ctx, comp, _lib.ptr(out)))
        return out

    def set_b_wrk(self, comp, arr):
        s = self.sim
        a = np.ascontiguousarray(arr, dtype=np.complex64)
        s._chk(s.lib.spx_set_bwrk(s._ctx, comp, _lib.ptr(a)))

    def deposit_ghosts(self, name):
        s = self.sim
        s._chk(s.lib.spx_deposit_ghosts(s._ctx, _lib.FIELD_IDS[name]))

    def update(self, sim=None):
        s = self.sim
        s._chk(s.lib.spx_fields_update(s._ctx))


class Prtl:
    """Handle on one device-resident species (src/prtls.rs:8-23)."""

    def __init__(self, sim, sid, charge, mass, vth):
        self.sim, self.sid = sim, sid
        self.charge, self.mass, self.vth = charge, mass, vth
        f = np.float32
        self.beta = (f(charge) / f(mass)) * f(0.5) * f(sim.dt)           # src/prtls.rs:61
        self.alpha = (f(charge) / f(mass)) * f(0.5) * f(sim.dt) / f(sim.c)  # src/prtls.rs:62

    def __len__(self):
        return int(self.sim.lib.spx_species_count(self.sim._ctx, self.sid))

    def state(self, stride=1):
        """dict of ix, iy (uint64), dx, dy, px, py, pz, psa (float32) in the reference order."""
        s = self.sim
        n = len(self)
        m = (n + stride - 1) // stride
        out = {k: np.empty(m, dtype=np.uint64) for k in ("ix", "iy")}
        out.update({k: np.empty(m, dtype=np.float32) for k in ("dx", "dy", "px", "py", "pz", "psa")})
        s._chk(s.lib.spx_get_species(s._ctx, self.sid, stride, *[_lib.ptr(out[k]) for k in
                                                                 ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa")]))
        return out

    def set_tags(self, tag=None, track=None):
        """Prtl::tag / Prtl::track (src/prtls.rs:21-22) in the reference's order (None keeps a table)."""
        s = self.sim
        t = None if tag is None else np.ascontiguousarray(tag, dtype=np.uint64)
        k = None if track is None else np.ascontiguousarray(track, dtype=np.uint8)
        for a in (t, k):
            if a is not None and len(a) != len(self):
                raise ValueError("one entry per particle")
        s._chk(s.lib.spx_set_tags(s._ctx, self.sid, _lib.ptr(t), _lib.ptr(k)))

    def tags(self, stride=1):
        """(tag uint64, track bool) every stride-th particle in the reference's order."""
        s = self.sim
        m = (len(self) + stride - 1) // stride
        t, k = np.empty(m, dtype=np.uint64), np.empty(m, dtype=np.uint8)
        s._chk(s.lib.spx_get_tags(s._ctx, self.sid, stride, _lib.ptr(t), _lib.ptr(k)))
        return t, k.astype(bool)

    def tracked(self):
        """The tracking output of save_output (src/save/mod.rs:82-97): x, y (in units of c) and
        gamma of the tracked particles, reference order, gathered on the device."""
        s = self.sim
        cnt = ctypes.c_uint64(0)
        s._chk(s.lib.spx_get_tracked(s._ctx, self.sid, 0, None, None, None, ctypes.byref(cnt)))  # count only
        k = int(cnt.value)
        x, y, g = (np.empty(k, dtype=np.float32) for _ in range(3))
        s._chk(s.lib.spx_get_tracked(s._ctx, self.sid, k, _lib.ptr(x), _lib.ptr(y), _lib.ptr(g), ctypes.byref(cnt)))
        return x, y, g

    def boris_push(self, sim=None, flds=None):
        self.sim._chk(self.sim.lib.spx_boris_push(self.sim._ctx, self.sid))


def run(cfg: Config, out_dir="output", on_step=None):
    """run (src/lib.rs:119-202): init, pre-loop move+deposit, then t_final+1
    iterations; save_output at every output_interval when write_output is set.
    The fused device step is used between saves."""
    from .save import save_output
    with Sim(cfg) as sim:
        sim.init_from_config()
        sim.prepare()
        t = 0
        while t <= sim.t_final:
            if cfg.output.write_output and t % cfg.output.output_interval == 0:
                save_output(t, sim, out_dir)
            # run until the next save step (or the end) in one fused call
            nxt = sim.t_final + 1
            if cfg.output.write_output:
                nxt = min(nxt, (t // cfg.output.output_interval + 1) * cfg.output.output_interval)
            sim.step(nxt - t)
            if on_step:
                on_step(sim, nxt - 1)
            t = nxt
        sim.flush()
        return sim.diag()


class _BorrowedSim(Sim):
    """A simulation owned by a Batch: same accessors as Sim, no ownership of the context."""

    def __init__(self, batch, index, cfg, ctx):
        self.lib = _lib.load()
        self.config = cfg
        p = cfg.params
        self.t = 0
        self.t_final = cfg.setup.t_final
        self.size_x, self.size_y, self.delta = p.size_x, p.size_y, p.delta
        self.dt, self.c, self.dens = p.dt, p.c, p.dens
        self.gamma_inj, self.n_pass = p.gamma_inj, p.n_pass
        self.prtl_num = p.dens * (p.size_x - 2 * p.delta) * p.size_y
        self._ctx = ctypes.c_void_p(ctx)
        self.flds = Flds(self)
        self.prtls = []
        self.batch, self.index = batch, index

    def close(self):  # the batch owns the context
        self._ctx = ctypes.c_void_p()


class Batch:
    """Independent simulations advanced together (spx_batch_*): one persistent
    particle launch over all (simulation, tile) items and one CUDA graph per step."""

    def __init__(self, cfgs, tile=None):
        """tile: (tx, ty) for every member, "auto" (tuned on the member with the most
        particles), or None (the configs' / the library's choice)."""
        self.lib = _lib.load()
        prms = (_lib.SpxParams * len(cfgs))()
        shape = None
        if tile is not None:  # tuned on the member with the most particles, used by all
            big = max(cfgs, key=lambda c: sum(s.ppc for s in c.species_list()) * c.params.size_x * c.params.size_y)
            shape = _layout_choice(big, tile)
        for i, cfg in enumerate(cfgs):
            p = cfg.params
            tx, ty, headroom, arrival = shape if shape else (p.tile_x, p.tile_y, p.slot_headroom, p.arrival_slots)
            prms[i] = _lib.SpxParams(
                size_x=p.size_x, size_y=p.size_y, delta=p.delta, dt=p.dt, c=p.c, dens=p.dens,
                gamma_inj=p.gamma_inj, n_pass=p.n_pass, periodic_x=1 if p.periodic_x else 0,
                left_wall=1 if p.left_wall else 0, path=_lib.PATH_SPLIT, tile_x=tx, tile_y=ty,
                slot_capacity=p.slot_capacity, device=device_index(), slot_headroom=headroom, arrival_slots=arrival)
        self._b = ctypes.c_void_p()
        code = self.lib.spx_batch_create(len(cfgs), prms, ctypes.byref(self._b))
        if code:
            raise _lib.SpxError(code, self.lib.spx_batch_last_error(None).decode())
        self.sims = [_BorrowedSim(self, i, cfg, self.lib.spx_batch_sim(self._b, i)) for i, cfg in enumerate(cfgs)]

    def _chk(self, code):
        if code:
            raise _lib.SpxError(code, self.lib.spx_batch_last_error(self._b).decode())

    def prepare(self):
        self._chk(self.lib.spx_batch_prepare(self._b))

    def step(self, n=1):
        self._chk(self.lib.spx_batch_step(self._b, n))
        for s in self.sims:
            s.t += n

    def set_timing(self, on=True):
        self._chk(self.lib.spx_batch_set_timing(self._b, 1 if on else 0))

    def timing(self):
        out = np.zeros(2, dtype=np.float32)
        self._chk(self.lib.spx_batch_get_timing(self._b, _lib.ptr(out)))
        return out

    def get_field(self, name, with_ghosts=True, out=None):
        """Field `name` of every member (spx_batch_get_field): a list of float32 (rows, cols)
        arrays, into `out` when given (one C-contiguous float32 array per member, e.g.
        page-locked buffers)."""
        shapes = [((s.size_y + 2, s.size_x + 2) if with_ghosts else (s.size_y, s.size_x)) for s in self.sims]
        if out is None:
            out = [np.empty(sh, dtype=np.float32) for sh in shapes]
        if len(out) != len(shapes):
            raise ValueError(f"out must hold {len(shapes)} arrays")
        for o, sh in zip(out, shapes):
            if o.shape != sh or o.dtype != np.float32 or not o.flags["C_CONTIGUOUS"]:
                raise ValueError(f"each out array must be C-contiguous float32 of its member's shape {sh}")
        ptrs = (ctypes.c_void_p * len(out))(*[o.ctypes.data for o in out])
        self._chk(self.lib.spx_batch_get_field(self._b, _lib.FIELD_IDS[name], 1 if with_ghosts else 0, ptrs))
        return out

    def stream(self):
        return int(self.lib.spx_batch_get_stream(self._b) or 0)

    def last_launch_count(self):
        return int(self.lib.spx_batch_last_launch_count(self._b))

    def close(self):
        if self._b:
            for s in self.sims:
                s.close()
            self.lib.spx_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
