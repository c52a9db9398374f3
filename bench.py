#!/usr/bin/env python
"""Benchmark of the spectral_rs per-timestep hot path on B200.

Metric: particle-steps/s (particles x steps / device time of the timed steps)
and the HBM roofline fraction of the fused push + move + deposit kernel, for
the batched split-position FP32 path against the plain FP32 path.

Default workload (one GPU): the batched uneven ensemble -- 64 independent
shock simulations (reflecting wall, mirror wall on the left) advanced together:
one persistent particle launch over a work queue of (simulation, tile) items
and one CUDA graph per step.  Grids from {128x128, 256x128, 512x256, 1024x256},
4-32 particles per cell per species, mass ratio in {1, 16, 64}, upstream drift
uniform in [0.05c, 0.3c], thermal spread 0.1c, seed 4242 (265,764,864
particles), c = 3.0, dt = 0.1 (Courant number 0.3; the reference algorithm is
numerically unstable for these plasmas at 0.45), 4 filter passes.  Synthetic
data from the build's own seeded generator; a "step" is one iteration of the
reference's loop for every member (zero sources, move + deposit, ghost fold,
Flds::update, Boris push).  The particle state (several GB) exceeds the 126 MB
L2, so no flush is needed between steps.

The line carries:
  value        device-resident, production launch path (one graph per step)
  roofline     the batch particle kernel: 48 B x particles + 44 B x member cells
               per launch / its CUDA-event time (a separate event-timed run)
  plain_fp32   the plain single-simulation FP32 GPU path on the same members
  cpu_baseline the C++ restatement of the reference CPU path (oracle/) on a
               sample of the members (all host threads)
  e2e          the same metric through the public API from pinned host buffers
  thermal_c2   the 4096 x 1024 thermal e-p plasma (536,870,912 particles)
  weibel_c5    the 8192 x 2048 Weibel pair plasma (1,073,741,824 particles)
  clocks       SM clocks sampled during the timed region

--workload thermal|shock|weibel runs one simulation instead (same keys).
--impl reference times the reference's CPU path (the oracle restatement; the
Rust crate cannot be built here) on all host cores, same metric and workload,
each step one step of a bounded sample of it.

Multi-GPU (torchrun): members are independent units with no exchange step.
N ranks run an ensemble of 64 N members, rank r the contiguous block of 64
starting at 64 r (the N = 1 workload is rank 0's block): every member runs on
exactly one rank, the work per GPU is fixed (weak scaling), no collective is on
the data path; the time is the max over ranks.  Single-simulation workloads run
independent replicas.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def _sp(q, m, vth, ppc, gamma=0.0, sign=1.0):
    return dict(q=q, m=m, vth=vth, ppc=ppc, gamma=gamma, sign=sign)


# Single-simulation workloads (species: ions first, as run() creates them, src/lib.rs:124-126).
WORKLOADS = {
    # the plain method at scale
    "thermal": dict(name="thermal_ep_4096x1024_ppc64", size_x=4096, size_y=1024, delta=0, dt=0.1, c=3.0, dens=64,
                    n_pass=4, periodic_x=True, left_wall=False,
                    species=[_sp(1.0, 64.0, 0.05, 64), _sp(-1.0, 1.0, 0.05, 64)],
                    small=(1024, 256), crop=(512, 256)),
    # small unmagnetized shock: drift 0.1c toward the reflecting wall (the
    # reference's wall is on the right), mirror wall on the left
    "shock": dict(name="shock_512x64_ppc16", size_x=512, size_y=64, delta=8, dt=0.1, c=3.0, dens=16,
                  n_pass=4, periodic_x=False, left_wall=True,
                  species=[_sp(1.0, 16.0, 0.1, 16, 1.0050378), _sp(-1.0, 1.0, 0.1, 16, 1.0050378)],
                  small=(512, 64), crop=(512, 64)),
    # large Weibel filamentation: counter-streaming pair beams along x at +-0.5c
    "weibel": dict(name="weibel_pair_8192x2048_ppc16x4", size_x=8192, size_y=2048, delta=0, dt=0.1, c=3.0,
                   dens=32, n_pass=8, periodic_x=True, left_wall=False,
                   species=[_sp(-1.0, 1.0, 0.05, 16, 1.1547005, 1.0), _sp(-1.0, 1.0, 0.05, 16, 1.1547005, -1.0),
                            _sp(1.0, 1.0, 0.05, 16, 1.1547005, 1.0), _sp(1.0, 1.0, 0.05, 16, 1.1547005, -1.0)],
                   small=(2048, 512), crop=(512, 256)),
}
WORKLOAD = WORKLOADS["thermal"]
FALLBACK_HBM_GBS = 6650.0
B_PER_PARTICLE = 48.0  # {cell, dx, dy, px, py, pz} read and written once
B_PER_CELL = 44.0      # E, B read (24 B); Jx, Jy, Jz, rho, dens written (20 B)
ENSEMBLE_SEED = 4242
ENSEMBLE_GRIDS = ((128, 128), (256, 128), (512, 256), (1024, 256))
ENSEMBLE_PER_RANK = 64
CPU_SAMPLE_PARTICLES = 16_000_000  # members sampled for the CPU legs, in list order


def params(w, **over):
    from spectral_rs_b200.config import Params
    sp = w["species"]
    d = dict(size_x=w["size_x"], size_y=w["size_y"], delta=w["delta"], dt=w["dt"], c=w["c"], dens=w["dens"],
             gamma_inj=max(1.0 + 1e-6, sp[0]["gamma"]), n_pass=w["n_pass"], mass_ratio=sp[0]["m"],
             vth=sp[0]["vth"], periodic_x=w["periodic_x"], left_wall=w["left_wall"])
    if w.get("tile"):
        d["tile_x"], d["tile_y"] = w["tile"]
    if w.get("compensated"):
        d["compensated"] = True
    d.update(over)
    return Params(**d)


def make_sim(w, path="split", seed=0):
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    cfg = Config(params(w), Setup(0), Output(False, False, 1, 1, 1, 1))
    sim = Sim(cfg, path=path)
    # seeded device init, columns [delta, size_x - delta) as the reference fills them
    for k, sp in enumerate(w["species"]):
        sim.init_species(sp["q"], sp["m"], sp["vth"], sp["ppc"], w["delta"], w["size_x"] - w["delta"], sp["gamma"],
                         sp["sign"], True, seed * len(w["species"]) + k + 1)
    return sim


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(0.15)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        rows = [r for r in self.rows if len(r) >= 7]
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(particles, cells, name="k_slot_traffic.json"):
    """dram bytes of the particle kernel from a committed ncu summary, scaled to this launch."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            t = json.load(f)
        return t["dram_bytes_per_particle"] * particles + t.get("dram_bytes_per_cell", 0.0) * cells
    except (OSError, KeyError, ValueError):
        return None


def profile_counters(name):
    """Counters of the committed ncu capture of a kernel (profiles/<name>), or {}."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def roofline(particles, cells, kern_ms, kernel, traffic_file):
    """traffic_file: the committed capture of this kernel on this workload (scaled to the
    launch), or None when no capture of the workload exists (traffic and counters null)."""
    peak, peak_kind = measured_peak()
    alg = B_PER_PARTICLE * particles + B_PER_CELL * cells
    achieved = alg / (kern_ms / 1e3) / 1e9
    prof = profile_counters(traffic_file) if traffic_file else {}
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_per_launch(particles, cells, traffic_file) if traffic_file else None,
            "peak_kind": peak_kind,
            "kernel": kernel, "kernel_ms": kern_ms, "alg_bytes_per_launch": alg,
            "alg_bytes": f"{B_PER_PARTICLE:g} B x {particles} particles + {B_PER_CELL:g} B x {cells} cells",
            # from the committed ncu capture (smsp__inst_executed / particles, and the lane
            # efficiency smsp__thread_inst_executed_per_inst_executed / 32)
            "warp_inst_per_particle": prof.get("warp_inst_per_particle"),
            "lane_efficiency": prof.get("lane_efficiency"), "counters_from": prof.get("source")}


def _events(stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    return e0, e1


# ---------------------------------------------------------------- the ensemble's members
def ensemble_members(n=64, seed=ENSEMBLE_SEED):
    """The uneven shock ensemble, drawn from a fixed seed: shocks against the
    reflecting wall, grids from ENSEMBLE_GRIDS, ppc in [4, 32], mass ratio in
    {1, 16, 64}, upstream drift uniform in [0.05c, 0.3c], thermal spread 0.1c.
    A longer list extends a shorter one (the first 64 members never change)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = ENSEMBLE_GRIDS[rng.integers(len(ENSEMBLE_GRIDS))]
        beta = float(rng.uniform(0.05, 0.3))
        out.append(dict(size_x=nx, size_y=ny, ppc=int(rng.integers(4, 33)),
                        mass_ratio=float(rng.choice([1.0, 16.0, 64.0])), beta=beta,
                        gamma=1.0 / np.sqrt(1.0 - beta * beta)))
    return out


def rank_members(per_rank, rank, world):
    """Member indices of `rank`: the contiguous block [per_rank * rank, per_rank * (rank + 1))
    of an ensemble of per_rank * world members (each member on exactly one rank)."""
    return list(range(per_rank * rank, per_rank * (rank + 1)))


def ensemble_config(m):
    from spectral_rs_b200.config import Config, Params, Setup, Output
    p = Params(size_x=m["size_x"], size_y=m["size_y"], delta=8, dt=0.1, c=3.0, dens=m["ppc"],
               gamma_inj=m["gamma"], n_pass=4, mass_ratio=m["mass_ratio"], vth=0.1, periodic_x=False,
               left_wall=True)
    return Config(p, Setup(0), Output(False, False, 1, 1, 1, 1))


def member_species(m):
    """(charge, mass, vth, ppc, drift gamma) of a member's two species, ions first."""
    return [(1.0, m["mass_ratio"], 0.1, m["ppc"], m["gamma"]), (-1.0, 1.0, 0.1, m["ppc"], m["gamma"])]


def member_particles(m):
    return 2 * m["ppc"] * (m["size_x"] - 16) * m["size_y"]


def member_arrays(m, seed):
    """Host arrays of a member's species (random positions in the cell, the build's seeded generator)."""
    from spectral_rs_b200.config import SpeciesSpec
    from spectral_rs_b200.init import species_arrays
    p = ensemble_config(m).params
    p.random_positions, p.seed = True, seed
    return [(q, mass, vth, species_arrays(p, SpeciesSpec(q, mass, vth, ppc, g, 1.0, 8, m["size_x"] - 8),
                                          seed_offset=k))
            for k, (q, mass, vth, ppc, g) in enumerate(member_species(m))]


def cpu_sample(members, target=CPU_SAMPLE_PARTICLES):
    """Indices of the members the CPU legs time: the list's first members up to `target` particles."""
    idx, acc = [], 0
    for i, m in enumerate(members):
        idx.append(i)
        acc += member_particles(m)
        if acc >= target:
            break
    return idx


# ---------------------------------------------------------------- CPU (oracle) arms
def oracle_crop_rate(w, seconds_target, steps=None, warmup=1):
    """The reference CPU path (C++ restatement, all host threads) on a crop of a single-simulation workload."""
    from oracle import oracle as orc
    from spectral_rs_b200.config import SpeciesSpec
    from spectral_rs_b200.init import species_arrays
    cx, cy = w["crop"]
    p = params(w, size_x=cx, size_y=cy, random_positions=True, seed=7)
    o = orc.OracleSim.from_params(p, dtype=np.float32)
    n = 0
    for k, sp in enumerate(w["species"]):
        spec = SpeciesSpec(charge=sp["q"], mass=sp["m"], vth=sp["vth"], ppc=sp["ppc"], drift_gamma=sp["gamma"],
                           drift_sign=sp["sign"], x0=w["delta"], x1=p.size_x - w["delta"])
        a = species_arrays(p, spec, seed_offset=k)
        o.add_species(sp["q"], sp["m"], sp["vth"], a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                      a["psa"])
        n += len(a["ix"])
    o.prepare()
    o.step(warmup)
    if steps is None:
        t0 = time.perf_counter()
        o.step(1)
        one = time.perf_counter() - t0
        steps = max(1, int(seconds_target / max(one, 1e-3)))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    sample = f"{cx}x{cy} crop, {len(w['species'])} species, {n} particles, {steps} steps"
    return n * steps / dt, orc.num_threads(), sample, dt


def oracle_ensemble_rate(members, seconds_target, steps=None, warmup=1):
    """The reference CPU path on a sample of the ensemble's members: one step is one
    loop iteration of every sampled member, one member after another (the reference
    runs one simulation per process, its push parallel over all host threads)."""
    from oracle import oracle as orc
    idx = cpu_sample(members)
    sims, n = [], 0
    for i in idx:
        m = members[i]
        o = orc.OracleSim.from_params(ensemble_config(m).params, dtype=np.float32)
        for q, mass, vth, a in member_arrays(m, 7000 + i):
            o.add_species(q, mass, vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"], a["psa"])
            n += len(a["ix"])
        o.prepare()
        sims.append(o)

    def one_step():
        for o in sims:
            o.step(1)

    for _ in range(warmup):
        one_step()
    if steps is None:
        t0 = time.perf_counter()
        one_step()
        steps = max(1, int(seconds_target / max(time.perf_counter() - t0, 1e-3)))
    t0 = time.perf_counter()
    for _ in range(steps):
        one_step()
    dt = time.perf_counter() - t0
    for o in sims:
        o.close()
    sample = (f"members {idx[0]}-{idx[-1]} of the ensemble ({len(idx)} of {len(members)} shocks, full size), "
              f"{n} particles, {steps} steps")
    return n * steps / dt, orc.num_threads(), sample, dt


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if w is None:
        members = ensemble_members(ENSEMBLE_PER_RANK)
        rate, cores, sample, dt = oracle_ensemble_rate(members, 0, steps=args.steps, warmup=args.warmup)
        cfg = {"workload": f"ensemble_{len(members)}_shocks", "seed": ENSEMBLE_SEED, "sample": sample}
    else:
        # bounded sample: the crop is ~1/32 of the workload; each step is one loop iteration of it
        rate, cores, sample, dt = oracle_crop_rate(w, 0, steps=args.steps, warmup=args.warmup)
        cfg = {"workload": w["name"], "grid": [w["size_x"], w["size_y"]],
               "ppc_per_species": [sp["ppc"] for sp in w["species"]], "sample": sample}
    line = {"metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                             "sample": sample + " (C++ restatement of the reference CPU path)"},
            "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- rank plumbing
def rank_seed(base_seed, rank):
    """Each replica draws its own plasma."""
    return base_seed + rank


def max_over_ranks(ms, device="cpu"):
    """The timed region's length is the slowest rank's (every rank calls this once)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist:
        dist.barrier()


# ---------------------------------------------------------------- single-simulation measurement
def measure_single(w, steps, warmup, seed, dist=None, sampler=None, timed_steps=3):
    """value: `steps` graph-launched steps (the production path), device-resident;
    then `timed_steps` event-timed steps for the phase split and the particle kernel's time."""
    import torch
    sim = make_sim(w, "split", seed)
    n_particles = sum(len(p) for p in sim.prtls)
    sim.prepare()
    sim.step(warmup)
    stream = torch.cuda.ExternalStream(sim.stream())
    _barrier(dist)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    e0, e1 = _events(stream)
    sim.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    ms = e0.elapsed_time(e1)
    launches = sim.last_launch_count()
    sim.set_timing(True)  # per-step CUDA events around each phase, on the library's stream
    sim.step(timed_steps)
    phases = [float(x) / timed_steps for x in sim.timing()]  # particles, fold, field update, step
    sim.set_timing(False)
    counters = sim.counters()
    diag = sim.diag()
    sim.close()
    cells = w["size_x"] * w["size_y"]
    return {"particles": n_particles, "ms": ms, "launches": launches, "clocks": clocks, "counters": counters,
            "value": n_particles * steps / (ms / 1e3), "ms_per_step": ms / steps,
            "phase_ms_per_step": dict(zip(("particles", "fold", "fields", "step"), phases)),
            # the committed k_slot capture is of the thermal plasma (a 1024 x 256 crop)
            "roofline": roofline(n_particles, cells, phases[0], "k_slot<push,move> (fused push + move + deposit)",
                                 "k_slot_traffic.json" if w["name"].startswith("thermal") else None),
            "diag": {"field_energy_E": diag[0], "field_energy_B": diag[1], "kinetic": diag[2]}}


def plain_single(w, steps, seed):
    import torch
    ps = make_sim(w, "plain", seed)
    n = sum(len(p) for p in ps.prtls)
    ps.prepare()
    ps.step(1)
    stream = torch.cuda.ExternalStream(ps.stream())
    torch.cuda.synchronize()
    a0, a1 = _events(stream)
    ps.step(steps)
    a1.record(stream)
    a1.synchronize()
    pms = a0.elapsed_time(a1)
    ps.close()
    return {"value": n * steps / (pms / 1e3), "unit": "particle-steps/s", "ms_per_step": pms / steps, "steps": steps,
            "path": "plain FP32 (global x = ix + dx, per-phase kernels, global atomics, no sort)"}


def e2e_single(w, steps, seed):
    """Same metric through the public API from pinned host buffers: upload every
    species, prepare, `steps` steps, read the saved fields (into pinned host
    buffers) and the diagnostics back."""
    import torch
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output
    from spectral_rs_b200.init import positions, draws, velocities
    p = params(w, random_positions=True, seed=seed)
    host = []
    for k, sp in enumerate(w["species"]):
        rng = np.random.default_rng([seed, k])
        ix, iy, dx, dy = positions(p.size_x, p.size_y, w["delta"], sp["ppc"], None, None, True, rng)
        n = len(ix)
        arrs = {}
        for name, src in (("ix", ix), ("iy", iy), ("dx", dx), ("dy", dy)):
            t = torch.empty(n, dtype=torch.int64 if name in ("ix", "iy") else torch.float32, pin_memory=True)
            t.numpy().view(src.dtype)[:] = src
            arrs[name] = t.numpy().view(src.dtype)
        del ix, iy, dx, dy
        for name in ("px", "py", "pz", "psa"):
            arrs[name] = torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
        chunk = 1 << 25
        for s0 in range(0, n, chunk):
            s1 = min(n, s0 + chunk)
            nrm, uni = draws(s1 - s0, rng)
            px, py, pz, psa = velocities(nrm, uni, p.c, sp["vth"], sp["gamma"], sp["sign"])
            arrs["px"][s0:s1], arrs["py"][s0:s1], arrs["pz"][s0:s1], arrs["psa"][s0:s1] = px, py, pz, psa
        host.append((sp, arrs))
    cfg = Config(p, Setup(steps), Output(False, False, 1, 1, 1, 1))
    sim = Sim(cfg)
    names = ("Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Dens")
    outs = [torch.empty((p.size_y, p.size_x), dtype=torch.float32, pin_memory=True).numpy() for _ in names]
    h2d = sum(a["ix"].nbytes + a["iy"].nbytes + 6 * a["dx"].nbytes for (_, a) in host)
    t0 = time.perf_counter()
    for sp, a in host:
        sim.add_species(sp["q"], sp["m"], sp["vth"], a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                        a["psa"])
    t1 = time.perf_counter()
    sim.prepare()
    t2 = time.perf_counter()
    sim.step(steps)
    t3 = time.perf_counter()
    out = [sim.flds.spatial(name, with_ghosts=False, out=o) for name, o in zip(names, outs)]
    d = sim.diag()
    dt = time.perf_counter() - t0
    d2h = sum(o.nbytes for o in out) + d.nbytes
    n = sum(len(a["ix"]) for (_, a) in host)
    sim.close()
    return {"value": n * steps / dt, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "wall_s": dt,
            "split_s": {"upload": t1 - t0, "prepare": t2 - t1, "steps": t3 - t2, "readback": t0 + dt - t3},
            "scope": "pinned host arrays -> spx_add_species per species -> spx_prepare -> spx_step(K) -> 10 fields "
                     "(into pinned host buffers) + diag to host"}


def run_single(args, w):
    import torch
    rank, world, local, dist = _init_ranks()
    seed = rank_seed(args.seed, rank)
    e2e = e2e_single(w, args.steps, seed) if rank == 0 and not args.no_e2e else None
    if e2e is not None:
        e2e["ranks_measured"] = 1
    r = measure_single(w, args.steps, args.warmup, seed, dist, ClockSampler(local))
    ms = max_over_ranks(r["ms"], device="cuda") if dist else r["ms"]
    value = r["particles"] * args.steps * world / (ms / 1e3)
    plain = plain_single(w, args.plain_steps, seed) if rank == 0 and not args.no_plain else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, sample, _ = oracle_crop_rate(w, args.cpu_seconds)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": "port",
               "sample": sample + " (C++ restatement of the reference CPU path, OpenMP push/FFT, serial deposit)"}
    if rank == 0:
        line = _line(args, world, value, ms, w["name"], r["launches"], r["clocks"])
        line["config"].update({"grid": [w["size_x"], w["size_y"]],
                               "species": [{"charge": sp["q"], "mass": sp["m"], "vth": sp["vth"], "ppc": sp["ppc"],
                                            "drift_gamma": sp["gamma"], "drift_sign": sp["sign"]}
                                           for sp in w["species"]],
                               "particles_per_gpu": r["particles"], "n_pass": w["n_pass"], "c": w["c"], "dt": w["dt"],
                               "delta": w["delta"], "periodic_x": w["periodic_x"], "left_wall": w["left_wall"],
                               "path": "split, one CUDA graph per step",
                               "parallelism": "replicas" if world > 1 else "single",
                               "l2": _l2_note(r["particles"])})
        line.update({"roofline": r["roofline"], "phase_ms_per_step": r["phase_ms_per_step"], "plain_fp32": plain,
                     "cpu_baseline": cpu, "e2e": e2e, "layout": r["counters"], "diag": r["diag"]})
        if plain:
            line["split_vs_plain"] = value / world / plain["value"]
        print(json.dumps(line), flush=True)
    _finish(dist)


def _l2_note(particles):
    return (f"inputs larger than L2 ({24 * particles / 1e9:.1f} GB particle state)" if 24 * particles > 126e6
            else "inputs smaller than L2 (no flush)")


def _line(args, world, value, ms, workload, launches, clocks):
    return {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": workload}, "gpu_launches": launches, "clocks": clocks}


def _init_ranks():
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local, dist


def _finish(dist):
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched uneven ensemble
def _build_batch(members, idx, tile=None):
    from spectral_rs_b200 import Batch
    b = Batch([ensemble_config(members[i]) for i in idx], tile=tile)
    for sim, i in zip(b.sims, idx):
        m = members[i]
        for k, (q, mass, vth, ppc, g) in enumerate(member_species(m)):
            sim.init_species(q, mass, vth, ppc, 8, m["size_x"] - 8, g, 1.0, True, 2 * i + k + 1)
    return b


def measure_ensemble(members, idx, steps, warmup, dist=None, sampler=None, timed_steps=3, tile=None):
    import torch
    b = _build_batch(members, idx, tile)
    n_particles = sum(len(p) for s in b.sims for p in s.prtls)
    cells = sum(members[i]["size_x"] * members[i]["size_y"] for i in idx)
    b.prepare()
    device_bytes = b.sims[0].counters()["device_bytes"]  # the device's memory in use (all members)
    b.step(warmup)
    stream = torch.cuda.ExternalStream(b.stream())
    _barrier(dist)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    e0, e1 = _events(stream)
    b.step(steps)
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop() if sampler else None
    ms = e0.elapsed_time(e1)
    launches = b.last_launch_count()
    b.set_timing(True)
    b.step(timed_steps)
    part_ms, step_ms = (float(x) / timed_steps for x in b.timing())
    b.close()
    return {"particles": n_particles, "cells": cells, "ms": ms, "launches": launches, "clocks": clocks,
            "device_bytes": device_bytes, "phase_ms_per_step": {"particles": part_ms, "step": step_ms},
            "roofline": roofline(n_particles, cells, part_ms,
                                 "k_slot_batch<push,move> (persistent fused push + move + deposit over all members)",
                                 "k_slot_batch_traffic.json")}


def plain_ensemble(members, idx, steps):
    """The plain single-simulation FP32 path on the same members, one after another."""
    import torch
    from spectral_rs_b200 import Sim
    total_ms, n = 0.0, 0
    for i in idx:
        m = members[i]
        s = Sim(ensemble_config(m), path="plain")
        for k, (q, mass, vth, ppc, g) in enumerate(member_species(m)):
            s.init_species(q, mass, vth, ppc, 8, m["size_x"] - 8, g, 1.0, True, 2 * i + k + 1)
        n += sum(len(p) for p in s.prtls)
        s.prepare()
        s.step(1)
        st = torch.cuda.ExternalStream(s.stream())
        a0, a1 = _events(st)
        s.step(steps)
        a1.record(st)
        a1.synchronize()
        total_ms += a0.elapsed_time(a1) / steps
        s.close()
    return {"value": n / (total_ms / 1e3), "unit": "particle-steps/s", "ms_per_step": total_ms, "steps": steps,
            "path": "plain FP32 (global x = ix + dx, per-phase kernels, global atomics), one simulation after another"}


def e2e_ensemble(members, idx, steps):
    """The same metric through the public API (spx_batch_*) from pinned host buffers:
    upload both species of every member (spx_add_species), spx_batch_prepare, `steps`
    batch steps, read 10 fields of every member (into pinned host buffers) and each
    member's diagnostics back."""
    import torch
    from spectral_rs_b200 import Batch
    arrays = [member_arrays(members[i], 9000 + i) for i in idx]
    n = sum(len(a["ix"]) for sp in arrays for (_, _, _, a) in sp)
    # page-locked host copies of every array (two large allocations, sliced per species)
    pin_i = torch.empty(2 * n, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    pin_f = torch.empty(6 * n, dtype=torch.float32, pin_memory=True).numpy()
    host, oi, of = [], 0, 0
    for sp in arrays:
        hs = []
        for q, mass, vth, a in sp:
            k = len(a["ix"])
            h = {}
            for name in ("ix", "iy"):
                h[name] = pin_i[oi:oi + k]
                h[name][:] = a[name]
                oi += k
            for name in ("dx", "dy", "px", "py", "pz", "psa"):
                h[name] = pin_f[of:of + k]
                h[name][:] = a[name]
                of += k
            hs.append((q, mass, vth, h))
        host.append(hs)
    del arrays
    names = ("Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Dens")
    cells = sum(members[i]["size_x"] * members[i]["size_y"] for i in idx)
    pin_o = torch.empty(len(names) * cells, dtype=torch.float32, pin_memory=True).numpy()
    b = Batch([ensemble_config(members[i]) for i in idx])
    t0 = time.perf_counter()
    for sim, hs in zip(b.sims, host):
        for q, mass, vth, h in hs:
            sim.add_species(q, mass, vth, h["ix"], h["iy"], h["dx"], h["dy"], h["px"], h["py"], h["pz"], h["psa"])
    t1 = time.perf_counter()
    b.prepare()
    t2 = time.perf_counter()
    b.step(steps)
    t3 = time.perf_counter()
    off = 0
    for name in names:  # one spx_batch_get_field per field: every member's copy, one synchronisation
        outs = []
        for sim in b.sims:
            c = sim.size_x * sim.size_y
            outs.append(pin_o[off:off + c].reshape(sim.size_y, sim.size_x))
            off += c
        b.get_field(name, with_ghosts=False, out=outs)
    diags = [sim.diag() for sim in b.sims]
    dt = time.perf_counter() - t0
    b.close()
    h2d = 40 * n  # ix, iy (8 B each), dx, dy, px, py, pz, psa (4 B each) per particle
    d2h = 4 * off + sum(d.nbytes for d in diags)
    return {"value": n * steps / dt, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "wall_s": dt,
            "split_s": {"upload": t1 - t0, "prepare": t2 - t1, "steps": t3 - t2, "readback": t0 + dt - t3},
            "scope": "pinned host arrays -> spx_add_species (2 per member) -> spx_batch_prepare -> "
                     "spx_batch_step(K) -> 10 fields of every member (spx_batch_get_field into pinned host "
                     "buffers) + spx_diag per member"}


def run_ensemble(args):
    rank, world, local, dist = _init_ranks()
    per = args.ensemble
    members = ensemble_members(per * world)
    idx = rank_members(per, rank, world)
    e2e = e2e_ensemble(members, idx, args.steps) if rank == 0 and not args.no_e2e else None
    if e2e is not None:
        e2e["ranks_measured"] = 1
    tile = tuple(int(v) for v in args.tile.lower().split("x")) if args.tile else None
    r = measure_ensemble(members, idx, args.steps, args.warmup, dist, ClockSampler(local), tile=tile)
    ms = max_over_ranks(r["ms"], device="cuda") if dist else r["ms"]
    value = r["particles"] * args.steps * world / (ms / 1e3)  # every rank holds the same number of members
    plain = plain_ensemble(members, idx, args.plain_steps) if rank == 0 and not args.no_plain else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, sample, _ = oracle_ensemble_rate(members[:per], args.cpu_seconds)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": "port",
               "sample": sample + " (C++ restatement of the reference CPU path, OpenMP push/FFT, serial deposit)"}
    extras = {}
    if rank == 0 and not args.no_extras:
        for key, wname in (("thermal_c2", "thermal"), ("weibel_c5", "weibel")):
            w = WORKLOADS[wname]
            x = measure_single(w, args.extra_steps, 3, args.seed)
            extras[key] = {"workload": w["name"], "particles": x["particles"], "value": x["value"],
                           "unit": "particle-steps/s", "steps": args.extra_steps, "ms_per_step": x["ms_per_step"],
                           "phase_ms_per_step": x["phase_ms_per_step"], "roofline": x["roofline"],
                           "gpu_launches": x["launches"]}
    if rank == 0:
        line = _line(args, world, value, ms, f"ensemble_{per}_shocks", r["launches"], r["clocks"])
        line["config"].update({"seed": ENSEMBLE_SEED, "members_per_gpu": per, "particles_per_gpu": r["particles"],
                               "cells_per_gpu": r["cells"],
                               "grids": [[members[i]["size_x"], members[i]["size_y"]] for i in idx],
                               "ppc": [members[i]["ppc"] for i in idx],
                               "mass_ratio": [members[i]["mass_ratio"] for i in idx],
                               "drift_beta": [round(members[i]["beta"], 4) for i in idx],
                               "vth": 0.1, "c": 3.0, "dt": 0.1, "n_pass": 4, "delta": 8, "walls": "right + left",
                               "path": "split, batched (persistent work-queue particle kernel, one graph per step)",
                               "tile": list(tile) if tile else [8, 8],
                               "device_gb": round(r["device_bytes"] / 1e9, 2),
                               "parallelism": f"member list partitioned over {world} ranks" if world > 1 else "single",
                               "l2": _l2_note(r["particles"])})
        line.update({"roofline": r["roofline"], "phase_ms_per_step": r["phase_ms_per_step"], "plain_fp32": plain,
                     "cpu_baseline": cpu, "e2e": e2e})
        if plain:
            line["split_vs_plain"] = value / world / plain["value"]
        line.update(extras)
        print(json.dumps(line), flush=True)
    _finish(dist)


# ---------------------------------------------------------------- precision study (two-stream)
def two_stream_study(args):
    """Symmetric two-stream electron beams (+-0.2c along x, thermal spread 0.01c, 32 per cell
    per beam, immobile neutralizing ions left out: their uniform background only touches
    k = 0, which the solver ignores) on the full 2048 x 2048 grid for 2000 steps, split,
    compensated and plain paths.  Compared with the FP64 oracle history of the 128 x 128
    crop (tests/golden/two_stream_energy.json): growth rate of the field energy, its
    saturated level per cell, and the error at the end of the linear phase."""
    import torch
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Params, Setup, Output
    with open(os.path.join(ROOT, "tests", "golden", "two_stream_energy.json")) as f:
        ref = json.load(f)
    st = ref["study"]
    n = args.study_size
    steps, every, dt = args.study_steps, st["every"], st["dt"]
    e64 = np.array(ref["fp64"]["E"]) / (st["size_x"] * st["size_y"])  # energy per cell
    t64 = (np.arange(len(e64)) + 1) * every * dt
    peak = int(np.argmax(e64))
    start = int(np.argmin(e64[:peak + 1]))
    end = start + int(np.flatnonzero(e64[start:] > 0.5 * e64[peak])[0])
    win = np.arange(start + (end - start) // 4, end + 1)
    g64 = np.polyfit(t64[win], np.log(e64[win]), 1)[0] / 2
    late64 = float(np.mean(e64[len(e64) * 3 // 4:]))
    out = {"study": "two-stream precision", "grid": [n, n], "steps": steps, "particles": 2 * st["ppc"] * n * n,
           "fp64_crop": {"grid": [st["size_x"], st["size_y"]], "growth_rate": g64, "late_energy_per_cell": late64,
                         "peak_energy_per_cell": float(e64[peak])}}
    for mode in args.study_modes.split(","):
        p = Params(size_x=n, size_y=n, delta=0, dt=dt, c=st["c"], dens=st["dens"], gamma_inj=st["gamma_inj"],
                   n_pass=st["n_pass"], periodic_x=True, compensated=mode == "compensated")
        sim = Sim(Config(p, Setup(steps), Output(False, False, 1, 1, 1, 1)), path="plain" if mode == "plain" else "split")
        for k, sign in enumerate((1.0, -1.0)):
            sim.init_species(-1.0, 1.0, st["vth"], st["ppc"], 0, n, st["gamma_inj"], sign, True, 77 + k)
        sim.prepare()
        hist = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(0, steps, every):
            sim.step(every)
            hist.append(float(sim.diag()[0]) / (n * n))
        wall = time.perf_counter() - t0
        sim.close()
        e = np.array(hist)
        t = (np.arange(len(e)) + 1) * every * dt
        pk = int(np.argmax(e))
        s0 = int(np.argmin(e[:pk + 1]))
        s1 = s0 + int(np.flatnonzero(e[s0:] > 0.5 * e[pk])[0])
        w = np.arange(s0 + (s1 - s0) // 4, s1 + 1)
        g = float(np.polyfit(t[w], np.log(e[w]), 1)[0] / 2) if len(w) >= 3 else None
        late = float(np.mean(e[len(e) * 3 // 4:]))
        out[mode] = {"growth_rate": g, "growth_rate_rel_err_vs_fp64": None if g is None else abs(g - g64) / g64,
                     "late_energy_per_cell": late, "late_rel_diff_vs_fp64": abs(late - late64) / late64,
                     "peak_energy_per_cell": float(e[pk]), "peak_step": (pk + 1) * every,
                     "fp64_peak_step": (peak + 1) * every, "wall_s": wall,
                     "history_every": every, "energy_per_cell": [round(x, 8) for x in e.tolist()]}
        print(json.dumps({mode: {k: v for k, v in out[mode].items() if k != "energy_per_cell"}}), flush=True)
    with open(args.study_out, "w") as f:
        json.dump(out, f)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--extra-steps", type=int, default=10, help="timed steps of the C2 / C5 extra keys")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="ensemble: skip the C2 / C5 keys")
    ap.add_argument("--small", action="store_true", help="single workloads: 1/16 of the grid (quick checks)")
    ap.add_argument("--workload", default="ensemble", choices=sorted(WORKLOADS) + ["ensemble", "two_stream"])
    ap.add_argument("--tile", default=None, help="split-path tile shape TXxTY (default: the library's choice)")
    ap.add_argument("--compensated", action="store_true", help="Kahan-compensated current sums (split path)")
    ap.add_argument("--ppc", type=int, default=None,
                    help="particles per cell of every species (field-phase profiling on the full grid)")
    ap.add_argument("--ensemble", type=int, default=ENSEMBLE_PER_RANK, help="members of the ensemble per GPU")
    ap.add_argument("--study-size", type=int, default=2048, help="two_stream: grid side")
    ap.add_argument("--study-steps", type=int, default=2000, help="two_stream: steps")
    ap.add_argument("--study-modes", default="split,compensated,plain", help="two_stream: paths")
    ap.add_argument("--study-out", default="two_stream_study.json", help="two_stream: result file")
    args = ap.parse_args()
    if args.workload == "two_stream":
        two_stream_study(args)
        return
    if args.workload == "ensemble":
        if args.impl == "reference":
            run_reference(args, None)
        else:
            run_ensemble(args)
        return
    w = dict(WORKLOADS[args.workload])
    if args.small:
        sx, sy = w["small"]
        w.update(size_x=sx, size_y=sy, name=f"{w['name']}_small_{sx}x{sy}")
    if args.tile:
        w["tile"] = tuple(int(v) for v in args.tile.lower().split("x"))
    if args.compensated:
        w["compensated"] = True
        w["name"] += "_compensated"
    if args.ppc:
        w["species"] = [dict(sp, ppc=args.ppc) for sp in w["species"]]
        w["name"] += f"_ppc{args.ppc}"
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_single(args, w)


if __name__ == "__main__":
    main()
