#!/usr/bin/env python
"""Benchmark of the spectral_rs per-timestep hot path on B200.

Metric: particle-steps/s (particles x steps / device time of the timed steps)
and the HBM roofline fraction of the fused push + move + deposit kernel.

Workload (one GPU): the plain method at scale -- a 2-D periodic thermal
electron-proton plasma on a 4096 x 1024 grid, mass ratio 64, 64 particles per
cell per species (536,870,912 particles), Maxwellian momenta with thermal
spread 0.05c drawn from a seed, FP32 fields and particles, 4 binomial filter
passes per step, c = 3.0, dt = 0.1 (Courant number c dt = 0.3; the reference
algorithm is numerically unstable for this plasma at c dt = 0.45).  Synthetic
data from the build's own seeded generator; a "step" is one iteration of the
reference's loop (zero sources, move + deposit both species, ghost fold,
Flds::update, Boris push).  The particle arrays (13 GB) exceed the 126 MB L2,
so no flush is needed between steps.

Besides `value` (device-resident, split path) the line carries:
  plain_fp32   the plain single-simulation FP32 GPU path on the same workload
  roofline     the fused particle kernel: algorithmic bytes / CUDA-event time
  cpu_baseline the C++ restatement of the reference CPU path (oracle/) on a crop
  e2e          the same metric through the public API from host buffers
  clocks       SM clocks sampled during the timed region

--impl reference times the reference's CPU path (the oracle restatement; the
Rust crate cannot be built here) on all host cores, same metric and workload,
each step a 512 x 256 crop of it.

Multi-GPU (torchrun): the workload does not shard without exchange steps, so
N > 1 runs N independent replicas (weak scaling); the time is the max over ranks.
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


# Workloads (species: ions first, as run() creates them, src/lib.rs:124-126).
# c = 3.0, dt = 0.1 everywhere: Courant number c dt = 0.3 (the reference
# algorithm is numerically unstable for these plasmas at c dt = 0.45).
WORKLOADS = {
    # the headline: the plain method at scale
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


def traffic_per_launch(particles, cells):
    """dram bytes of the fused kernel from the committed ncu summary, scaled to this launch."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_slot_traffic.json")) as f:
            t = json.load(f)
        return t["dram_bytes_per_particle"] * particles + t.get("dram_bytes_per_cell", 0.0) * cells
    except (OSError, KeyError, ValueError):
        return None


# ---------------------------------------------------------------- CPU (oracle) arms
def oracle_crop_rate(w, seconds_target, steps=None, warmup=1):
    """The reference CPU path (C++ restatement, all host threads) on a crop of the workload."""
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


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # bounded sample: the crop is ~1/32 of the workload; each step is one loop iteration of it
    rate, cores, sample, dt = oracle_crop_rate(w, 0, steps=args.steps, warmup=args.warmup)
    line = {"metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": w["name"], "grid": [w["size_x"], w["size_y"]],
                       "ppc_per_species": [sp["ppc"] for sp in w["species"]], "sample": sample},
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


# ---------------------------------------------------------------- GPU arm
def e2e_run(w, steps, seed):
    """Same metric through the public API from pinned host buffers: upload both
    species, prepare, `steps` steps, read the saved fields (into pinned host
    buffers) and the diagnostics back."""
    import torch
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.config import Config, Setup, Output, SpeciesSpec
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
    # page-locked result buffers, like the inputs
    outs = [torch.empty((p.size_y, p.size_x), dtype=torch.float32, pin_memory=True).numpy() for _ in names]
    h2d = sum(a["ix"].nbytes + a["iy"].nbytes + 6 * a["dx"].nbytes for (_, a) in host)
    t0 = time.perf_counter()
    per_species = []
    for sp, a in host:
        ts = time.perf_counter()
        sim.add_species(sp["q"], sp["m"], sp["vth"], a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"], a["pz"],
                        a["psa"])
        per_species.append(time.perf_counter() - ts)
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
            "split_s": {"upload": t1 - t0, "upload_per_species": per_species, "prepare": t2 - t1, "steps": t3 - t2,
                        "readback": t0 + dt - t3},
            "scope": "pinned host arrays -> spx_add_species x2 -> spx_prepare -> spx_step(K) -> 10 fields "
                     "(into pinned host buffers) + diag to host"}


def run_gpu(args, w):
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
    seed = rank_seed(args.seed, rank)

    # end to end through the public API, first, on the clean device; rank 0 only (the pinned
    # host copy of the workload is 21 GB per rank)
    e2e = e2e_run(w, args.steps, seed) if rank == 0 and not args.no_e2e else None
    if e2e is not None:
        e2e["ranks_measured"] = 1

    sim = make_sim(w, "split", seed)
    n_particles = sum(len(p) for p in sim.prtls)
    cells = w["size_x"] * w["size_y"]
    sim.prepare()
    sim.step(args.warmup)
    stream = torch.cuda.ExternalStream(sim.stream())
    sim.set_timing(True)  # per-step CUDA events around each phase, on the library's stream
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    phases = sim.timing()  # [particles, fold, field update, step] summed over the steps
    launches = sim.last_launch_count()
    counters = sim.counters()
    sim.set_timing(False)
    diag = sim.diag()
    if dist:
        ms = max_over_ranks(ms, device="cuda")
        dist.barrier()
    sim.close()
    del sim
    value = n_particles * args.steps * world / (ms / 1e3)

    peak, peak_kind = measured_peak()
    kern_ms = float(phases[0]) / args.steps
    alg_bytes = B_PER_PARTICLE * n_particles + B_PER_CELL * cells
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    traffic = traffic_per_launch(n_particles, cells)


    plain = None
    if not args.no_plain and rank == 0:
        ps = make_sim(w, "plain", seed)
        ps.prepare()
        ps.step(1)
        stream_p = torch.cuda.ExternalStream(ps.stream())
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream_p)
        ps.step(args.plain_steps)
        a1.record(stream_p)
        a1.synchronize()
        pms = a0.elapsed_time(a1)
        ps.close()
        plain = {"value": n_particles * args.plain_steps / (pms / 1e3), "unit": "particle-steps/s",
                 "ms_per_step": pms / args.plain_steps, "steps": args.plain_steps,
                 "path": "plain FP32 (global x = ix + dx, per-phase kernels, global atomics, no sort)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, sample, _ = oracle_crop_rate(w, args.cpu_seconds)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": "port",
               "sample": sample + " (C++ restatement of the reference CPU path, OpenMP push/FFT, serial deposit)"}

    if rank == 0:
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded device init)",
                "config": {"workload": w["name"], "grid": [w["size_x"], w["size_y"]],
                           "species": [{"charge": sp["q"], "mass": sp["m"], "vth": sp["vth"], "ppc": sp["ppc"],
                                        "drift_gamma": sp["gamma"], "drift_sign": sp["sign"]}
                                       for sp in w["species"]],
                           "particles_per_gpu": n_particles, "n_pass": w["n_pass"], "c": w["c"], "dt": w["dt"],
                           "delta": w["delta"], "periodic_x": w["periodic_x"], "left_wall": w["left_wall"],
                           "path": "split", "parallelism": "replicas" if world > 1 else "single",
                           "l2": f"inputs larger than L2 ({24 * n_particles / 1e9:.1f} GB particle state)"
                           if 24 * n_particles > 126e6 else "inputs smaller than L2 (no flush)"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": "k_slot<push,move> (fused push + move + deposit)",
                             "kernel_ms": kern_ms, "alg_bytes_per_launch": alg_bytes},
                "phase_ms_per_step": {"particles": float(phases[0]) / args.steps,
                                      "fold": float(phases[1]) / args.steps,
                                      "fields": float(phases[2]) / args.steps,
                                      "step": float(phases[3]) / args.steps},
                "plain_fp32": plain, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches, "layout": counters,
                "diag": {"field_energy_E": diag[0], "field_energy_B": diag[1], "kinetic": diag[2]}}
        if plain:
            line["split_vs_plain"] = value / world / plain["value"]
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched uneven ensemble
ENSEMBLE_SEED = 4242
ENSEMBLE_GRIDS = ((128, 128), (256, 128), (512, 256), (1024, 256))


def ensemble_members(n=64, seed=ENSEMBLE_SEED):
    """The uneven shock ensemble, drawn from a fixed seed: shocks against the
    reflecting wall, grids from ENSEMBLE_GRIDS, ppc in [4, 32], mass ratio in
    {1, 16, 64}, upstream drift uniform in [0.05c, 0.3c], thermal spread 0.1c."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = ENSEMBLE_GRIDS[rng.integers(len(ENSEMBLE_GRIDS))]
        beta = float(rng.uniform(0.05, 0.3))
        out.append(dict(size_x=nx, size_y=ny, ppc=int(rng.integers(4, 33)),
                        mass_ratio=float(rng.choice([1.0, 16.0, 64.0])), beta=beta,
                        gamma=1.0 / np.sqrt(1.0 - beta * beta)))
    return out


def ensemble_config(m):
    from spectral_rs_b200.config import Config, Params, Setup, Output
    p = Params(size_x=m["size_x"], size_y=m["size_y"], delta=8, dt=0.1, c=3.0, dens=m["ppc"],
               gamma_inj=m["gamma"], n_pass=4, mass_ratio=m["mass_ratio"], vth=0.1, periodic_x=False,
               left_wall=True)
    return Config(p, Setup(0), Output(False, False, 1, 1, 1, 1))


def run_ensemble(args):
    import torch
    from spectral_rs_b200 import Batch, Sim
    members = ensemble_members(args.ensemble)
    cfgs = [ensemble_config(m) for m in members]
    b = Batch(cfgs)
    for k, (sim, m) in enumerate(zip(b.sims, members)):
        x0, x1 = 8, m["size_x"] - 8
        sim.init_species(1.0, m["mass_ratio"], 0.1, m["ppc"], x0, x1, m["gamma"], 1.0, True, 2 * k + 1)
        sim.init_species(-1.0, 1.0, 0.1, m["ppc"], x0, x1, m["gamma"], 1.0, True, 2 * k + 2)
    n_particles = sum(len(p) for s in b.sims for p in s.prtls)
    b.prepare()
    b.step(args.warmup)
    stream = torch.cuda.ExternalStream(b.stream())
    torch.cuda.synchronize()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = b.last_launch_count()
    b.set_timing(True)
    b.step(3)
    part_ms, step_ms = (float(x) / 3 for x in b.timing())
    b.close()
    value = n_particles * args.steps / (ms / 1e3)
    # the plain single-simulation FP32 path on the same members, one after the other
    plain_ms = 0.0
    if not args.no_plain:
        for k, (cfg, m) in enumerate(zip(cfgs, members)):
            s = Sim(cfg, path="plain")
            x0, x1 = 8, m["size_x"] - 8
            s.init_species(1.0, m["mass_ratio"], 0.1, m["ppc"], x0, x1, m["gamma"], 1.0, True, 2 * k + 1)
            s.init_species(-1.0, 1.0, 0.1, m["ppc"], x0, x1, m["gamma"], 1.0, True, 2 * k + 2)
            s.prepare()
            s.step(1)
            st = torch.cuda.ExternalStream(s.stream())
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(st)
            s.step(args.plain_steps)
            a1.record(st)
            a1.synchronize()
            plain_ms += a0.elapsed_time(a1) / args.plain_steps
            s.close()
    line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded device init)",
            "config": {"workload": f"ensemble_{args.ensemble}_shocks", "seed": ENSEMBLE_SEED,
                       "particles": n_particles, "grids": [[m["size_x"], m["size_y"]] for m in members],
                       "path": "split, batched (persistent work-queue particle kernel, one graph per step)"},
            "phase_ms_per_step": {"particles": part_ms, "step": step_ms}, "gpu_launches": launches,
            "clocks": clocks}
    if plain_ms:
        line["plain_fp32"] = {"value": n_particles / (plain_ms / 1e3), "unit": "particle-steps/s",
                              "ms_per_step": plain_ms, "path": "plain FP32, one simulation after another"}
        line["split_vs_plain"] = value / line["plain_fp32"]["value"]
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--small", action="store_true", help="1/16 of the workload (quick checks)")
    ap.add_argument("--workload", default="thermal", choices=sorted(WORKLOADS) + ["ensemble"])
    ap.add_argument("--tile", default=None, help="split-path tile shape TXxTY (default: the library's choice)")
    ap.add_argument("--compensated", action="store_true", help="Kahan-compensated current sums (split path)")
    ap.add_argument("--ppc", type=int, default=None,
                    help="particles per cell of every species (field-phase profiling on the full grid)")
    ap.add_argument("--ensemble", type=int, default=64, help="members of the batched ensemble")
    args = ap.parse_args()
    if args.workload == "ensemble":
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
        run_gpu(args, w)


if __name__ == "__main__":
    main()
