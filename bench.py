"""Benchmark of the FFT translational-rotational search (rotations/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 64^3 grids at 0.5 A, K = 9 receptor grids (8 vdW + elec) from a seeded synthetic
receptor of 2,500 atoms in a 32 A cube; a 40-atom ligand, 100 conformers x 1,000 uniform
quaternions = 1e5 rotations per rank per step. One step = one full search of those
rotations through the C-ABI. With N ranks (torchrun, one process per GPU) every rank
searches its own 1e5 rotations (weak scaling, no collective inside the search); value is
the rotations of all ranks over the slowest rank's device time.

Timed region: W untimed warm-up steps, then a barrier + synchronize, K steps each bracketed
by CUDA events on the search stream, a 256 MiB L2 flush between steps (outside the events),
barrier + synchronize, max over ranks. `e2e` repeats the measurement through cdk_search with
pinned host buffers (H2D of the inputs and D2H of the results inside the timed region).

--impl reference times the reference's CPU implementation of the path (cpuNaive's dense
direct correlation, restated in oracle/, all host threads) on a bounded sample of the same
workload per step; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "docked rotations/s @64³ K=9: tensor-core vs FP32 form, ≤1e-3 rel err; p99 lat"
WORKLOAD = "c1_64"
N_CONF, N_Q = 100, 1000


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"cdk_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        smax.append(float(parts[2]))
                    except ValueError:
                        continue
                    for nm, v in zip(names, parts[5:9]):
                        if v.lower() == "active":
                            reasons.add(nm)
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_rank_workload(rank: int, world: int):
    """The global job is world x 100 conformers; rank r owns conformers [r*100, (r+1)*100)."""
    from cdocker_b200 import synth
    from cdocker_b200.shard import conformer_range
    w = synth.make_workload(WORKLOAD, seed=0, n_conf=1, n_q=1)
    total_conf = N_CONF * world
    b, e = conformer_range(total_conf, rank, world)
    xyz, radii, eps, charge = synth.make_ligand(40, synth.CONFIGS[WORKLOAD][4], 1)
    coor_all = synth.make_conformers(xyz, total_conf, 2)
    from cdocker_b200 import api
    q_all = api.quaternion_uniform_sampling(3, total_conf, N_Q)
    w.coor = np.ascontiguousarray(coor_all[b:e])
    w.quats = np.ascontiguousarray(q_all[b:e])
    return w


def cpu_baseline(w, budget_s: float = 15.0, threads: int = 0) -> dict:
    """cpuNaive's dense direct correlation (oracle port) on the host cores, bounded sample."""
    from oracle import oracle as O
    cores = threads or os.cpu_count() or 1
    q = w.quats.reshape(-1, 4)
    n = max(cores, 1)
    done, t_total, start = 0, 0.0, 0
    while t_total < budget_s and start + n <= q.shape[0]:
        t0 = time.perf_counter()
        O.search_direct(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot,
                        q[start:start + n][None], prec=0, dense=1, nthreads=cores)
        t_total += time.perf_counter() - t0
        done += n
        start += n
        if t_total > budget_s / 3:
            break
    return {"value": done / t_total, "unit": "rotations/s", "cores": cores, "kind": "port",
            "sample": f"{done} rotations of conformer 0 (64^3, K=9, 40 atoms), cpuNaive dense "
                      f"loop (src/cpuNaive.cpp:194-216) restated, {cores} threads, "
                      f"{t_total:.1f} s"}


def reference_cufft_sample(w, n_rot: int = 1000) -> dict:
    """The reference's own cuFFT path (oracle/_ref, batch 50, host fill, PCIe copies)."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_CUFFT_LIB):
        return {"unavailable": "oracle/_ref/libcdk_ref_cufft.so not built"}
    L = O.refcufft()
    q = np.ascontiguousarray(w.quats.reshape(-1, 4)[:n_rot])
    minE = np.empty(n_rot, np.float32)
    idx = np.empty((n_rot, 3), np.int32)
    times = np.zeros(6, np.float64)
    rc = L.refcufft_search(w.n, w.n, w.n, w.spacing, 8, O._pf(O._f32(w.grid_radii)),
                           O._pf(O._f32(w.all_grids)), w.coor.shape[1],
                           O._pf(np.ascontiguousarray(w.coor[0])), O._pf(O._f32(w.charge)),
                           O._pf(O._f32(w.eps)), O._pf(O._f32(w.radii)), n_rot, O._pf(q), 50,
                           O._pf(minE), O._pi(idx), times.ctypes.data_as(O._dp))
    if rc != 0:
        return {"unavailable": f"reference cuFFT path returned {rc}"}
    tot = times[5] / 1e3
    return {"value": n_rot / tot, "unit": "rotations/s",
            "sample": f"{n_rot} rotations of conformer 0, batch 50, 1 host thread",
            "stage_ms": {"fill": round(times[0], 1), "h2d": round(times[1], 1),
                         "gpu_fft_conj_sum": round(times[2], 1), "d2h": round(times[3], 1),
                         "argmin": round(times[4], 1)}}


def run_reference(args, rank, world):
    if rank != 0:
        return
    w = make_rank_workload(0, 1)
    cores = os.cpu_count() or 1
    q = w.quats.reshape(-1, 4)
    per_step = cores
    step_times = []
    total = args.warmup + args.steps
    for s in range(total):
        qs = q[(s * per_step) % q.shape[0]:][:per_step]
        from oracle import oracle as O
        t0 = time.perf_counter()
        O.search_direct(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot, qs[None],
                        prec=0, dense=1, nthreads=cores)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            step_times.append(dt)
    t = sum(step_times)
    value = per_step * len(step_times) / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rotations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / len(step_times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "64^3 grid, K=9, 40-atom ligand (config 1); each step a bounded "
                               f"sample of {per_step} rotations",
                   "grid": 64, "K": 9, "ligand_atoms": 40},
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} rotations per step, cpuNaive dense loop "
                                   "(src/cpuNaive.cpp:82-216) restated in oracle/, "
                                   f"{cores} threads"},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from cdocker_b200 import Receptor

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = make_rank_workload(rank, world)
    n_conf, n_atom = w.coor.shape[0], w.coor.shape[1]
    n_rot = n_conf * N_Q
    rec = Receptor(w.grids, w.spacing, device=local_rank, wave_rotations=args.wave,
                   col_tile=args.col_tile, use_graphs=args.graphs)
    # resident inputs
    d_coor = torch.from_numpy(w.coor).to(dev)
    d_charge = torch.from_numpy(w.charge).to(dev)
    d_eps = torch.from_numpy(w.eps).to(dev)
    d_slot = torch.from_numpy(w.slot).to(dev)
    d_q = torch.from_numpy(w.quats).to(dev)
    d_e = torch.empty(n_rot, device=dev)
    d_i = torch.empty(n_rot, 3, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step_device():
        rec.search_device(n_atom, n_conf, d_coor.data_ptr(), d_charge.data_ptr(),
                          d_eps.data_ptr(), d_slot.data_ptr(), N_Q, d_q.data_ptr(),
                          d_e.data_ptr(), d_i.data_ptr(), stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local_rank)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    barrier()
    sampler.start()
    time.sleep(0.3)
    for s in range(args.steps):
        with torch.cuda.stream(stream):
            evs[s][0].record(stream)
            step_device()
            evs[s][1].record(stream)
            flush.fill_(s & 0xff)
    barrier()
    clocks = sampler.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    dev_ms = max_over_ranks(dev_ms)
    stats = rec.stats()
    launches_per_step = stats["launches"]
    value = world * n_rot * args.steps / (dev_ms / 1e3)

    # per-kernel timing of one search on the same stream (events around each launch group are
    # not available through the C-ABI, so the roofline kernel is timed by the profile pass)
    # e2e: host buffers through cdk_search, pinned memory, copies inside the timed region
    h_coor = torch.from_numpy(w.coor).pin_memory()
    h_q = torch.from_numpy(w.quats).pin_memory()
    h_e = torch.empty(n_rot, dtype=torch.float32).pin_memory()
    h_i = torch.empty(n_rot, 3, dtype=torch.int32).pin_memory()
    from cdocker_b200 import _lib as L
    import ctypes as C
    lib = L.lib()
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    charge = np.ascontiguousarray(w.charge, np.float32)
    eps = np.ascontiguousarray(w.eps, np.float32)
    slot = np.ascontiguousarray(w.slot, np.int32)

    def step_e2e():
        L.check(lib.cdk_search(rec.handle, n_atom, n_conf, C.cast(h_coor.data_ptr(), fp),
                               charge.ctypes.data_as(fp), eps.ctypes.data_as(fp),
                               slot.ctypes.data_as(ip), N_Q, C.cast(h_q.data_ptr(), fp),
                               C.cast(h_e.data_ptr(), fp), C.cast(h_i.data_ptr(), ip),
                               C.c_void_p(stream.cuda_stream)))

    for _ in range(max(1, args.warmup)):
        step_e2e()
    barrier()
    e2e_ms = 0.0
    for s in range(args.steps):
        t0 = time.perf_counter()
        step_e2e()  # returns after the D2H of the results has completed
        e2e_ms += 1e3 * (time.perf_counter() - t0)
        with torch.cuda.stream(stream):
            flush.fill_(s & 0xff)
        torch.cuda.synchronize(dev)
    barrier()
    e2e_ms = max_over_ranks(e2e_ms)
    e2e_val = world * n_rot * args.steps / (e2e_ms / 1e3)
    h2d = w.coor.nbytes + w.quats.nbytes + charge.nbytes + eps.nbytes + slot.nbytes
    d2h = n_rot * 4 + n_rot * 12
    # correctness spot check of the timed results (rank 0, a few rotations vs the oracle)
    check = None
    if rank == 0 and not args.no_check:
        from oracle import oracle as O
        sel = np.arange(0, n_rot, max(1, n_rot // 8))[:8]
        qs = w.quats.reshape(-1, 4)[sel]
        errs = []
        for j, r in enumerate(sel):
            _, ri, r64 = O.search_direct(w.grids, w.spacing, w.coor[r // N_Q], w.charge, w.eps,
                                         w.slot, qs[j][None, None], prec=1)
            errs.append(abs(float(h_e[r]) - r64[0]) / max(1.0, abs(r64[0])))
        check = {"rotations_checked": int(len(sel)), "max_rel_err_vs_fp64": max(errs)}

    if rank == 0:
        hbm, peak_kind = _peaks()
        nc = 64 * 64 * 33  # half-spectrum points of one grid
        b_rot = 8 * 9 * 64 ** 3 + 16 * 9 * nc + 16 * nc + 8 * 64 ** 3
        rps = value / world
        line = {
            "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "config 1: 64^3 grid at 0.5 A, K=9, 2,500-atom synthetic "
                                   "receptor, 40-atom ligand, 100 conformers x 1,000 "
                                   "quaternions = 1e5 rotations per rank per step",
                       "form": "fp32", "grid": 64, "K": 9, "rotations_per_step": n_rot * world,
                       "l2": "256 MiB written between timed steps; per-step scratch "
                             f"{rec.stats().get('waves', 0)} waves, far above L2",
                       "wave_rotations": args.wave, "parallelism": f"rotation shards x{world}"},
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks,
            "e2e": {"value": e2e_val, "unit": "rotations/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "fft_roofline": {"bytes_per_rotation": b_rot, "achieved_gbs": rps * b_rot / 1e9,
                             "peak_gbs": hbm, "frac": rps * b_rot / 1e9 / hbm,
                             "peak_kind": peak_kind,
                             "note": "staged-pipeline algorithmic bytes B_rot = 8KN + 16K*Nc + "
                                     "16Nc + 8N per rotation, per GPU"},
            "check": check,
        }
        if args.roofline_json and os.path.exists(args.roofline_json):
            with open(args.roofline_json) as f:
                line["roofline"] = json.load(f)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w, budget_s=args.cpu_budget)
        if args.ref_cufft:
            line["reference_cufft"] = reference_cufft_sample(w)
        print(json.dumps(line), flush=True)
    rec.close()


def profile_run(args):
    """One warm-up and one timed search of `--profile-run` rotations (first conformers of the
    config-1 workload), per-kernel device times from events around every launch."""
    import torch
    from cdocker_b200 import Receptor
    w = make_rank_workload(0, 1)
    n_q = N_Q
    n_conf = max(1, min(N_CONF, (args.profile_run + n_q - 1) // n_q))
    if args.profile_run < n_q:
        n_q = args.profile_run
    dev = torch.device("cuda", 0)
    coor = torch.from_numpy(np.ascontiguousarray(w.coor[:n_conf])).to(dev)
    q = torch.from_numpy(np.ascontiguousarray(w.quats[:n_conf, :n_q])).to(dev)
    ch = torch.from_numpy(w.charge).to(dev)
    ep = torch.from_numpy(w.eps).to(dev)
    sl = torch.from_numpy(w.slot).to(dev)
    n_rot = n_conf * n_q
    e = torch.empty(n_rot, device=dev)
    i = torch.empty(n_rot, 3, dtype=torch.int32, device=dev)
    out = {}
    with Receptor(w.grids, w.spacing, wave_rotations=args.wave, col_tile=args.col_tile,
                  profile=True) as rec:
        for it in range(2):
            rec.search_device(w.coor.shape[1], n_conf, coor.data_ptr(), ch.data_ptr(),
                              ep.data_ptr(), sl.data_ptr(), n_q, q.data_ptr(), e.data_ptr(),
                              i.data_ptr(), 0)
        out = rec.stats()
    out["rotations_per_s"] = n_rot / (out["device_ms"] / 1e3)
    print(json.dumps({"profile_run": n_rot, **out}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--wave", type=int, default=0)
    ap.add_argument("--col-tile", type=int, default=0)
    ap.add_argument("--graphs", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--ref-cufft", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--roofline-json", default="")
    ap.add_argument("--profile-run", type=int, default=0,
                    help="run one search of this many rotations with per-kernel events and "
                         "print the timings (the small case used for ncu captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile_run:
        profile_run(args)
        return
    import torch
    import torch.distributed as dist
    import datetime
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
