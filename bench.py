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


def _tensor_peak():
    """Dense BF16 TFLOP/s: the sustained measured figure (the x pass runs inside a long
    step), else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured (sustained)"
    return 1400.0, "fallback (sustained)"


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


def cpu_leg(w, args, outputs: dict, centers) -> tuple:
    """The CPU leg of the bench line: the timed CPU baseline and, as the checker of the GPU
    results, the oracle's FP64 energies of a sample of the timed rotations (per form) and the
    oracle's conformer selection (same centres required)."""
    from oracle import oracle as O
    base = None if args.no_cpu_baseline else cpu_baseline(w, budget_s=args.cpu_budget)
    acc = {}
    if not args.no_check:
        for name, (e, i) in outputs.items():
            acc[name] = _accuracy_sample(w, e, i)
    clus = None
    if centers is not None:
        x, en, cutoff, max_centers = centers["inputs"]
        t0 = time.perf_counter()
        want = O.cluster_conformers(x, en, cutoff, max_centers)
        clus = {"cpu_oracle_ms": round(1e3 * (time.perf_counter() - t0), 1),
                "identical_to_oracle": bool(np.array_equal(centers["got"], want)),
                "cpu_threads": 1}
    return base, acc, clus


def clustering_sample(n_conf: int = 1000, n_atoms: int = 40, max_centers: int = 100) -> dict:
    """Conformer selection (the greedy leader clustering of GeneDiverseConformations) on the
    GPU for n_conf random-rotor conformers; the CPU leg checks the centres."""
    import torch
    from cdocker_b200 import conformers, synth
    x, e = synth.conformer_ensemble(17, n_atoms=n_atoms, n_conf=n_conf, n_rotors=6)
    conformers.cluster_conformers(x, e, 1.5, max_centers)  # first call: module load, launch
    torch.cuda.synchronize()
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        got = conformers.cluster_conformers(x, e, 1.5, max_centers)
    t_gpu = (time.perf_counter() - t0) / reps
    return {"conformers": n_conf, "atoms": n_atoms, "centers": int(len(got)),
            "gpu_ms": round(t_gpu * 1e3, 3),
            "note": "host call: H2D of coordinates, pair-RMSD and greedy kernels, D2H of centres",
            "_check": {"inputs": (x, e, 1.5, max_centers), "got": got}}


def pose_agreement(w, forms: dict, tol: float = 1e-3) -> dict:
    """Best translation of every rotation of the timed step: each tensor-core form against the
    FP32 form (3e-7 from FP64 on the checked sample). Where they differ, both poses are
    re-scored in FP64 on the GPU (direct trilinear grid-energy sum): a difference within `tol`
    relative is a near-tie, anything else a real mismatch."""
    if "fp32" not in forms:
        return {}
    ref_e, ref_i = forms["fp32"]["e"], forms["fp32"]["i"]
    rec = forms["fp32"]["rec"]
    q = w.quats.reshape(-1, 4)
    n_q = w.quats.shape[1]
    out = {}
    for name, v in forms.items():
        if name == "fp32":
            continue
        e, i = v["e"], v["i"]
        valid = np.isfinite(ref_e)
        same = np.all(i == ref_i, axis=1) & valid
        mism = np.nonzero(valid & ~same)[0]
        near = worse = 0
        if mism.size:
            rc = (mism // n_q).astype(np.int32)
            e_t = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, rc, q[mism], i[mism])
            e_r = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, rc, q[mism], ref_i[mism])
            bar = tol * np.maximum(1.0, np.abs(e_r))
            near = int(np.sum(np.abs(e_t - e_r) <= bar))
            worse = int(np.sum(e_t - e_r > bar))
        nv = int(valid.sum())
        out[name] = {"rotations": nv, "identical": int(same.sum()),
                     "identical_frac": float(same.sum()) / max(1, nv),
                     "differ_near_tie": near, "differ_worse_in_fp64": worse,
                     "differ_better_in_fp64": int(mism.size - near - worse),
                     "identical_or_near_tie_frac": float(same.sum() + near) / max(1, nv),
                     "tie_tolerance": tol}
    return out


def receptor_grids_sample(n: int = 64, n_atoms: int = 2500, box: float = 32.0) -> dict:
    """Receptor grid generation for the benchmark receptor's size (8 probe radii + elec): the
    GPU call against the multithreaded host generator it must match bit for bit."""
    import os as _os

    from cdocker_b200 import api, synth
    rng = np.random.default_rng(11)
    xyz = rng.uniform(0.0, box, size=(n_atoms, 3)).astype(np.float32)
    rad = rng.uniform(1.5, 2.0, n_atoms).astype(np.float32)
    se = np.sqrt(rng.uniform(0.05, 0.2, n_atoms)).astype(np.float32)
    q = rng.normal(0.0, 0.3, n_atoms).astype(np.float32)
    origin = np.full(3, box / 2 - (n - 1) * 0.25, np.float32)
    args = (n, 0.5, origin, xyz, rad, se, q, synth.PROBE_RADII)
    api.synth_receptor_grids(*args, device=0)  # first call: module load
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        dev = api.synth_receptor_grids(*args, device=0)
    t_gpu = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    host = api.synth_receptor_grids(*args)
    t_host = time.perf_counter() - t0
    return {"n": n, "receptor_atoms": n_atoms, "grids": int(dev.shape[0]),
            "gpu_ms": round(t_gpu * 1e3, 3), "host_ms": round(t_host * 1e3, 3),
            "host_threads": _os.cpu_count(),
            "bit_identical": bool(np.array_equal(dev.view(np.uint32), host.view(np.uint32))),
            "note": "host call each: H2D of atoms, one kernel, D2H of the grids"}


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


class _RefWorkload:
    """The benchmark workload's conformer 0 built by the oracle (oracle.reference_inputs): the
    same grids, ligand, quaternions and slots as make_rank_workload, without loading the
    product library, so that the reference arm runs no code of this repository's product."""

    def __init__(self, n_q):
        from oracle import oracle as O
        d = O.reference_inputs(WORKLOAD, seed=0, n_conf=1, n_q=n_q)
        for k, v in d.items():
            setattr(self, k, v)
        self.w_n = d["n"]


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O
    w = _RefWorkload(N_Q)
    w.n = w.w_n
    cores = os.cpu_count() or 1
    q = w.quats.reshape(-1, 4)
    per_step = cores
    step_times = []
    total = args.warmup + args.steps
    for s in range(total):
        qs = q[(s * per_step) % q.shape[0]:][:per_step]
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
                   "grid": 64, "K": 9, "ligand_atoms": 40,
                   "inputs": f"built by the oracle ({w.source}); no product library loaded"},
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} rotations per step, cpuNaive dense loop "
                                   "(src/cpuNaive.cpp:82-216) restated in oracle/, "
                                   f"{cores} threads"},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if args.ref_cufft:
        # beside it, the reference's own GPU path (cuFFT, host fill and argmin, PCIe copies)
        try:
            line["reference_cufft"] = reference_cufft_sample(w)
        except Exception as ex:  # no GPU or harness not built: say so, keep the CPU line
            line["reference_cufft"] = {"unavailable": str(ex)[:200]}
    print(json.dumps(line), flush=True)


TENSOR_STEP_FLOP = 3 * 2 * 128 * 128 * 16  # one K-step of the streamed-tile x pass: 3 BF16 MMAs
# split-FP16 form: 2 FP16 MMAs per K-step and FP16 ligand rows (half the bytes of split BF16)
TENSOR_STEP_FLOP_FP16 = 2 * 2 * 128 * 128 * 16
MMA_UNIT_FLOP = 2 * 128 * 8 * 16  # Hankel x pass work counter unit: 128 x 8 x 16 multiply-adds


def FORMS(fp32, bf16x3, fp16x2):
    """(name, form) of the three search forms, in bench order."""
    return (("fp32", fp32), ("bf16x3_tensor_core", bf16x3), ("fp16x2_tensor_core", fp16x2))


def _kernel_roofline(stats: dict, n: int, K: int, hbm: float, peak_kind: str, traffic: dict):
    """Roofline of the dominant kernel of the last search, from the library's exact work
    counters over its average launch time (events in the timed region).

    HBM view: algorithmic bytes = the ligand planes it reads (x planes spread), the window
    planes it writes, and per wave the receptor data it needs (FP32 x pass: the K receptor
    spectra; Hankel tensor-core x pass: P~ of every column, K x n complex, from which each CTA
    builds its resident operator; streamed-tile x pass: the operator tiles of the box's K-steps).
    Tensor view (tensor-core x pass): the MMA flops it issued over the measured dense BF16 peak.
    The issued flops include the split products and the dense circulant (more than the FFT's
    algorithmic flops), so the HBM view is the bound reported for the path."""
    ncol = n * (n // 2 + 1)
    waves = max(1, stats["waves"])
    km = stats["kernel_ms"]
    dom = max(km, key=km.get)
    plane = ncol * 8
    rot = stats["rotations"]
    kind = stats.get("xpass_kind")
    fp16 = kind in ("tcgen05_streamed_fp16", "tcgen05_hankel_fp16")
    hankel = kind in ("tcgen05_hankel", "tcgen05_hankel_fp16")
    tiles = kind in ("tcgen05_streamed", "tcgen05_streamed_fp16")
    lig = plane // 2 if fp16 else plane  # ligand bytes per plane: FP16 rows, split BF16 or FP32
    jc = (stats["box"] + 7) // 8
    receptor = (K * ncol * n * 8 if hankel else
                K * ncol * 2 * jc * 4096 if tiles else K * n * plane)
    alg = {
        "xpass": stats["planes_spread"] * lig + stats["planes_window"] * plane + waves * receptor,
        "spread_yz": stats["planes_spread"] * lig,
        "yz_inv_argmin": stats["planes_window"] * plane,
        "prep": rot * 1024,
        "finalize": rot * 32,
    }
    per_launch = alg[dom] / waves
    t = km[dom] / waves / 1e3
    achieved = per_launch / t / 1e9
    tr = traffic.get(dom)
    out = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
           "frac": achieved / hbm, "peak_kind": peak_kind,
           "traffic": (tr * rot / waves) if tr is not None else None,
           "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": t * 1e3,
           "share_of_device_time": km[dom] / max(1e-9, sum(km.values())), "kernel_ms": km}
    if dom == "xpass" and (hankel or tiles):
        tp, tkind = _tensor_peak()
        if hankel:
            flop = stats.get("mma_units", 0) * MMA_UNIT_FLOP / waves
        else:
            flop = stats["tensor_steps"] * (TENSOR_STEP_FLOP_FP16 if fp16 else TENSOR_STEP_FLOP) / waves
        tach = flop / t / 1e12
        out["tensor_view"] = {"achieved": tach, "peak": tp, "unit": "TFLOP/s", "frac": tach / tp,
                              "peak_kind": tkind, "flop_per_launch": flop,
                              "note": "issued MMA flops (split products, dense circulant)"}
    return out


def all_rotation_fp64_error(rec, w, e, i, n_q):
    """Error of every rotation's returned minimum against the FP64 energy of the same pose: the
    FP64 direct trilinear grid-energy sum on the GPU (cdk_rescore_fp64) of each rotation at its
    returned translation; |E - E64| / max(|E64|, 1) over all rotations with a window."""
    valid = np.isfinite(e)
    idx = np.nonzero(valid)[0]
    q = w.quats.reshape(-1, 4)
    e64 = np.full(e.shape[0], np.nan)
    step = 250_000
    for b in range(0, idx.size, step):
        sel = idx[b:b + step]
        e64[sel] = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, (sel // n_q).astype(np.int32),
                                    q[sel], i[sel])
    err = np.abs(e[valid].astype(np.float64) - e64[valid]) / np.maximum(np.abs(e64[valid]), 1.0)
    return {"rotations": int(valid.sum()), "max_rel_err_vs_fp64": float(err.max()) if err.size else None,
            "median_rel_err_vs_fp64": float(np.median(err)) if err.size else None,
            "p999_rel_err_vs_fp64": float(np.quantile(err, 0.999)) if err.size else None,
            "note": "every rotation: returned minimum vs the FP64 energy of its returned pose"}


def _accuracy_sample(w, e, i, n_sample=24):
    """Per-rotation errors of a sample of the timed results against the FP64 oracle."""
    from oracle import oracle as O
    from tests.parity import rel_err
    n_rot = e.shape[0]
    sel = np.linspace(0, n_rot - 1, n_sample).astype(int)
    q = w.quats.reshape(-1, 4)
    r64 = np.empty(len(sel))
    ri = np.empty((len(sel), 3), np.int32)
    for j, r in enumerate(sel):
        _, ii, m = O.search_direct(w.grids, w.spacing, w.coor[r // N_Q], w.charge, w.eps, w.slot,
                                   q[r][None, None], prec=1)
        r64[j], ri[j] = m[0], ii[0]
    err = rel_err(e[sel], r64)
    return {"rotations_checked": int(len(sel)), "max_rel_err_vs_fp64": float(err.max()),
            "median_rel_err_vs_fp64": float(np.median(err)),
            "best_translation_agreement": float(np.mean(np.all(i[sel] == ri, axis=1)))}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, CDK_FORM_FP32, Receptor

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = make_rank_workload(rank, world)
    n_conf, n_atom = w.coor.shape[0], w.coor.shape[1]
    n_rot = n_conf * N_Q
    d_coor = torch.from_numpy(w.coor).to(dev)
    d_charge = torch.from_numpy(w.charge).to(dev)
    d_eps = torch.from_numpy(w.eps).to(dev)
    d_slot = torch.from_numpy(w.slot).to(dev)
    d_q = torch.from_numpy(w.quats).to(dev)
    d_e = torch.empty(n_rot, device=dev)
    d_i = torch.empty(n_rot, 3, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

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

    def timed_form(form):
        # config 1 as specified: searches captured into a CUDA graph (the warm-up steps autotune
        # the x pass, grow the scratch and capture; the timed steps replay) with the x-pass shape
        # picked by the autotuner
        rec = Receptor(w.grids, w.spacing, device=local_rank, wave_rotations=args.wave,
                       col_tile=args.col_tile, form=form, profile=True,
                       use_graphs=args.graphs, autotune=bool(args.autotune))

        def step():
            rec.search_device(n_atom, n_conf, d_coor.data_ptr(), d_charge.data_ptr(),
                              d_eps.data_ptr(), d_slot.data_ptr(), N_Q, d_q.data_ptr(),
                              d_e.data_ptr(), d_i.data_ptr(), stream.cuda_stream)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier()
        sampler = ClockSampler(local_rank)
        sampler.start()
        time.sleep(0.3)
        for s in range(args.steps):
            with torch.cuda.stream(stream):
                evs[s][0].record(stream)
                step()
                evs[s][1].record(stream)
                flush.fill_(s & 0xff)
        barrier()
        clocks = sampler.stop()
        ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs))
        stats = rec.stats()
        e = d_e.cpu().numpy()
        i = d_i.cpu().numpy()
        return rec, ms, stats, clocks, e, i

    forms = {}
    for name, form in FORMS(CDK_FORM_FP32, CDK_FORM_BF16X3, CDK_FORM_FP16X2):
        if args.forms not in ("both", "all") and args.forms != name:
            continue
        rec, ms, stats, clocks, e, i = timed_form(form)
        forms[name] = {"rec": rec, "ms": ms, "stats": stats, "clocks": clocks, "acc": None,
                       "e": e, "i": i, "value": world * n_rot * args.steps / (ms / 1e3)}
        # checker, outside the timed region: every rotation's minimum against the FP64 energy
        # of its returned pose
        forms[name]["fp64_all"] = (all_rotation_fp64_error(rec, w, e, i, N_Q)
                                   if rank == 0 and not args.no_check else None)
    clustering = clustering_sample() if rank == 0 else None
    grids_gen = receptor_grids_sample() if rank == 0 else None
    cpu_base, clus_check = None, None
    if rank == 0:
        base, acc, clus_check = cpu_leg(w, args, {k: (v["e"], v["i"]) for k, v in forms.items()},
                                        clustering.pop("_check") if clustering else None)
        cpu_base = base
        for k, v in acc.items():
            forms[k]["acc"] = v
    agreement = pose_agreement(w, forms) if rank == 0 else None
    # headline: the fastest form that meets its error bar on the checked sample (24 rotations
    # against the full FP64 search) and on every rotation (minimum vs FP64 of its pose)
    bars = {"fp32": 1e-4, "bf16x3_tensor_core": 1e-3, "fp16x2_tensor_core": 1e-3}
    ok = [k for k, v in forms.items()
          if (v["acc"] is None or v["acc"]["max_rel_err_vs_fp64"] <= bars[k]) and
          (v["fp64_all"] is None or v["fp64_all"]["max_rel_err_vs_fp64"] <= bars[k])]
    head = max(ok or list(forms), key=lambda k: forms[k]["value"])
    if world > 1:
        # only rank 0 checked accuracy: every rank times the e2e leg on rank 0's choice
        names = list(forms)
        t = torch.tensor([names.index(head)], dtype=torch.int64, device=dev)
        dist.broadcast(t, src=0)
        head = names[int(t.item())]
    H = forms[head]
    rec = H["rec"]

    # e2e through cdk_search with pinned host buffers, copies inside the timed region
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

    serving = None
    if rank == 0 and args.serve_secs > 0:
        serving = serving_sample(w, rec, args.serve_secs)

    if rank == 0:
        hbm, peak_kind = _peaks()
        nc = 64 * 64 * 33  # half-spectrum points of one grid
        b_rot = 8 * 9 * 64 ** 3 + 16 * 9 * nc + 16 * nc + 8 * 64 ** 3
        traffic = {}
        tp = os.path.join(ROOT, "profiles", "dram_bytes_per_rotation.json")
        if os.path.exists(tp):
            with open(tp) as f:
                traffic = json.load(f).get(head, {})
        dram_rot = sum(v for v in traffic.values() if isinstance(v, (int, float))) if traffic else None
        value = H["value"]
        rps = value / world
        line = {
            "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": H["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp32": "f32", "bf16x3_tensor_core": "bf16x3 (f32 accumulate)",
                      "fp16x2_tensor_core": "fp16x2 (f32 accumulate)"}.get(head, head),
            "data": "synthetic",
            "config": {"workload": "config 1: 64^3 grid at 0.5 A, K=9, 2,500-atom synthetic "
                                   "receptor, 40-atom ligand, 100 conformers x 1,000 "
                                   "quaternions = 1e5 rotations per rank per step",
                       "form": head, "grid": 64, "K": 9, "rotations_per_step": n_rot * world,
                       "l2": "256 MiB written between timed steps (and every step's wave "
                             "scratch is GBs, far above L2)",
                       "wave_rotations": H["stats"]["wave_rotations"],
                       "cuda_graph": H["stats"]["graph_state"] == 2,
                       "autotuned_xpass": {"kind": H["stats"]["xpass_kind"],
                                           "columns_per_cta": H["stats"]["col_tile"]},
                       "parallelism": f"rotation shards x{world}"},
            "gpu_launches": int(H["stats"]["launches"] * args.steps),
            "clocks": H["clocks"],
            "e2e": {"value": e2e_val, "unit": "rotations/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "form": head},
            "roofline": _kernel_roofline(H["stats"], 64, 9, hbm, peak_kind, traffic),
            "staged_equivalent": {
                "bytes_per_rotation": b_rot, "equivalent_gbs": rps * b_rot / 1e9,
                "note": "not a roofline: the bytes a staged cuFFT pipeline would move per "
                        "rotation (B_rot = 8KN + 16K*Nc + 16Nc + 8N, Nc = n*n*(n/2+1)) times the "
                        "rotation rate; the fused path moves far fewer bytes"},
            "step_dram": {
                "bytes_per_rotation": dram_rot,
                "achieved_gbs": rps * dram_rot / 1e9 if dram_rot else None, "peak_gbs": hbm,
                "frac": rps * dram_rot / 1e9 / hbm if dram_rot else None, "peak_kind": peak_kind,
                "note": "DRAM bytes per rotation of all kernels of the step (ncu, "
                        "profiles/dram_bytes_per_rotation.json) times the rotation rate"},
            "forms": {k: {"value": v["value"], "ms_per_step": v["ms"] / args.steps,
                          "accuracy": v["acc"], "all_rotations_vs_fp64": v["fp64_all"],
                          "xpass_kind": v["stats"]["xpass_kind"],
                          "kernel_ms_last_step": v["stats"]["kernel_ms"]}
                      for k, v in forms.items()},
        }
        if serving is not None:
            line["serving"] = serving
        if clustering is not None:
            if clus_check:
                clustering.update(clus_check)
            line["clustering"] = clustering
        if grids_gen is not None:
            line["receptor_grids"] = grids_gen
        if agreement is not None:
            line["best_pose_agreement"] = agreement
        if cpu_base is not None:
            line["cpu_baseline"] = cpu_base
        print(json.dumps(line), flush=True)
    for v in forms.values():
        v["rec"].close()


def serving_sample(w, rec_unused, secs: float) -> dict:
    """Continuous-batching server on the same 64^3 receptor (all 8 vdW grids + elec): Poisson
    arrivals of requests with ligands of 10-80 atoms, 10-50 conformers, 500-2,000 rotations,
    served by each form (the precision form runs its waves on the streamed tensor-core x
    pass; `tc_waves` counts them)."""
    from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, CDK_FORM_FP32, Receptor, synth
    from cdocker_b200.serving import Server, make_requests, poisson_arrivals, run_load
    rate = 40.0
    arr = poisson_arrivals(rate, secs, seed=7)
    reqs = make_requests(len(arr), 21, w.spacing, w.length, synth.PROBE_RADII, atoms=(10, 80),
                         confs=(10, 50), rots=(500, 2000))
    out = {}
    for name, form in FORMS(CDK_FORM_FP32, CDK_FORM_BF16X3, CDK_FORM_FP16X2):
        with Receptor(w.all_grids, w.spacing, max_atoms=96, form=form) as r:
            with Server(r, arena_bytes=512 << 20, wave_rotations=1024, max_atoms=96) as srv:
                res = run_load(srv, reqs, arr)
                st = srv.stats()
        res.update({"rate_hz": rate, "grid": 64, "waves": st["waves"], "tc_waves": st["tc_waves"],
                    "request_mix": "ligand U(10,80) atoms, conformers U(10,50), rotations "
                                   "U(500,2000), Poisson arrivals"})
        out[name] = res
    return out


def serve_sweep(args):
    """Config 3: one resident 96^3 receptor (6,000 atoms in a 48 A cube, all 9 grids: 8 vdW +
    elec), requests with ligands of 10-80 atoms, 10-200 conformers and 500-5,000 rotations,
    Poisson arrivals; every form. Per form, a burst of requests submitted at once measures the
    server's capacity (rotations/s); then five Poisson rates at 0.25, 0.5, 0.75, 0.9 and 1.1 of
    that capacity (the top one saturates the device), each for --serve-secs of arrivals. Prints
    one JSON line per (form, rate) and a summary line (not the bench line)."""
    from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, CDK_FORM_FP32, Receptor, synth
    from cdocker_b200.serving import Server, make_requests, poisson_arrivals, run_load
    grids, mid, length = synth.make_receptor(96, 6000, 48.0, seed=0)
    secs = max(2.0, args.serve_secs)
    mix = dict(atoms=(10, 80), confs=(10, 200), rots=(500, 5000))
    burst = make_requests(24, 999, 0.5, length, synth.PROBE_RADII, **mix)
    summary = {}
    for form_name, form in FORMS(CDK_FORM_FP32, CDK_FORM_BF16X3, CDK_FORM_FP16X2):
        if args.forms not in ("both", "all") and args.forms != form_name:
            continue
        with Receptor(grids, 0.5, max_atoms=96, form=form) as rec:
            srv_kw = dict(arena_bytes=2 << 30, wave_rotations=1024, max_atoms=96, max_box=40)
            with Server(rec, **srv_kw) as srv:
                run_load(srv, burst[:4], np.zeros(4))  # warm-up: module load, scratch first touch
                cap = run_load(srv, burst, np.zeros(len(burst)))
                st = srv.stats()
            capacity = cap["rotations"] / cap["wall_s"]
            mean_rot = float(np.mean([r["rotations"] for r in burst]))
            lines = []
            for frac in (0.25, 0.5, 0.75, 0.9, 1.1):
                rate = frac * capacity / mean_rot
                arr = poisson_arrivals(rate, secs, seed=int(frac * 100))
                reqs = make_requests(len(arr), int(frac * 1000) + 7, 0.5, length, synth.PROBE_RADII, **mix)
                with Server(rec, **srv_kw) as srv:
                    res = run_load(srv, reqs, arr)
                    st = srv.stats()
                res.update({"config": "serving, 96^3 K=9, 6,000-atom receptor", "form": form_name,
                            "rate_hz": rate, "load_frac_of_capacity": frac,
                            "offered_rotations_per_s": rate * mean_rot,
                            "waves": st["waves"], "tc_waves": st["tc_waves"],
                            "request_mix": "ligand U(10,80) atoms, conformers U(10,200), rotations "
                                           "U(500,5000), Poisson arrivals"})
                print(json.dumps(res), flush=True)
                lines.append({k: res[k] for k in ("rate_hz", "load_frac_of_capacity", "p50_ms",
                                                  "p99_ms", "rotations_per_s", "requests")})
            summary[form_name] = {"capacity_rotations_per_s": capacity,
                                  "capacity_tc_waves": st["tc_waves"], "rates": lines}
    print(json.dumps({"serve_sweep": "config 3", "grid": 96, "forms": summary}), flush=True)


def config4_run(args):
    """Config 4, the largest single search: 128^3 grid at 0.5 A, K = 9 (8 vdW + elec) from a
    12,000-atom synthetic receptor in a 64 A cube; a 60-atom ligand, 500 conformers x 2,000
    uniform quaternions = 1e6 rotations, streamed in memory-sized waves. Each form (FP32,
    split-BF16, split-FP16) runs one untimed warm-up search of the first 20 conformers, then the
    whole search timed on the device (CUDA events on the search stream) with clocks sampled, and
    the whole search again through cdk_search with host buffers (e2e). The checker then gives
    the error of every rotation's minimum against the FP64 energy of its returned pose, and the
    FP64 oracle's full search of 16 rotations (minimum and argmin). Prints one JSON line."""
    import torch
    from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, CDK_FORM_FP32, Receptor, synth
    from oracle import oracle as O
    from tests.parity import rel_err
    n_conf, n_q = args.c4_conformers, args.c4_quaternions
    t0 = time.perf_counter()
    w = synth.make_workload("c4_128", seed=0, n_conf=n_conf, n_q=n_q)
    t_inputs = time.perf_counter() - t0
    dev = torch.device("cuda", 0)
    n_atom, n_rot = w.coor.shape[1], n_conf * n_q
    d_coor = torch.from_numpy(w.coor).to(dev)
    d_charge = torch.from_numpy(w.charge).to(dev)
    d_eps = torch.from_numpy(w.eps).to(dev)
    d_slot = torch.from_numpy(w.slot).to(dev)
    d_q = torch.from_numpy(w.quats).to(dev)
    d_e = torch.empty(n_rot, device=dev)
    d_i = torch.empty(n_rot, 3, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sample = np.linspace(0, n_rot - 1, 16).astype(int)
    qq = w.quats.reshape(-1, 4)
    r64 = np.empty(sample.size)
    ri = np.empty((sample.size, 3), np.int32)
    for j, r in enumerate(sample):
        _, ii, m = O.search_direct(w.grids, w.spacing, w.coor[r // n_q], w.charge, w.eps, w.slot,
                                   qq[r][None, None], prec=1)
        r64[j], ri[j] = m[0], ii[0]
    hbm, peak_kind = _peaks()
    out = {}
    for name, form in FORMS(CDK_FORM_FP32, CDK_FORM_BF16X3, CDK_FORM_FP16X2):
        if args.forms not in ("both", "all") and args.forms != name:
            continue
        with Receptor(w.grids, w.spacing, form=form, profile=True) as rec:
            warm = min(n_conf, 20)
            rec.search_device(n_atom, warm, d_coor.data_ptr(), d_charge.data_ptr(), d_eps.data_ptr(),
                              d_slot.data_ptr(), n_q, d_q.data_ptr(), d_e.data_ptr(), d_i.data_ptr(),
                              stream.cuda_stream)
            torch.cuda.synchronize(dev)
            sampler = ClockSampler(0)
            sampler.start()
            time.sleep(0.3)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                ev0.record(stream)
                rec.search_device(n_atom, n_conf, d_coor.data_ptr(), d_charge.data_ptr(),
                                  d_eps.data_ptr(), d_slot.data_ptr(), n_q, d_q.data_ptr(),
                                  d_e.data_ptr(), d_i.data_ptr(), stream.cuda_stream)
                ev1.record(stream)
            torch.cuda.synchronize(dev)
            clocks = sampler.stop()
            ms = ev0.elapsed_time(ev1)
            st = rec.stats()
            e, i = d_e.cpu().numpy(), d_i.cpu().numpy()
            # e2e: host buffers through cdk_search, copies inside the timing
            t1 = time.perf_counter()
            e2, i2 = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            e2e_s = time.perf_counter() - t1
            same = bool(np.array_equal(e2.view(np.uint32), e.view(np.uint32)) and np.array_equal(i2, i))
            allrot = all_rotation_fp64_error(rec, w, e, i, n_q)
            err = rel_err(e[sample], r64)
            rl = _kernel_roofline(st, 128, w.K, hbm, peak_kind, {})
        out[name] = {
            "rotations_per_s": n_rot / (ms / 1e3), "device_ms": ms,
            "e2e_rotations_per_s": n_rot / e2e_s, "e2e_identical_to_device_run": same,
            "xpass_kind": st["xpass_kind"], "waves": st["waves"], "wave_rotations": st["wave_rotations"],
            "box_planes": st["box"], "kernel_ms": st["kernel_ms"], "clocks": clocks,
            "all_rotations_vs_fp64": allrot,
            "fp64_full_search_sample": {"rotations": int(sample.size),
                                        "max_rel_err": float(err.max()),
                                        "median_rel_err": float(np.median(err)),
                                        "best_translation_agreement": float(np.mean(np.all(i[sample] == ri, axis=1)))},
            "dominant_kernel_roofline": rl,
        }
        print(json.dumps({"config4_form": name, **out[name]}), flush=True)
    line = {"config": "config 4: 128^3 grid at 0.5 A, K=9, 12,000-atom synthetic receptor, 60-atom "
                      f"ligand, {n_conf} conformers x {n_q} quaternions = {n_rot} rotations, streamed",
            "unit": "rotations/s", "data": "synthetic", "input_build_s": round(t_inputs, 1),
            "forms": out}
    print(json.dumps(line), flush=True)


def profile_run(args):
    """One warm-up and one timed search of `--profile-run` rotations (first conformers of the
    config-1 workload, or of the config-4 workload with --profile-config c4_128), per-kernel
    device times from events around every launch."""
    import torch
    from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, CDK_FORM_FP32, Receptor, synth
    if args.profile_config == "c4_128":
        w = synth.make_workload("c4_128", seed=0, n_conf=max(1, (args.profile_run + 1999) // 2000),
                                n_q=min(2000, args.profile_run))
        n_q = w.quats.shape[1]
        n_conf = w.quats.shape[0]
    else:
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
    form = {"bf16x3_tensor_core": CDK_FORM_BF16X3,
            "fp16x2_tensor_core": CDK_FORM_FP16X2}.get(args.forms, CDK_FORM_FP32)
    with Receptor(w.grids, w.spacing, wave_rotations=args.wave, col_tile=args.col_tile,
                  profile=True, form=form) as rec:
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
    ap.add_argument("--graphs", type=int, default=1,
                    help="1: capture each search into a CUDA graph and replay it (default)")
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: autotune the x pass on the first search (default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--ref-cufft", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--forms", default="all",
                    choices=["all", "both", "fp32", "bf16x3_tensor_core", "fp16x2_tensor_core"])
    ap.add_argument("--serve-secs", type=float, default=3.0)
    ap.add_argument("--serve-sweep", action="store_true",
                    help="config 3: 96^3 receptor, Poisson request streams at 5 rates; one JSON "
                         "line per rate (not the bench line)")
    ap.add_argument("--profile-config", default="c1_64", choices=["c1_64", "c4_128"])
    ap.add_argument("--config4", action="store_true",
                    help="config 4: 128^3, 1e6 rotations, all forms, error vs FP64 on every "
                         "rotation; one JSON line (not the bench line)")
    ap.add_argument("--c4-conformers", type=int, default=500)
    ap.add_argument("--c4-quaternions", type=int, default=2000)
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
    if args.serve_sweep:
        serve_sweep(args)
        return
    if args.config4:
        config4_run(args)
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
