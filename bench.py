"""Benchmark of the SOD stage: halos/s on a synthetic clustered box.

A step is one pass of the hot path over one box: the cell sort of the
particles (the reference's linked list), CIC density, seed order and the SOD
(spherover) through psod_run.  ``value`` is whole-job halos/s with the
particles already in HBM; ``e2e`` is the same through the C-ABI from pinned
host buffers, with the host-to-device copy of the particles and the
device-to-host copy of the halo table inside the timed region.

The default mode is the learned bracket: before anything is timed, the
bracket network is trained on samples from 128^3 boxes with the engine's GPU
training kernels; the timed steps include its per-round inference.  The same
box then runs once in the batched mode (no network) and once in the plain
mode for comparison.

One process per GPU (torchrun for N > 1).  The SOD of one box does not
shard, so every rank runs an independent replica on its own box (weak
scaling); the ranks only meet at a barrier and a max-reduction of the
timings.

``--impl reference`` times the reference algorithm on the host cores: the
CPU oracle (a C restatement of the Fortran, reference arithmetic) on a
bounded sample of the workload, one sample box per core.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# synthetic workloads: the reference's box sizes with the NFW-mixture generator
WORKLOADS = {
    128: dict(nmax_halo=20000, box="128^3, 82.03125 Mpc/h, halo N in [20, 2e4]"),
    256: dict(nmax_halo=50000, box="256^3, halo N in [20, 5e4]"),
    512: dict(nmax_halo=200000, box="512^3, 656.25 Mpc/h, halo N in [20, 2e5]"),
    1024: dict(nmax_halo=1000000, box="1024^3, 1312.5 Mpc/h, halo N in [20, 1e6]"),
}
# the heavy-tail stress box: the 1024^3 law plus 16 clusters of 5e6 particles
# (NFW c = 4, axis ratios 1:0.8:0.6), -npu 1e7, Delta 200 and 500, 64 bins
HEAVY = dict(nx=1024, nmax_halo=1000000, n_clusters=16, cluster_size=5_000_000, npu=10_000_000,
             delta_extra=(500.0,), nbins=64,
             box="1024^3 + 16 clusters of 5e6 (c=4, axes 1:0.8:0.6), halo N in [20, 1e6], Delta 200/500, 64 bins")


# the 1024^3 workload computes three thresholds in one pass, with 48 bins
EXTRA_DELTAS = (500.0, 178.0)
EXTRA_BINS = 48

METRIC = "SOD halos/s (delta=200, N200 exact)"


def npu_for(nx):
    return {128: 0, 256: 0, 512: 200000, 1024: 1000000}.get(nx, 0)


def inputs_fit_l2(nx):
    """True when one box's positions and IDs (20 B a particle) would stay in
    the 126 MB L2 between steps, so that the timed loop must flush it."""
    return nx**3 * (12 + 8) < (126 << 20) * 2


def workload_config(nx, ndelta, heavy=False):
    """The ``config`` object of both arms: the workload alone (no
    implementation or measurement keys), so the two lines name the same
    configuration."""
    if heavy:
        return {"workload": HEAVY["box"], "nx": HEAVY["nx"], "particles": HEAVY["nx"] ** 3, "npu": HEAVY["npu"],
                "delta": [200.0, 500.0], "nbins": HEAVY["nbins"], "l2": "inputs larger than L2"}
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    return {
        "workload": wl["box"],
        "nx": nx,
        "particles": nx**3,
        "npu": npu_for(nx),
        "delta": [200.0, 500.0, 178.0] if ndelta else [200.0],
        "nbins": EXTRA_BINS if ndelta else 60,
        "l2": "flushed between steps" if inputs_fit_l2(nx) else "inputs larger than L2",
    }


def table_digest(sod, members):
    """Checksum of the whole halo table, computed on the device: every field
    (IDs, masses, ranks, centres, radii, seuil2 and extra-delta masses,
    profiles, member offsets and member indices) mixed with its position."""
    import torch

    from psod_b200.sod import HaloTable

    h, m = sod.halo_count()
    nb, ne = sod.params.nbins, sod.params.ndelta_extra
    dev = f"cuda:{torch.cuda.current_device()}"
    sizes = dict(halo_id=h, halo_mass=h, halo_rank=h, halo_center=3 * h, halo_rdelta=h, halo_mass2=h,
                 halo_mextra=h * ne, halo_profile=h * nb, member_offset=h + 1, member_index=m, member_id=m)
    dt = dict(halo_center=torch.float32, halo_rdelta=torch.float64)
    out = HaloTable(**{f: torch.zeros(max(1, k), dtype=dt.get(f, torch.int64), device=dev) for f, k in sizes.items()})
    t = sod.halos(members=True, out=out)
    acc = 0
    for k, f in enumerate(("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2",
                           "halo_mextra", "halo_profile", "member_offset", "member_index", "member_id")):
        a = getattr(t, f).reshape(-1)
        if a.numel() == 0:
            continue
        x = a.view(torch.int32).to(torch.int64) if a.dtype == torch.float32 else a.view(torch.int64)
        i = torch.arange(x.numel(), dtype=torch.int64, device=dev)
        y = x * -7046029254386353131 + (i + 1) * -4658895280553007687 + k * 1442695040888963407
        y = y ^ (y >> 29)
        acc = (acc * 6364136223846793005 + int(y.sum().item()) + members) & ((1 << 64) - 1)
    del out
    return f"{h}:{m}:{acc:016x}"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=6)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].strip() == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup(backend: str | None = None):
    """World size, rank and local rank from the torchrun environment; for
    N > 1 a process group over NCCL (GPU) or gloo (CPU, host-side tests)."""
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        import datetime

        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def _reduce(x: float, world: int, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return _reduce(x, world, "max")


def combine_replicas(ms: float, nhalo: int, world: int) -> tuple[float, int]:
    """Whole-job time and halo count of N independent replicas: the slowest
    rank's time and the halos of all ranks (each rank runs its own box)."""
    return max_over_ranks(ms, world), int(round(_reduce(float(nhalo), world, "sum")))


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_ours(args):
    import numpy as np
    import torch

    from psod_b200 import synth
    from psod_b200.sod import HaloTable, SphericalOverdensity

    world, rank, local = dist_setup()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    nx = HEAVY["nx"] if args.heavy else args.nx
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    thresholds = dict(delta_extra=EXTRA_DELTAS, nbins=EXTRA_BINS) if args.ndelta else {}
    if args.heavy:
        thresholds = dict(delta_extra=HEAVY["delta_extra"], nbins=HEAVY["nbins"])
    model, bracket = None, None
    if args.mode == "learned":
        model, bracket = train_bracket(args, dev, thresholds)
    clusters = dict(n_clusters=HEAVY["n_clusters"], cluster_size=HEAVY["cluster_size"]) if args.heavy else {}
    box = synth.make_box(nx, nmax_halo=wl["nmax_halo"], seed=args.seed + rank, device=f"cuda:{dev}", **clusters)
    pos_d, ids_d = box.pos, box.ids
    del box
    torch.cuda.empty_cache()  # hand the generator's temporaries back before the engine allocates
    n = int(pos_d.shape[0])
    params = dict(npu=HEAVY["npu"] if args.heavy else npu_for(nx), mode=args.mode_id, **thresholds)
    sod = SphericalOverdensity(nx, device=dev, **params)
    if model is not None:
        sod.learn_set_features("fof")
        sod.learn_set_model(model)
        # the FoF catalogue the SOD stage starts from (the previous stage of
        # the reference's pipeline; untimed), then its working arrays freed
        sod.load(pos_d, ids_d)
        sod.fof(percolation=0.2, mmin=20)
        sod.fof_release()
    # L2 flush buffer (used when the inputs are smaller than L2)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    inputs_bytes = n * (12 + 8)
    need_flush = inputs_fit_l2(nx)

    def step_device():
        if need_flush:
            flush.zero_()
        sod.load(pos_d, ids_d)
        return sod.run()

    for _ in range(args.warmup):
        st = step_device()
    tuning = None
    if args.autotune and args.mode != "plain":
        # scheduling thresholds picked on this box (untimed; the table does
        # not depend on them)
        tuning = sod.autotune()
    else:
        tuning = sod.get_tuning()
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats_list = []
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            stats_list.append(step_device())
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    nhalo_rank = stats_list[-1]["nhalo"]
    ms, nhalo_all = combine_replicas(ms, nhalo_rank, world)
    stage_ms = time_stages(sod, pos_d, ids_d)

    # e2e: pinned host buffers through the C-ABI, copies inside the timed region
    pos_h = pos_d.cpu().pin_memory()
    ids_h = ids_d.cpu().pin_memory()
    t = sod.halos(members=True)
    # pinned host buffers for the halo table, reused every step
    tdt = {np.dtype(np.int64): torch.int64, np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}
    out = HaloTable(**{f: torch.empty(max(1, getattr(t, f).size), dtype=tdt[getattr(t, f).dtype], pin_memory=True)
                       for f in HaloTable.__dataclass_fields__})
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sod.load(pos_h, ids_h)
        sod.run()
        sod.halos(members=True, out=out)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    d2h = t.halo_id.nbytes + t.halo_mass.nbytes + t.halo_rank.nbytes + t.halo_center.nbytes + t.halo_rdelta.nbytes \
        + t.halo_mass2.nbytes + t.halo_mextra.nbytes + t.halo_profile.nbytes + t.member_offset.nbytes \
        + t.member_index.nbytes + t.member_id.nbytes

    s = stats_list[-1]
    peak, peak_kind = load_peaks()
    # Gather/distance kernel (k_cross and its warp form, the rounds the host
    # launches): HBM-bound.  Algorithmic bytes: 16 B per record of the cube
    # cells meeting each ball out to its stopping particle, plus 12 B per
    # member written (d2 key + index).  The device tail loop's crossings are
    # counted apart (they share a launch with the refinement).
    alg_bytes = 16.0 * (s["cross_touch"] - s["tail_touch"]) + 12.0 * s["cross_members"]
    cross_s = s["ms_cross"] / 1000.0
    achieved = alg_bytes / cross_s / 1e9 if cross_s > 0 else 0.0
    launches = max(1, s["rounds"])
    # DRAM bytes per launch: the ratio of DRAM traffic to algorithmic bytes
    # measured by ncu on the 256^3 box, applied to this workload's launches
    tr = load_traffic("k_cross")
    traffic = None
    if tr:
        traffic = {"bytes_per_launch": int(tr["dram_bytes_per_algorithmic_byte"] * alg_bytes / launches),
                   "dram_per_algorithmic_byte": tr["dram_bytes_per_algorithmic_byte"],
                   "from": "ncu DRAM capture at 256^3, scaled by algorithmic bytes"}
    value = nhalo_all / (ms / 1000.0)
    # the refinement kernel dominates: FP32 pair tests fed from shared memory
    ref_s = s["ms_refine"] / 1000.0
    pairs_per_s = s["refine_pairs"] / ref_s if ref_s > 0 else 0.0
    # issue ceiling of the pair test: 12 warp instructions per 32 pairs (one
    # shared load, 3 FADD + 3 FFMA for d2 + eps^2, edge FADD + FMNMX, FSETP,
    # MUFU.RSQ, predicated FADD), one instruction per clock per sub-partition
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    props = torch.cuda.get_device_properties(dev)
    ceiling = props.multi_processor_count * 4 * sm_mhz * 1e6 * 32 / 12.0
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "halos/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic NFW-mixture box (seeded); inputs resident in HBM",
        "mode": args.mode,
        "parallelism": f"replicas x{world}",
        "config": workload_config(nx, args.ndelta, args.heavy),
        "detail": {
            "halos": nhalo_all,
            "members": s["nmember"],
            "seeds": s["npart_new"],
            "processed_seeds": s["nprocessed"],
            "rounds": s["rounds"],
            "stage_ms": {k: round(v, 2) for k, v in stage_ms.items()},
            "sod_phase_ms": {k: round(s[k], 2) for k in ("ms_setup", "ms_sched", "ms_prep", "ms_refine", "ms_select",
                                                         "ms_cross", "ms_tail", "ms_output")},
            "tail_rounds": s["tail_rounds"],
            "tuning": tuning,
        },
        "e2e": {
            "value": round(nhalo_all / (e2e_ms / 1000.0), 2),
            "unit": "halos/s",
            "h2d_bytes_per_step": int(n * (12 + 8)),
            "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(e2e_ms, 3),
        },
        "gpu_launches": int(s["kernel_launches"]) + 12,
        "roofline": {
            "bound": "hbm",
            "kernel": "k_cross (radial gather, distances, crossing, profile, claims)",
            "achieved": round(achieved, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind,
            "traffic": traffic,
            "launches": launches,
            "alg_bytes_per_launch": int(alg_bytes / launches),
            "kernel_ms": round(s["ms_cross"], 3),
        },
        "refine": {
            "kernel": "k_refine_warp (dominant by time: FP32/MUFU pair tests fed from shared memory)",
            "bound": "instruction issue (neither hbm nor tensor)",
            "pairs": int(s["refine_pairs"]),
            "pairs_per_s": round(pairs_per_s, 1),
            "issue_ceiling_pairs_per_s": round(ceiling, 1),
            "frac_of_issue_ceiling": round(pairs_per_s / ceiling, 4) if ceiling > 0 else None,
            "lane_utilization": round(s["refine_pairs"] / max(1, s["refine_slots"]), 4),
            "kernel_ms": round(s["ms_refine"], 3),
        },
        "clocks": clocks,
    }
    if bracket is not None:
        bracket.update(hit_rate=round(s["bracket_hits"] / max(1, s["bracket_seeds"]), 4),
                       fallback_rate=round(1.0 - s["bracket_hits"] / max(1, s["bracket_seeds"]), 4),
                       seeds=int(s["bracket_seeds"]), cross_balls=int(s["cross_balls"]),
                       cross_records=int(s["cross_records"]), ms_learn=round(s["ms_learn"], 2))
        line["bracket"] = bracket
    if args.compare_plain and args.mode != "plain" and world == 1:
        # the same box through the other modes: their tables must be
        # identical to this one (device checksums of every field)
        digests = {args.mode: table_digest(sod, 0)}
        if args.mode == "learned":
            line["batched"] = mode_reference(nx, params, pos_d, ids_d, sod, 1, tuning)
            line["vs_batched"] = round(line["batched"]["ms_per_step"] / ms, 3)
            digests["batched"] = line["batched"].pop("digest")
            sod = None
        line["plain"] = mode_reference(nx, params, pos_d, ids_d, sod, 0, tuning)
        line["vs_plain"] = round(line["plain"]["ms_per_step"] / ms, 3)
        digests["plain"] = line["plain"].pop("digest")
        sod = None
        line["modes_identical"] = len(set(digests.values())) == 1
        line["table_digests"] = digests
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args, nx, wl, cores=1, boxes_per_core=4 if nx > 128 else 1)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if sod is not None:
        sod.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def load_traffic(kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


def time_stages(sod, pos, ids):
    """Device time of each stage of one step (CUDA events, current stream)."""
    import torch

    out = {}
    for name, fn in (("load", lambda: sod.load(pos, ids)), ("cic", lambda: sod.cic()),
                     ("cicm1", lambda: sod.cicm1(want_rho=False)), ("tri_cic", lambda: sod.tri_cic(want_isort=False)),
                     ("spherover", lambda: sod.spherover())):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b)
    return out


def mode_reference(nx, params, pos_d, ids_d, sod, mode, tuning=None):
    """The same box through another GPU mode (0 plain: full-cube gathers; 1
    batched: growing balls from 1.5 cells, no network), one untimed and one
    timed step.  Closes ``sod`` first to free its memory."""
    import torch

    from psod_b200.sod import SphericalOverdensity

    if sod is not None:
        sod.close()
    torch.cuda.empty_cache()
    p = dict(params)
    p["mode"] = mode
    sp = SphericalOverdensity(nx, device=torch.cuda.current_device(), **p)
    if tuning:
        # the main run's scheduling thresholds, so that the modes compare
        # on the same settings
        sp.set_tuning(**{k: tuning[k] for k in ("warp_cross_min_ready", "bound_min_cand", "tail_max_ready",
                                                 "tail_max_cand")})
    sp.load(pos_d, ids_d)
    sp.run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    sp.load(pos_d, ids_d)
    st = sp.run()
    b.record()
    torch.cuda.synchronize()
    msp = a.elapsed_time(b)
    digest = table_digest(sp, 0)
    sp.close()
    out = {"mode": {0: "plain", 1: "batched"}[mode], "ms_per_step": round(msp, 3), "halos": st["nhalo"],
           "value": round(st["nhalo"] / (msp / 1000.0), 2), "unit": "halos/s",
           "sod_phase_ms": {k: round(st[k], 2) for k in ("ms_setup", "ms_sched", "ms_prep", "ms_refine", "ms_select",
                                                         "ms_cross", "ms_tail", "ms_output")}, "digest": digest,
           "tail_rounds": st["tail_rounds"]}
    if mode == 1:
        out.update(hit_rate=round(st["bracket_hits"] / max(1, st["bracket_seeds"]), 4),
                   cross_balls=int(st["cross_balls"]), cross_records=int(st["cross_records"]))
    return out


def train_bracket(args, dev, thresholds):
    """The learned bracket network, trained untimed on the engine's own
    samples from configuration-1 boxes (128^3, halo N in [20, 2e4]) with the
    GPU training kernels: Adam, lr 1e-3, 20 epochs, batch 4096."""
    import torch

    from psod_b200 import synth
    from psod_b200.sod import SphericalOverdensity

    nbox = 32
    t0 = time.perf_counter()
    with SphericalOverdensity(128, device=dev, mode=1, **thresholds) as s:
        # the FoF features of the learned-seed configuration: each box's
        # FoF catalogue (b = 0.2, 20 particles) before its SOD run
        s.learn_set_features("fof")
        s.learn_collect(1 << 21)
        for i in range(nbox):
            b = synth.make_box(128, nmax_halo=20000, seed=args.seed + 1000 + i, device=f"cuda:{dev}")
            s.load(b.pos, b.ids)
            s.fof(percolation=0.2, mmin=20)
            s.run()
            del b
        x, _ = s.learn_samples()
        loss = s.learn_train(epochs=20, batch=4096, lr=1e-3, seed=args.seed)
        model = s.learn_get_model()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return model, {"trained_on": f"{nbox} boxes of 128^3 (halo N in [20, 2e4]), batched-mode samples",
                   "features": "FoF group of the seed: log N_FoF, inertia axis ratios, log peak overdensity, "
                               "peak - centre-of-mass offset, R_FoF, RMS radius; targets log(R_stop/R_FoF), "
                               "centre offset",
                   "samples": int(x.shape[0]), "epochs": 20, "batch": 4096, "lr": 1e-3,
                   "loss_first_last": [round(float(loss[0]), 4), round(float(loss[-1]), 4)],
                   "train_s": round(time.perf_counter() - t0, 2)}


def sample_nx(nx):
    """Side of the CPU sample boxes: the workload itself up to 128^3 (the
    oracle runs a full 128^3 box in about 20 s on one core), else 48^3 boxes
    drawn with the workload's generator law (1-5 s each on one core, so that
    a step of one box per core stays bounded)."""
    return nx if nx <= 128 else 48


def _oracle_params(snx, npu, ndelta):
    """Oracle parameters of one sample box: the ones -npu derives
    (main:211-219) and the workload's thresholds and bins."""
    import math

    from oracle import oracle as O

    kw = {}
    if npu > 0:
        ncut = math.ceil(((npu * 2.0 / 200.0) ** (1.0 / 3.0)) / 2.0)
        kw = dict(ncut=ncut, nxbuffer=4 * ncut, nsel=math.ceil((2 * ncut + 1.0) ** 3 * 200.0 * 4.0))
    if ndelta:
        kw.update(delta_extra=EXTRA_DELTAS, nbins=EXTRA_BINS)
    return O.Params(nx=snx, **kw)


def _oracle_worker(seeds, snx, nmax, npu, ndelta, inq, outq):
    """One host core of the CPU arms.  Builds its sample boxes once, before
    any clock starts, then runs cic/cicm1/tri_cic/spherover of the oracle
    (reference arithmetic) on them for every "run" it receives and returns
    (halos, seconds of oracle work)."""
    import torch

    from oracle import oracle as O
    from psod_b200 import synth

    torch.set_num_threads(1)
    boxes = []
    for sd in seeds:
        b = synth.make_box(snx, nmax_halo=nmax, seed=sd)
        boxes.append((b.pos.numpy().copy(), b.ids.numpy().copy()))
    params = _oracle_params(snx, npu, ndelta)
    O.lib()
    outq.put((0, 0.0))
    while inq.get() == "run":
        halos, busy = 0, 0.0
        for pos, ids in boxes:
            t0 = time.perf_counter()
            r = O.run(params, pos, ids, O.REFERENCE)
            busy += time.perf_counter() - t0
            halos += r.nhalo
        outq.put((halos, busy))


class OracleCores:
    """``cores`` worker processes (spawned), each holding its own sample
    boxes.  ``step()`` runs every worker once and returns the halos found,
    the oracle seconds summed over workers and the step's wall time."""

    def __init__(self, cores, boxes_per_core, seed, snx, nmax, npu, ndelta):
        import multiprocessing as mp

        from oracle import oracle as O

        O.build()
        ctx = mp.get_context("spawn")
        self.out = ctx.Queue()
        self.ins, self.procs = [], []
        for c in range(cores):
            q = ctx.Queue()
            seeds = [seed + 100 + c * boxes_per_core + j for j in range(boxes_per_core)]
            pr = ctx.Process(target=_oracle_worker, args=(seeds, snx, nmax, npu, ndelta, q, self.out), daemon=True)
            pr.start()
            self.ins.append(q)
            self.procs.append(pr)
        for _ in self.procs:
            self.out.get()
        self.cores = cores

    def step(self):
        t0 = time.perf_counter()
        for q in self.ins:
            q.put("run")
        res = [self.out.get() for _ in self.ins]
        return sum(r[0] for r in res), sum(r[1] for r in res), time.perf_counter() - t0

    def close(self):
        for q in self.ins:
            q.put("stop")
        for pr in self.procs:
            pr.join(timeout=30)


def cpu_baseline(args, nx, wl, cores=1, boxes_per_core=2, steps=1, warmup=0):
    """The reference algorithm on ``cores`` host cores: the oracle in
    reference arithmetic on sample boxes built before the clock starts.
    value = halos / (oracle seconds / cores), i.e. only oracle work is timed;
    the wall time of the steps is reported beside it."""
    snx = sample_nx(nx)
    nmax = wl["nmax_halo"]
    npu = npu_for(nx)
    pool = OracleCores(cores, boxes_per_core, args.seed, snx, nmax, npu, args.ndelta)
    try:
        for _ in range(warmup):
            pool.step()
        halos, busy, wall = 0, 0.0, 0.0
        vals = []
        for _ in range(steps):
            h, b, w = pool.step()
            halos, busy, wall = halos + h, busy + b, wall + w
            vals.append(h / (b / cores) if b > 0 else 0.0)
    finally:
        pool.close()
    what = "the workload's own box" if snx == nx else f"box(es) of {snx}^3 cells from the workload's generator law"
    return {
        "value": round(halos / (busy / cores), 3) if busy > 0 else 0.0,
        "unit": "halos/s",
        "cores": cores,
        "kind": "port",
        "sample": f"{cores * boxes_per_core} {what} (halo N in [20, {nmax}], npu {npu}, seeds from {args.seed + 100}), "
                  f"{'Delta 200/500/178, 48 bins, ' if args.ndelta else 'Delta 200, 60 bins, '}"
                  f"cic/cicm1/tri_cic/spherover of the C oracle in reference arithmetic, one core each; "
                  f"{halos // max(1, steps)} halos and {busy / max(1, steps):.1f} core-seconds of oracle work a step; "
                  f"boxes built before timing; wall {wall / max(1, steps):.1f} s a step",
        "step_values": [round(v, 3) for v in vals],
    }


def run_reference(args):
    """The driver's reference arm: the reference's algorithm (the C oracle,
    reference arithmetic; the Fortran itself cannot be built here) on all
    host cores, rank 0 only, same metric, unit and config as our arm."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    nx = args.nx
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    cores = max(1, min(os.cpu_count() or 1, 64))
    cb = cpu_baseline(args, nx, wl, cores=cores, boxes_per_core=1, steps=args.steps, warmup=args.warmup)
    v = cb["value"]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "halos/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic NFW-mixture boxes (seeded)",
        "mode": "reference CPU oracle",
        "config": workload_config(nx, args.ndelta),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": v, "unit": "halos/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


FOF_METRIC = "FoF particles/s (b=0.2, Mmin=20, one rank, periodic)"


def run_fof(args):
    """The friends-of-friends stage (psod_fof) on the workload's box: one
    step = linking-cell sort, union-find, labels, member lists, centres and
    radii over all particles.  value: particles per second with the particles
    resident in HBM; e2e: host positions/IDs/velocities in, the catalogue
    (halo table and member IDs) out, through the public API."""
    import numpy as np
    import torch

    from psod_b200 import synth
    from psod_b200.sod import SphericalOverdensity

    nx = args.nx
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    torch.cuda.set_device(0)
    box = synth.make_box(nx, nmax_halo=wl["nmax_halo"], seed=args.seed, device="cuda:0")
    pos_d, ids_d = box.pos, box.ids
    del box
    gen = torch.Generator(device="cuda:0")
    gen.manual_seed(args.seed + 7)
    vel_d = torch.randn(pos_d.shape, generator=gen, device="cuda:0", dtype=torch.float32) * 300.0
    torch.cuda.empty_cache()
    n = int(pos_d.shape[0])
    sod = SphericalOverdensity(nx, device=0)
    sod.load(pos_d, ids_d, vel=vel_d)
    for _ in range(args.warmup):
        st = sod.fof(percolation=0.2, mmin=20)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(0) as clk:
        ev0.record()
        for _ in range(args.steps):
            stats.append(sod.fof(percolation=0.2, mmin=20))
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    st = stats[-1]
    # e2e through the public API: pinned host arrays in, catalogue out
    pos_h, ids_h, vel_h = (x.cpu().pin_memory() for x in (pos_d, ids_d, vel_d))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sod.load(pos_h, ids_h, vel=vel_h)
        sod.fof(percolation=0.2, mmin=20)
        cat = sod.fof_halos()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    d2h = sum(getattr(cat, f).nbytes for f in cat.__dataclass_fields__)
    sod.close()
    peak, peak_kind = load_peaks()
    # union-find linking: each record's position (16 B) read and its parent
    # (4 B) written once per launch is the algorithmic floor of the kernel
    link_s = st["ms_link"] / 1000.0
    alg = 20.0 * n
    achieved = alg / link_s / 1e9 if link_s > 0 else 0.0
    line = {
        "metric": FOF_METRIC, "value": round(n / (ms / 1000.0), 1), "unit": "particles/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (friend test), f64 (centres, radii)",
        "data": "synthetic NFW-mixture box (seeded); inputs resident in HBM",
        "config": {"workload": wl["box"] + ", FoF b=0.2, Mmin=20", "nx": nx, "particles": n,
                   "l2": "inputs larger than L2" if n * 16 > 126e6 else "inputs fit in L2 (no flush)"},
        "detail": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()},
        "e2e": {"value": round(n / (e2e_ms / 1000.0), 1), "unit": "particles/s",
                "h2d_bytes_per_step": int(n * (12 + 8 + 12)), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": round(e2e_ms, 3)},
        "roofline": {"bound": "hbm", "kernel": "k_fof_link_thread + k_fof_link_warp (union-find over linking cells)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "peak_kind": peak_kind, "traffic": None, "alg_bytes_per_launch": int(alg),
                     "kernel_ms": round(st["ms_link"], 3)},
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        # the oracle's sequential pFoF on the 128^3 box of the same law
        from oracle import oracle as O

        snx = min(nx, 128)
        b = synth.make_box(snx, nmax_halo=WORKLOADS.get(snx, wl)["nmax_halo"], seed=args.seed + 100)
        p, i = b.pos.numpy(), b.ids.numpy()
        t0 = time.perf_counter()
        r = O.fof(p, i, percolation=0.2, nres=snx, mmin=20)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(len(p) / dt, 1), "unit": "particles/s", "cores": 1, "kind": "port",
                                "sample": f"one {snx}^3 box of the workload's law ({len(p)} particles, {r.nhalo} "
                                          f"halos), the C oracle's sequential pFoF scan + merge + observables, "
                                          f"{dt:.2f} s"}
    print(json.dumps(line), flush=True)


PROPS_METRIC = "halo properties halos/s (haloanalyzer halo_properties on the SOD table)"
# units of a RAMSES run of this box size: 100 Mpc/h per 128 cells, z = 0
PROPS_UNITS = dict(unit_d=2.7e-30, unit_t=4.4e17, aexp=1.0, h0=70.0, hz=1.0, delta_vir=178.0)


def run_props(args):
    """The halo-properties stage (psod_halo_properties) on the SOD table of
    the workload's box: one step = every halo's moments, potential energy,
    profiles, R178 and inertia eigen solve.  value: halos per second with the
    particles and the table resident in HBM; e2e adds the copy of every
    output to host memory."""
    import numpy as np
    import torch

    from psod_b200 import synth
    from psod_b200.sod import SphericalOverdensity

    nx = args.nx
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    torch.cuda.set_device(0)
    box = synth.make_box(nx, nmax_halo=wl["nmax_halo"], seed=args.seed, device="cuda:0")
    pos_d, ids_d = box.pos, box.ids
    del box
    gen = torch.Generator(device="cuda:0")
    gen.manual_seed(args.seed + 7)
    vel_d = torch.randn(pos_d.shape, generator=gen, device="cuda:0", dtype=torch.float32) * 0.3
    torch.cuda.empty_cache()
    units = dict(PROPS_UNITS, unit_l=3.08568e24 * 100 / 0.7 * nx / 128, levelmin=int(round(np.log2(nx))))
    sod = SphericalOverdensity(nx, device=0, npu=npu_for(nx), mode=1)
    sod.load(pos_d, ids_d, vel=vel_d)
    sst = sod.run()
    for _ in range(args.warmup):
        sod.halo_properties(**units, source="sod")
    torch.cuda.synchronize()
    stats = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            stats.append(sod.halo_properties(**units, source="sod")[1])
    ms = sum(s["ms_total"] for s in stats) / len(stats)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out, st = sod.halo_properties(**units, source="sod")
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    nh = int(st["nhalo"])
    line = {
        "metric": PROPS_METRIC, "value": round(nh / (ms / 1000.0), 1), "unit": "halos/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (sums), f32 (pair terms, outputs)",
        "data": "synthetic NFW-mixture box (seeded), random velocities; SOD table resident in HBM",
        "config": {"workload": wl["box"] + ", SOD batched, then halo_properties", "nx": nx, "halos": nh,
                   "members": int(st["nmember"])},
        "detail": {"potential_items": int(st["potential_items"]), "sod_ms": round(sst["ms_total"], 1)},
        "e2e": {"value": round(nh / (e2e_ms / 1000.0), 1), "unit": "halos/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(a.nbytes for a in out.values())), "ms_per_step": round(e2e_ms, 3)},
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        t = sod.halos()
        pos_h = pos_d.cpu().numpy()
        vel_h = vel_d.cpu().numpy()
        # a bounded sample: every k-th halo, about 20 s of one core at most
        k = max(1, nh // 4000)
        sel = np.arange(0, nh, k)
        off = [0]
        mem = []
        for hh in sel:
            m = t.member_index[t.member_offset[hh]: t.member_offset[hh + 1]]
            mem.append(m)
            off.append(off[-1] + len(m))
        t0 = time.perf_counter()
        O.halo_properties(np.array(off), np.concatenate(mem), pos_h, vel_h, **units)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(len(sel) / dt, 2), "unit": "halos/s", "cores": 1, "kind": "port",
                                "sample": f"every {k}th halo of the same table ({len(sel)} halos, "
                                          f"{off[-1]} members), the C oracle's halo_properties, {dt:.2f} s"}
    sod.close()
    print(json.dumps(line), flush=True)


def relaunch_with_torchrun(args):
    """``--gpus N`` without a torchrun environment: start the N ranks here
    (one process per GPU) with the same arguments, and return their status."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def run_zones(args):
    """The reference's zone decomposition on one GPU: the workload's box cut
    into K^3 zones (-npu's buffer, main:211-219), each zone's particles and
    buffer selected by the FP64 test of psod_select_zone (main:578-584, here
    on the device over the resident box), and a zone context per zone
    running the SOD stage (cell sort, CIC, seed order, spherover) on them in
    turn.  value: kept halos of all zones per second of summed device time
    of the zone steps (the selection and the context set-up untimed); the
    zone catalogues together are compared with the one-zone run's halo
    count.  A report run, not the bench contract's timing."""
    import torch

    from psod_b200 import synth
    from psod_b200.sod import SphericalOverdensity

    nx, k = args.nx, args.zones
    wl = WORKLOADS.get(nx, dict(nmax_halo=20000, box=f"{nx}^3"))
    thresholds = dict(delta_extra=EXTRA_DELTAS, nbins=EXTRA_BINS) if args.ndelta else {}
    # the learned mode needs a trained bracket: zones run batched (or plain)
    params = dict(npu=npu_for(nx), mode=0 if args.mode_id == 0 else 1, **thresholds)
    torch.cuda.set_device(0)
    box = synth.make_box(nx, nmax_halo=wl["nmax_halo"], seed=args.seed, device="cuda:0")
    pos_d, ids_d = box.pos, box.ids
    del box
    torch.cuda.empty_cache()
    n = int(pos_d.shape[0])
    one_st = {"nhalo": None}
    if args.zone_only < 0:  # the one-zone run, for the catalogue comparison
        with SphericalOverdensity(nx, device=0, **params) as one:
            one.load(pos_d, ids_d)
            one_st = one.run()
        torch.cuda.empty_cache()
    nxzone = nx // k
    # the buffer -npu derives (main:211-219, as psod_ctx_create does), else half a zone
    npu = params["npu"]
    nxb = 4 * math.ceil((npu * 2.0 / 200.0) ** (1.0 / 3.0) / 2.0) if npu > 0 else nxzone // 2
    rs = (0.5 + nxb / float(nxzone)) / float(k)

    def axis_keep(col, i):
        xc = ((i / float(k)) + ((i + 1) / float(k))) / 2.0
        d = (pos_d[:, col].double() - xc).abs()
        return (d < rs) | (d > 1.0 - rs)

    total_ms, halos, parts = 0.0, 0, 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for z in (range(k ** 3) if args.zone_only < 0 else [args.zone_only]):
        ix, iy, iz = z // (k * k), (z // k) % k, z % k
        keep = axis_keep(0, ix) & axis_keep(1, iy) & axis_keep(2, iz)
        sel = torch.nonzero(keep).squeeze(1)
        p, i = pos_d[sel].contiguous(), ids_d[sel].contiguous()
        del keep, sel
        with SphericalOverdensity(nx, device=0, nxcpu=k, nzone=z, **params) as s:
            s.load(p, i, npart_total=n)  # warm-up: sizes the context's buffers
            s.run()
            torch.cuda.synchronize()
            ev0.record()
            s.load(p, i, npart_total=n)
            st = s.run()
            ev1.record()
            torch.cuda.synchronize()
        total_ms += ev0.elapsed_time(ev1)
        halos += st["nhalo"]
        parts += int(p.shape[0])
        del p, i
        torch.cuda.empty_cache()
    line = {
        "metric": METRIC + ", zone decomposition",
        "value": round(halos / (total_ms / 1000.0), 2),
        "unit": "halos/s",
        "n_gpus": 1,
        "zones": k ** 3 if args.zone_only < 0 else 1,
        "ms_all_zones": round(total_ms, 1),
        "halos": halos,
        "one_zone_halos": one_st["nhalo"],
        "particles_loaded": parts,
        "particles": n,
        "nxbuffer": nxb,
        "config": workload_config(nx, args.ndelta, False),
        "data": "synthetic NFW-mixture box (seeded); zone particles resident in HBM",
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--mode", default="learned", choices=["plain", "batched", "learned"])
    ap.add_argument("--no-compare-plain", dest="compare_plain", action="store_false")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--delta200-only", dest="ndelta", action="store_false",
                    help="Delta = 200 and 60 bins only (default: 200, 500 and 178 in one pass, 48 bins)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default scheduling thresholds instead of psod_autotune in the warm-up")
    ap.add_argument("--props", action="store_true",
                    help="time the halo-properties stage (psod_halo_properties) on the SOD table; one GPU")
    ap.add_argument("--fof", action="store_true",
                    help="time the friends-of-friends stage (psod_fof) instead of SOD; one GPU")
    ap.add_argument("--zones", type=int, default=0,
                    help="report run of the reference's zone decomposition: the box as K^3 zones in turn; one GPU")
    ap.add_argument("--zone-only", dest="zone_only", type=int, default=-1,
                    help="with --zones: run only this zone (no one-zone comparison)")
    ap.add_argument("--heavy", action="store_true",
                    help="the heavy-tail stress box (1024^3 + 16 clusters of 5e6, -npu 1e7, Delta 200/500, 64 bins)")
    args = ap.parse_args()
    args.mode_id = {"plain": 0, "batched": 1, "learned": 2}[args.mode]
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_with_torchrun(args))
    if args.impl == "reference":
        run_reference(args)
    elif args.fof:
        run_fof(args)
    elif args.props:
        run_props(args)
    elif args.zones > 0:
        run_zones(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
