"""Benchmark of the P3M + short-range force path (particle-steps/s).

Workload (default): the single large system of 2^20 monovalent ions (half
+1, half -1) at number density 0.5 in a cubic box of side 128 on a jittered
lattice, LJ eps=1 sigma=1 cutoff 2.5 (shift auto), P3M cao 7, r_cut 3.5 and
a 256^3 mesh with alpha tuned for an rms force error estimate <= 1e-4 (at
r_cut 3.5 and cao 7 the error estimate of a 128^3 mesh bottoms out at
3.9e-3 whatever alpha, so 256^3 is the smallest mesh reaching 1e-4), FP32-mixed
mesh/FFT path.  One step = one full force evaluation (k-space + real-space
Coulomb + LJ through the Verlet list) of the whole system; positions stay
fixed, so the Verlet list is reused (its rebuild cost is measured apart:
`verlet_rebuild_ms`).  Inputs (>= 1 GB resident with the neighbour list)
exceed the 126 MB L2.

After the headline timing (outside its timed region) the same run adds:
`variants` -- the plain FP64 GPU path on the same workload and the batched
512-replica Langevin step (one CUDA graph per step) -- so that the metric's
four cells (FP32-mixed vs FP64, single vs batched) sit on one line; and
`accuracy` -- the rms Coulomb force error of the FP32-mixed and FP64 paths
and of the oracle's CPU P3M against the FP64 direct Ewald sum on a seeded
20 000-ion subsample (forces from all 2^20 sources).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the
workload on its own GPU (replicas only: the path has no exchange step);
value = all particles of all ranks / max-over-ranks time.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at rms force err <=1e-4 (FP32-mixed P3M+LJ force evaluation)"
HBM_FALLBACK = 6650.0
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--cao", type=int, default=7)
    ap.add_argument("--r_cut", type=float, default=3.5)
    ap.add_argument("--accuracy", type=float, default=1e-4)
    ap.add_argument("--fp64", action="store_true", help="plain FP64 path instead of FP32-mixed")
    ap.add_argument("--box", type=float, default=128.0,
                    help="box side; N = 0.5 box^3 (128 -> 2^20); smaller boxes for ncu captures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="single",
                    choices=["single", "batched", "elc", "melt", "pe_sweep", "dipolar"],
                    help="single large system (default), batched replicas, the single "
                         "system as a slab with an empty gap along z (P3M + ELC), a bead-spring "
                         "melt, a salt sweep of polyelectrolyte replicas, or point dipoles "
                         "(dipolar P3M)")
    ap.add_argument("--dipoles", type=int, default=1 << 20,
                    help="dipole count of --workload dipolar (density 0.5)")
    ap.add_argument("--gap", type=float, default=16.0, help="ELC gap size (--workload elc)")
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--skin", type=float, default=None,
                    help="Verlet skin (default 0.4 single system; 0.8 batched: the fastest of "
                         "0.4/0.6/0.8/1.0 in timed trials of the batched Langevin run, as a "
                         "skin tuning would choose)")
    ap.add_argument("--profile-only", action="store_true",
                    help="setup + a few evaluations, no JSON (for ncu captures)")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the FP64 and batched variant timings of the default run")
    ap.add_argument("--no-ewald", action="store_true",
                    help="skip the full-size accuracy check against the direct Ewald sum")
    ap.add_argument("--variant-steps", type=int, default=20)
    ap.add_argument("--sample-every", type=int, default=0,
                    help="batched: record temperature and potential energy every K steps "
                         "(outside the timed chunks), e.g. --steps 10000 --sample-every 1000")
    return ap.parse_args()


def make_workload(seed=0, box=128.0, jitter=0.2):
    """Jittered simple-cubic lattice at density 0.5 with alternating charges,
    thinned symmetrically to exactly 0.5 box^3 neutral ions (2^20 at 128)."""
    n_target = int(round(0.5 * box ** 3))
    n_target -= n_target % 2
    n_side = int(np.ceil(n_target ** (1.0 / 3.0)))
    n_side += n_side % 2
    rng = np.random.default_rng(seed)
    a = box / n_side
    idx = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    q = np.where(idx.sum(1) % 2 == 0, 1.0, -1.0)
    pos = (idx + 0.5) * a + rng.uniform(-jitter, jitter, idx.shape)
    drop = (len(q) - n_target) // 2
    plus = np.flatnonzero(q > 0)
    minus = np.flatnonzero(q < 0)
    keep = np.ones(len(q), bool)
    keep[rng.choice(plus, drop, replace=False)] = False
    keep[rng.choice(minus, drop, replace=False)] = False
    return pos[keep].copy(), q[keep].copy(), box


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


class ClockSampler:
    def __init__(self, index=0):
        self.samples = []
        self.index = index
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 2 + k and s[2 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons}


def cpu_reference_step(pos, q, box, mesh, cao, alpha, r_cut, tab):
    from oracle import oracle as O
    p = O.make_params(box, mesh, cao, alpha, r_cut, 1.0)
    t0 = time.perf_counter()
    fk, _, _ = O.p3m_kspace(p, pos, q)
    fr, _, _, _ = O.short_range(p, pos, q, None, 1, tab)
    return time.perf_counter() - t0


def lj_table_oracle():
    from oracle import oracle as O
    cut = 2.5
    shift = -((1 / cut) ** 12 - (1 / cut) ** 6)
    return O.pair_table(1, {(0, 0): dict(lj_eps=1.0, lj_sig=1.0, lj_cut=cut, lj_shift=shift)})


def config_dict(args, n, alpha, nranks):
    return {"workload": f"single system: {n} ions, density 0.5, box {args.box:g}, LJ 2.5, "
                        f"P3M mesh {args.mesh}^3 cao {args.cao} r_cut {args.r_cut}",
            "n_particles_per_rank": int(n), "box": args.box, "mesh": args.mesh, "cao": args.cao,
            "r_cut": args.r_cut, "alpha": alpha, "accuracy_target": args.accuracy,
            "lj": {"epsilon": 1.0, "sigma": 1.0, "cutoff": 2.5},
            "precision": "fp64" if args.fp64 else "fp32-mixed",
            "step": "one full force evaluation, Verlet list reused",
            "l2": "inputs larger than L2 (neighbour list ~1 GB)",
            "parallelism": f"replicas x{nranks}" if nranks > 1 else "single GPU"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    pos, q, box = make_workload(box=args.box)
    n = len(q)
    # alpha of the tuned GPU configuration (same error-estimate formula)
    alpha = tuned_alpha(args, n, float(np.sum(q * q)), box)
    tab = lj_table_oracle()
    for _ in range(args.warmup):
        cpu_reference_step(pos, q, box, args.mesh, args.cao, alpha, args.r_cut, tab)
    times = [cpu_reference_step(pos, q, box, args.mesh, args.cao, alpha, args.r_cut, tab)
             for _ in range(args.steps)]
    t = float(np.mean(times))
    v = n / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(args, n, alpha, 1),
        "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": ncores, "kind": "port",
                         "sample": "full workload per step: FP64 CPU restatement of the "
                                   "reference CPU P3M + link-cell LJ/real-space (OpenMP)"},
        "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def time_single_variant(lib, h, n, pos_d, q_d, t_d, f_d, stream, sp, args):
    """ms per force evaluation of handle h on the resident inputs (CUDA
    events on the launching stream), its stage profile and its dominant
    stage; same step definition as the headline."""
    import torch
    from espresso_b200 import _lib
    flags = _lib.P3MX_DEVICE_PTRS | _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE

    def step():
        _lib.check(lib.p3mx_forces(h, n, _lib.dptr(pos_d), _lib.dptr(q_d), _lib.dptr(t_d),
                                   _lib.dptr(f_d), None, None, flags, sp), h)
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    k = max(args.variant_steps, 10)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1) / k
    names = (ctypes.c_char_p * 32)()
    ms = (ctypes.c_double * 32)()
    nst = ctypes.c_int()
    _lib.check(lib.p3mx_profile(h, 3, ms, names, 32, ctypes.byref(nst)), h)
    stages = {names[j].decode(): ms[j] for j in range(nst.value)}
    dom = max(stages, key=stages.get)
    return {"value": n / (t_ms * 1e-3), "unit": "particle-steps/s", "ms_per_step": t_ms,
            "steps": k, "dtype": "f64", "stages_ms": stages,
            "dominant_stage": {"kernel": dom, "ms": stages[dom]}}


EWALD_SUBSAMPLE = 20000
EWALD_PARAMS = dict(alpha=0.15, r_cut=27.0, kmax=30)


def ewald_accuracy(pos, q, box, alpha, args, f32, f64):
    """rms Coulomb force error on a seeded 20 000-ion subsample against the
    FP64 direct Ewald sum over all sources (oracle.ewald_targets; real-space
    and reciprocal truncation terms exp(-16) and exp(-24)), for the
    FP32-mixed and FP64 GPU forces and for the oracle's CPU P3M."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    sub = np.sort(np.random.default_rng(2024).choice(len(q), min(EWALD_SUBSAMPLE, len(q)),
                                                     replace=False))
    if min(box, box, box) < 2 * EWALD_PARAMS["r_cut"]:
        return {"rms_force_err_vs_ewald_20k": None, "ewald_note": "box too small"}
    fe = O.ewald_targets([box] * 3, pos, q, sub, 1.0, **EWALD_PARAMS)
    p = O.make_params(box, args.mesh, args.cao, alpha, args.r_cut, 1.0)
    fk, _, _ = O.p3m_kspace(p, pos, q)
    fr, _, _, _ = O.short_range(p, pos, q)
    fo = (fk + fr)[sub]

    def rms(a):
        return float(np.sqrt(((a - fe) ** 2).sum(1).mean()))
    return {"rms_force_err_vs_ewald_20k": rms(f32[sub]),
            "rms_force_err_vs_ewald_20k_fp64": rms(f64[sub]),
            "rms_force_err_vs_ewald_20k_oracle_cpu_p3m": rms(fo),
            "ewald": {"subsample": int(len(sub)), "seed": 2024, **EWALD_PARAMS,
                      "seconds": time.perf_counter() - t0}}


def tuned_alpha(args, n, sum_q2, box):
    """alpha_L from calculate_accuracy (p3m.cpp:636-655) at fixed r_cut."""
    from math import log, sqrt
    L = box
    r_iL = args.r_cut / L
    V = L ** 3
    rs0 = 2.0 * sum_q2 / sqrt(n * r_iL * L * V)
    aL = sqrt(log(sqrt(2.0) * rs0 / args.accuracy)) / r_iL if sqrt(2.0) * rs0 > args.accuracy else 0.1
    return aL / L


def serpentine_lattice(n):
    """Sites of an n^3 simple-cubic lattice in boustrophedon order: every
    step between consecutive sites is one lattice spacing."""
    k = np.arange(n ** 3)
    z = k // (n * n)
    yi = (k // n) % n
    y = np.where(z % 2 == 0, yi, n - 1 - yi)
    row = z * n + yi
    xi = k % n
    x = np.where(row % 2 == 0, xi, n - 1 - xi)
    return np.stack([x, y, z], 1).astype(float)


def make_melt(seed=0, n_chains=4000, chain_len=250, salt=0.1, density=0.85, jitter=0.05):
    """Polyelectrolyte melt: n_chains bead-spring chains of chain_len beads,
    every other bead charged -1, +1 counterions and 1:1 salt at number
    density `salt` per species, at total density `density`.  Chains follow
    a boustrophedon walk over a simple-cubic lattice (consecutive beads one
    spacing ~1.05 apart, no overlaps), cut into segments of chain_len sites
    of which n_chains random ones hold the chains (spread over the whole
    box); counterions and salt take random free sites.  Returns positions,
    charges, FENE bond list (type 0, i, j), box."""
    n_bead = n_chains * chain_len
    n_mon_q = n_chains * ((chain_len + 1) // 2)
    n_tot = int(round((n_bead + n_mon_q) / (1.0 - 2.0 * salt / density)))
    n_salt = (n_tot - n_bead - n_mon_q) // 2
    n_tot = n_bead + n_mon_q + 2 * n_salt
    L = (n_tot / density) ** (1.0 / 3.0)
    side = int(np.ceil(n_tot ** (1.0 / 3.0)))
    a = L / side
    rng = np.random.default_rng(seed)
    sites = serpentine_lattice(side)
    n_seg = len(sites) // chain_len
    seg = rng.choice(n_seg, n_chains, replace=False)
    in_chain = np.zeros(len(sites), bool)
    chain_idx = (seg[:, None] * chain_len + np.arange(chain_len)[None, :]).ravel()
    in_chain[chain_idx] = True
    chain_sites = sites[chain_idx]
    free = sites[~in_chain]
    pick = rng.choice(len(free), n_mon_q + 2 * n_salt, replace=False)
    pos = np.vstack([chain_sites, free[pick]]) * a + 0.5 * a
    pos += rng.uniform(-jitter, jitter, pos.shape)
    bead = np.arange(n_bead) % chain_len
    q = np.concatenate([np.where(bead % 2 == 0, -1.0, 0.0), np.ones(n_mon_q),
                        np.ones(n_salt), -np.ones(n_salt)])
    first = (np.arange(n_chains) * chain_len)[:, None] + np.arange(chain_len - 1)[None, :]
    i = first.ravel()
    bonds = np.stack([np.zeros_like(i), i, i + 1], 1).astype(np.int32)
    return pos, q, bonds, L


def make_replicas(n_rep, seed=0, density=0.3, nmin=1000, nmax=50000):
    """Batched workload: n_rep cubic systems, N log-uniform in [nmin, nmax]
    (even), density 0.3, all charges +z/-z with z in {1, 2} per replica,
    Bjerrum length U[0.5, 4] (prefactor at kT = 1), random sites of a
    jittered lattice."""
    rng = np.random.default_rng(seed)
    boxes, prefs, pos, q, offs = [], [], [], [], [0]
    for _ in range(n_rep):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))) // 2 * 2
        L = (n / density) ** (1 / 3)
        side = int(np.ceil(n ** (1 / 3)))
        sel = rng.choice(side ** 3, n, replace=False)
        idx = np.stack(np.unravel_index(sel, (side,) * 3), -1).astype(float)
        p = (idx + 0.5) * (L / side) + rng.uniform(-0.1, 0.1, idx.shape)
        z = float(rng.choice([1.0, 2.0]))
        qq = np.concatenate([np.full(n // 2, z), np.full(n // 2, -z)])
        rng.shuffle(qq)
        boxes.append([L, L, L])
        prefs.append(float(rng.uniform(0.5, 4.0)))
        pos.append(p)
        q.append(qq)
        offs.append(offs[-1] + n)
    return (np.array(boxes), np.array(prefs), np.vstack(pos), np.concatenate(q),
            np.array(offs, dtype=np.int64))


def run_batched(args):
    """Batched replicas (config 4): all replicas advance by one graph launch
    per MD step (velocity Verlet + Langevin kT=1, gamma=1, dt=0.01)."""
    res = batched_measure(args, args.steps, args.warmup, cpu=not args.no_cpu_baseline,
                          fp64=args.fp64)
    if res is not None:
        print(json.dumps(res))


def batched_measure(args, steps, warmup, cpu=True, fp64=False, clocks=True):
    """Times `steps` graph-captured Langevin steps of the batched replicas
    (CUDA events on the batch's stream) and returns the bench line as a
    dict: value, ms_per_step, stage profile, tuning summary and (cpu=True)
    the oracle's CPU rate on a sample of the replicas."""
    import torch
    from espresso_b200 import _lib
    P = ctypes.POINTER
    lib = _lib.load()
    torch.cuda.set_device(0)
    boxes, prefs, pos, q, offs = make_replicas(args.replicas)
    n = len(q)
    d = _lib.BatchDesc()
    d.n_rep = len(prefs)
    d.box = boxes.ctypes.data_as(P(ctypes.c_double))
    d.prefactor = prefs.ctypes.data_as(P(ctypes.c_double))
    d.offset = offs.ctypes.data_as(P(ctypes.c_longlong))
    d.accuracy = args.accuracy
    d.skin = args.skin if args.skin is not None else 0.8
    d.single_precision = 0 if fp64 else 1
    d.mesh_min, d.mesh_max, d.cao_min, d.cao_max = 16, 64, 3, 7
    tab = (_lib.PairParams * 1)()
    tab[0].wca_eps = 1.0
    tab[0].wca_sig = 1.0
    types = np.zeros(n, dtype=np.int32)
    h = ctypes.c_void_p()
    t0 = time.perf_counter()
    rc = lib.p3mx_batch_create(ctypes.byref(d), pos.ctypes.data_as(P(ctypes.c_double)),
                               q.ctypes.data_as(P(ctypes.c_double)),
                               types.ctypes.data_as(P(ctypes.c_int)), 1, tab, ctypes.byref(h))
    t_tune = time.perf_counter() - t0
    if rc:
        raise RuntimeError(lib.p3mx_batch_last_error(h).decode())
    stream = torch.cuda.ExternalStream(lib.p3mx_batch_stream(h))
    _lib.check(lib.p3mx_batch_run(h, max(3, warmup), 0.01, 1.0, 1.0, 7), h,
               lib.p3mx_batch_last_error)
    if getattr(args, "profile_only", False):
        # `steps` graph steps inside a profiler range (ncu --profile-from-start
        # off captures them without the tuner's trial launches)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        _lib.check(lib.p3mx_batch_run(h, steps, 0.01, 1.0, 1.0, 7), h, lib.p3mx_batch_last_error)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        lib.p3mx_batch_destroy(h)
        return None
    lc0, lc1 = ctypes.c_longlong(), ctypes.c_longlong()
    lib.p3mx_batch_launch_count(h, ctypes.byref(lc0))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    series = []
    chunk = getattr(args, "sample_every", 0) or steps
    t_total = 0.0
    with ClockSampler(0) as clk:
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            e0.record(stream)
            _lib.check(lib.p3mx_batch_run(h, k, 0.01, 1.0, 1.0, 7), h,
                       lib.p3mx_batch_last_error)
            e1.record(stream)
            torch.cuda.synchronize()
            t_total += e0.elapsed_time(e1)
            done += k
            if chunk < steps:
                # stability record outside the timed chunks: per-replica
                # kinetic temperature and the total potential energy
                ep = np.zeros(len(prefs))
                _lib.check(lib.p3mx_batch_forces(h, ep.ctypes.data_as(P(ctypes.c_double))), h,
                           lib.p3mx_batch_last_error)
                v = np.zeros((n, 3))
                _lib.check(lib.p3mx_batch_get(h, None, None, v.ctypes.data_as(P(ctypes.c_double))),
                           h, lib.p3mx_batch_last_error)
                tr = np.array([(v[offs[r]:offs[r + 1]] ** 2).mean() for r in range(len(prefs))])
                series.append({"step": done, "kT_mean": float(tr.mean()),
                               "kT_min": float(tr.min()), "kT_max": float(tr.max()),
                               "e_pot_per_particle": float(ep.sum() / n),
                               "finite": bool(np.isfinite(v).all())})
    lib.p3mx_batch_launch_count(h, ctypes.byref(lc1))
    t_ms = t_total / steps
    # stage profile of one force evaluation of the whole batch (outside the
    # timed region)
    names = (ctypes.c_char_p * 32)()
    sms = (ctypes.c_double * 32)()
    nst = ctypes.c_int()
    _lib.check(lib.p3mx_batch_profile(h, 3, sms, names, 32, ctypes.byref(nst)), h,
               lib.p3mx_batch_last_error)
    stages = {names[k].decode(): sms[k] for k in range(nst.value)}
    tuned = []
    for r in range(len(prefs)):
        t = _lib.Tuned()
        lib.p3mx_batch_get_tuned(h, r, ctypes.byref(t))
        tuned.append((t.mesh[0], t.cao, t.r_cut, t.accuracy))
    meshes = np.array([x[0] for x in tuned])
    acc = np.array([x[3] for x in tuned])
    rcs = np.array([x[2] for x in tuned])
    nrep = np.diff(offs).astype(float)
    # full-list Verlet candidates per step: N (4/3) pi (r_cut + skin)^3 rho
    pair_cand = float((nrep * 4.18879 * (np.maximum(rcs, 2 ** (1 / 6)) + d.skin) ** 3 *
                       nrep / boxes[:, 0] ** 3).sum())
    cpu_line = None
    if cpu:
        # sample: the first 8 replicas, one force evaluation each, FP64 oracle
        from oracle import oracle as O
        otab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
        ns, ts = 0, 0.0
        for r in range(min(8, len(prefs))):
            t = _lib.Tuned()
            lib.p3mx_batch_get_tuned(h, r, ctypes.byref(t))
            sl = slice(offs[r], offs[r + 1])
            p = O.make_params(boxes[r], list(t.mesh), t.cao, t.alpha, t.r_cut, prefs[r])
            t1 = time.perf_counter()
            O.p3m_kspace(p, pos[sl], q[sl])
            O.short_range(p, pos[sl], q[sl], None, 1, otab)
            ts += time.perf_counter() - t1
            ns += offs[r + 1] - offs[r]
        cpu_line = {"value": ns / ts, "unit": "particle-steps/s", "cores": os.cpu_count(),
                    "kind": "port",
                    "sample": "one force evaluation of each of the first 8 replicas, "
                              "FP64 CPU restatement (OpenMP, all host cores)"}
    lib.p3mx_batch_destroy(h)
    return {
        "metric": METRIC.replace("single", "batched"), "value": n / (t_ms * 1e-3),
        "unit": "particle-steps/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if fp64 else "f32-mixed (f64 positions/accumulators)",
        "data": "synthetic",
        "config": {"workload": f"batched: {len(prefs)} cubic replicas, N log-uniform "
                               f"[1e3, 5e4] (total {n}), density 0.3, +/-1 or +/-2 ions, "
                               f"l_B U[0.5, 4], WCA, P3M accuracy {args.accuracy}, meshes "
                               f"16-64 and cao 3-7 autotuned, Langevin VV dt 0.01 in one "
                               f"CUDA graph per step, Verlet skin {d.skin:g}",
                   "total_particles": int(n), "tuning_s": t_tune,
                   "mesh_hist": {int(m): int((meshes == m).sum()) for m in np.unique(meshes)},
                   "cao_hist": {int(c): int(sum(1 for t in tuned if t[1] == c))
                                for c in sorted({t[1] for t in tuned})},
                   "max_accuracy_estimate": float(acc.max()),
                   "r_cut_range": [float(rcs.min()), float(rcs.max())],
                   "verlet_candidates_per_step_est": pair_cand},
        "stages_ms": stages, "cpu_baseline": cpu_line,
        "stability": series or None,
        "clocks": clk.summary() if clocks else None,
        "gpu_launches": int(lc1.value - lc0.value)}


def run_melt(args):
    """Polyelectrolyte melt (config 3): 4000 FENE chains of 250 beads (K 30,
    R0 1.5), every other bead -1, +1 counterions, 1:1 salt at 0.1 per
    species, density 0.85 (1.96M particles), WCA, P3M mesh 256^3, cao 6,
    accuracy 1e-4 (r_cut and alpha tuned).  Times one force evaluation
    (P3M + WCA + FENE, device pointers) of the FP32-mixed and of the FP64
    path, and reports both paths' rms Coulomb force error against the FP64
    direct Ewald sum on a 20 000-ion subsample and their energy difference."""
    import torch
    import espresso_b200 as eb
    from espresso_b200 import _lib
    from espresso_b200.electrostatics import P3M, P3MGPU

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    pos, q, bonds, box = make_melt(seed=0)
    n = len(q)
    s = eb.System(box_l=[box] * 3)
    s.time_step = 0.01
    s.cell_system.skin = args.skin if args.skin is not None else 0.4
    s.part.add(pos=pos, q=q)
    s.non_bonded_inter[0, 0].wca.set_params(epsilon=1.0, sigma=1.0)
    t0 = time.perf_counter()
    act = P3MGPU(prefactor=1.0, accuracy=args.accuracy, mesh=256, cao=6, tune=True, timings=2,
                 verbose=False)
    s.electrostatics.solver = act
    t_tune = time.perf_counter() - t0
    prm = act.get_params()
    types = np.zeros(n, dtype=np.int32)
    fene = (_lib.BondParams * 1)()
    fene[0] = _lib.BondParams(_lib.P3MX_BOND_FENE, 30.0, 0.0, 1.5)
    bl = np.ascontiguousarray(bonds.reshape(-1), dtype=np.int32)
    pos_d = torch.from_numpy(pos).to(dev)
    q_d = torch.from_numpy(q).to(dev)
    t_d = torch.from_numpy(types).to(dev)
    f_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    flags = _lib.P3MX_DEVICE_PTRS | _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE

    def timed(h):
        def step():
            _lib.check(lib.p3mx_forces(h, n, _lib.dptr(pos_d), _lib.dptr(q_d), _lib.dptr(t_d),
                                       _lib.dptr(f_d), None, None, flags, sp), h)
        for _ in range(3):
            step()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    def with_bonds(h):
        _lib.check(lib.p3mx_set_bonds(h, 1, fene, len(bonds),
                                      bl.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), h)
        s._sync_pairs(h, types)

    with_bonds(act._handle)
    with ClockSampler(0) as clk:
        t32 = timed(act._handle)
    act64 = P3M(prefactor=1.0, accuracy=args.accuracy, mesh=256, cao=6, r_cut=prm["r_cut"],
                alpha=prm["alpha"], tune=False)
    s.electrostatics.clear()
    s.electrostatics.solver = act64
    with_bonds(act64._handle)
    t64 = timed(act64._handle)
    # Coulomb only (no WCA, no bonds) for the accuracy comparison, and the
    # energies of both paths (FP32 observables for the mixed path)
    zero_tab = (_lib.PairParams * 1)()
    res, en = [], []
    hflags = _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE
    for h, mixed in ((act._handle, True), (act64._handle, False)):
        _lib.check(lib.p3mx_set_pair_params(h, 1, zero_tab), h)
        _lib.check(lib.p3mx_set_bonds(h, 1, fene, 0, None), h)
        ff = np.zeros((n, 3))
        e3 = np.zeros(3)
        fl = hflags | _lib.P3MX_ENERGY | (_lib.P3MX_MIXED_OBSERVABLES if mixed else 0)
        _lib.check(lib.p3mx_forces(h, n, _lib.dptr(pos), _lib.dptr(q), _lib.dptr(types),
                                   _lib.dptr(ff), e3.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   None, fl, None), h)
        res.append(ff)
        en.append(float(e3[0] + e3[1]))
    acc = {}
    if not args.no_ewald:
        from oracle import oracle as O
        t1 = time.perf_counter()
        sub = np.sort(np.random.default_rng(2024).choice(n, EWALD_SUBSAMPLE, replace=False))
        fe = O.ewald_targets([box] * 3, pos, q, sub, 1.0, **EWALD_PARAMS)

        def rms(a):
            return float(np.sqrt(((a[sub] - fe) ** 2).sum(1).mean()))
        acc = {"rms_force_err_vs_ewald_20k_fp32_mixed": rms(res[0]),
               "rms_force_err_vs_ewald_20k_fp64": rms(res[1]),
               "ewald": {"subsample": EWALD_SUBSAMPLE, "seed": 2024, **EWALD_PARAMS,
                         "seconds": time.perf_counter() - t1}}
    out = {
        "metric": "particle-steps/s", "impl": "ours", "workload": "melt",
        "value": n / (t32 * 1e-3), "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps,
        "ms_per_step": t32, "ms_per_step_fp64": t64,
        "value_fp64": n / (t64 * 1e-3), "higher_is_better": True,
        "dtype": "f32-mixed (f64 positions/accumulators)", "data": "synthetic",
        "accuracy": {"rms_force_err_estimate": prm["accuracy"],
                     "fp32_vs_fp64_rms_coulomb_force_diff":
                         float(np.sqrt(((res[0] - res[1]) ** 2).sum(1).mean())),
                     "rms_coulomb_force": float(np.sqrt((res[1] ** 2).sum(1).mean())),
                     "coulomb_energy_fp32_mixed": en[0], "coulomb_energy_fp64": en[1],
                     "coulomb_energy_rel_diff": abs(en[0] - en[1]) / abs(en[1]), **acc},
        "clocks": clk.summary(),
        "config": {"workload": f"polyelectrolyte melt: 4000 FENE chains x 250 (K 30, R0 1.5), "
                               f"every other bead -1, +1 counterions, 1:1 salt 0.1 per species, "
                               f"{n} particles at density 0.85 (box {box:.2f}), WCA, P3M mesh "
                               f"256^3 cao 6, r_cut {prm['r_cut']:.4f}, alpha {prm['alpha']:.5f}, "
                               f"accuracy {args.accuracy:g}",
                   "tuning_s": t_tune, "bonds": int(len(bonds)),
                   "inputs": "resident in HBM, larger than L2"},
    }
    print(json.dumps(out))


def make_pe_sweep(n_rep=64, seed=0, n_chains=200, chain_len=100, volume=220000.0,
                  salt_lo=0.001, salt_hi=0.5):
    """Batched polyelectrolyte solutions (config 5): per replica n_chains
    chains of chain_len beads, every bead -1, +1 counterions, and 1:1 salt
    at a total salt-ion concentration swept log-uniformly over [salt_lo,
    salt_hi], in a cubic box of the given volume (40k-150k particles, total
    density 0.18-0.68).  Chains and ions sit on a jittered lattice of
    spacing <= 0.95 (boustrophedon chain segments at random places, ions at
    random free sites).  Returns boxes, prefactors (Bjerrum length 1),
    positions, charges, offsets, FENE bond list over the whole batch, and
    the salt concentrations."""
    rng = np.random.default_rng(seed)
    L = volume ** (1.0 / 3.0)
    salts = np.exp(np.linspace(np.log(salt_lo), np.log(salt_hi), n_rep))
    boxes, prefs, pos, q, offs, bonds = [], [], [], [], [0], []
    for r in range(n_rep):
        n_bead = n_chains * chain_len
        n_salt = int(round(0.5 * salts[r] * volume))
        n = 2 * n_bead + 2 * n_salt
        # lattice spacing <= 0.95 (FENE bonds well inside R0 = 1.5 at any
        # salt), finer where the particles need more sites
        side = max(int(np.ceil(n ** (1.0 / 3.0))), int(np.ceil(L / 0.95)))
        a = L / side
        sites = serpentine_lattice(side)
        n_seg = len(sites) // chain_len
        seg = rng.choice(n_seg, n_chains, replace=False)
        chain_idx = (seg[:, None] * chain_len + np.arange(chain_len)[None, :]).ravel()
        in_chain = np.zeros(len(sites), bool)
        in_chain[chain_idx] = True
        free = sites[~in_chain]
        pick = rng.choice(len(free), n_bead + 2 * n_salt, replace=False)
        p = np.vstack([sites[chain_idx], free[pick]]) * a + 0.5 * a
        p += rng.uniform(-0.05, 0.05, p.shape)
        qq = np.concatenate([-np.ones(n_bead), np.ones(n_bead), np.ones(n_salt), -np.ones(n_salt)])
        first = (np.arange(n_chains) * chain_len)[:, None] + np.arange(chain_len - 1)[None, :]
        i = first.ravel() + offs[-1]
        bonds.append(np.stack([np.zeros_like(i), i, i + 1], 1))
        boxes.append([L, L, L])
        prefs.append(1.0)
        pos.append(p)
        q.append(qq)
        offs.append(offs[-1] + n)
    return (np.array(boxes), np.array(prefs), np.vstack(pos), np.concatenate(q),
            np.array(offs, dtype=np.int64), np.vstack(bonds).astype(np.int32), salts)


def radial_distribution(x, box, ia, ib, r_max=6.0, nbins=60):
    """g(r) between particle sets ia and ib of one replica (minimum image),
    normalised by the ideal-gas pair density."""
    from scipy.spatial import cKDTree
    xa = np.mod(x[ia], box)
    xb = np.mod(x[ib], box)
    tree = cKDTree(xb, boxsize=box)
    pairs = tree.query_ball_point(xa, r_max, return_sorted=False)
    d = []
    for k, lst in enumerate(pairs):
        if lst:
            dv = xb[lst] - xa[k]
            dv -= box * np.round(dv / box)
            d.append(np.linalg.norm(dv, axis=1))
    d = np.concatenate(d) if d else np.zeros(0)
    d = d[d > 1e-9]
    hist, edges = np.histogram(d, bins=nbins, range=(0.0, r_max))
    shell = 4.0 / 3.0 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    ideal = len(ia) * len(ib) / box ** 3 * shell
    return 0.5 * (edges[1:] + edges[:-1]), hist / ideal


def run_pe_sweep(args):
    """Batched polyelectrolyte salt sweep (config 5): 64 replicas of 200
    FENE chains x 100 beads (all -1), +1 counterions, salt ions at 0.001-0.5
    (40k-150k particles each), WCA + P3M at accuracy 1e-4, Langevin
    kT 1, dt 0.01, one CUDA graph per step, in FP32-mixed and in FP64.
    Reports the step rates, the total-energy drift of a velocity-Verlet
    (gamma 0) continuation per replica, and the monomer-counterion g(r) of
    the FP32-mixed run against the FP64 run for the lowest- and highest-salt
    replicas."""
    import torch
    from espresso_b200 import _lib
    P = ctypes.POINTER
    lib = _lib.load()
    torch.cuda.set_device(0)
    boxes, prefs, pos, q, offs, bonds, salts = make_pe_sweep(n_rep=args.replicas
                                                             if args.replicas != 512 else 64)
    R = len(prefs)
    n = len(q)
    types = np.zeros(n, dtype=np.int32)
    tab = (_lib.PairParams * 1)()
    tab[0].wca_eps = 1.0
    tab[0].wca_sig = 1.0
    fene = (_lib.BondParams * 1)()
    fene[0] = _lib.BondParams(_lib.P3MX_BOND_FENE, 30.0, 0.0, 1.5)
    bl = np.ascontiguousarray(bonds.reshape(-1))
    results = {}
    for label, single in (("f32_mixed", 1), ("f64", 0)):
        d = _lib.BatchDesc()
        d.n_rep = R
        d.box = boxes.ctypes.data_as(P(ctypes.c_double))
        d.prefactor = prefs.ctypes.data_as(P(ctypes.c_double))
        d.offset = offs.ctypes.data_as(P(ctypes.c_longlong))
        d.accuracy = args.accuracy
        d.skin = args.skin if args.skin is not None else 0.4
        d.single_precision = single
        # meshes up to 128: at 40k-150k ions in a box of 48 the real-space
        # cutoff a 64^3 mesh would need makes the Verlet lists outgrow HBM
        d.mesh_min, d.mesh_max, d.cao_min, d.cao_max = 16, 128, 3, 7
        h = ctypes.c_void_p()
        t0 = time.perf_counter()
        rc = lib.p3mx_batch_create(ctypes.byref(d), pos.ctypes.data_as(P(ctypes.c_double)),
                                   q.ctypes.data_as(P(ctypes.c_double)),
                                   types.ctypes.data_as(P(ctypes.c_int)), 1, tab, ctypes.byref(h))
        if rc:
            raise RuntimeError(lib.p3mx_batch_last_error(h).decode())
        t_tune = time.perf_counter() - t0
        _lib.check(lib.p3mx_batch_set_bonds(h, 1, fene, len(bonds),
                                            bl.ctypes.data_as(P(ctypes.c_int))), h,
                   lib.p3mx_batch_last_error)
        stream = torch.cuda.ExternalStream(lib.p3mx_batch_stream(h))
        # relax the lattice start, then time Langevin steps
        _lib.check(lib.p3mx_batch_run(h, max(args.warmup, 50), 0.005, 1.0, 1.0, 11), h,
                   lib.p3mx_batch_last_error)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        _lib.check(lib.p3mx_batch_run(h, args.steps, 0.01, 1.0, 1.0, 11), h,
                   lib.p3mx_batch_last_error)
        e1.record(stream)
        torch.cuda.synchronize()
        t_ms = e0.elapsed_time(e1) / args.steps

        def energies():
            ep = np.zeros(R)
            _lib.check(lib.p3mx_batch_forces(h, ep.ctypes.data_as(P(ctypes.c_double))), h,
                       lib.p3mx_batch_last_error)
            v = np.zeros((n, 3))
            x = np.zeros((n, 3))
            _lib.check(lib.p3mx_batch_get(h, x.ctypes.data_as(P(ctypes.c_double)), None,
                                          v.ctypes.data_as(P(ctypes.c_double))), h,
                       lib.p3mx_batch_last_error)
            ek = np.array([0.5 * (v[offs[r]:offs[r + 1]] ** 2).sum() for r in range(R)])
            return ep + ek, ek, x
        # energy drift: velocity Verlet without thermostat (gamma 0, kT 0)
        et0, ek0, x_end = energies()
        n_nve = 100
        _lib.check(lib.p3mx_batch_run(h, n_nve, 0.005, 0.0, 0.0, 11), h, lib.p3mx_batch_last_error)
        et1, _, _ = energies()
        drift = np.abs(et1 - et0) / (ek0 + 1e-300)
        results[label] = {"ms_per_step": t_ms, "value": n / (t_ms * 1e-3), "tuning_s": t_tune,
                          "nve_steps": n_nve, "nve_dt": 0.005,
                          "energy_drift_rel_to_kinetic_max": float(drift.max()),
                          "energy_drift_rel_to_kinetic_median": float(np.median(drift)),
                          "x": x_end}
        lib.p3mx_batch_destroy(h)
    gr = {}
    for r in (0, R - 1):
        a0, a1 = int(offs[r]), int(offs[r + 1])
        nb = 200 * 100
        mono = np.arange(a0, a0 + nb)
        ci = np.arange(a0 + nb, a0 + 2 * nb)
        g = [radial_distribution(results[k]["x"], boxes[r][0], mono, ci)[1]
             for k in ("f32_mixed", "f64")]
        m = g[1] > 0.2
        gr[f"replica_{r}_salt_{salts[r]:.3g}"] = {
            "max_abs_diff_g_mono_ci": float(np.abs(g[0] - g[1])[m].max()),
            "peak_g_f32_mixed": float(g[0].max()), "peak_g_f64": float(g[1].max())}
    for k in results:
        results[k].pop("x")
    print(json.dumps({
        "metric": "particle-steps/s", "impl": "ours", "workload": "pe_sweep",
        "value": results["f32_mixed"]["value"], "unit": "particle-steps/s", "n_gpus": 1,
        "steps": args.steps, "ms_per_step": results["f32_mixed"]["ms_per_step"],
        "higher_is_better": True, "dtype": "f32-mixed (f64 positions/accumulators)",
        "data": "synthetic", "paths": results, "g_r": gr,
        "config": {"workload": f"batched polyelectrolyte salt sweep: {R} replicas of 200 FENE "
                               f"chains x 100 beads (all -1), +1 counterions, "
                               f"salt ions {salts[0]:g}-{salts[-1]:g}, box "
                               f"{boxes[0][0]:.2f}, {n} particles, WCA, P3M accuracy "
                               f"{args.accuracy:g} (meshes 16-128, cao 3-7 autotuned per "
                               f"replica), Langevin kT 1 dt 0.01, one CUDA graph per step",
                   "total_particles": int(n)}}))


def run_elc(args):
    """Slab workload: the single-system ions (density 0.5, LJ 2.5) shifted
    into z in [0.3, box + 0.7) of a box box x box x (box + 1 + gap), P3M over
    the whole box plus the electrostatic layer correction (maxPWerror =
    accuracy); forces only through p3mx_forces with device pointers.  Prints
    one JSON line: the step rate with ELC, the same system without ELC, and
    the ELC stage times with the mode count."""
    import torch
    import espresso_b200 as eb
    from espresso_b200 import _lib
    from espresso_b200.electrostatics import ELC, P3M, P3MGPU

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    pos, q, box = make_workload(seed=0, box=args.box)
    pos = pos - np.floor(pos / box) * box
    pos[:, 2] += 0.3
    n = len(q)
    lz = box + 1.0 + args.gap
    boxv = [box, box, lz]
    # the z mesh at the x-y spacing, rounded to a multiple of 32 (FFT-friendly)
    mz = int(round(args.mesh * lz / box / 32.0)) * 32
    cls = P3M if args.fp64 else P3MGPU
    act = cls(prefactor=1.0, accuracy=args.accuracy, mesh=[args.mesh, args.mesh, mz],
              cao=args.cao, r_cut=args.r_cut, tune=True, timings=2, verbose=False)
    s = eb.System(box_l=boxv)
    s.time_step = 0.01
    s.cell_system.skin = args.skin if args.skin is not None else 0.4
    s.part.add(pos=pos, q=q)
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5,
                                                      shift="auto")
    pos_d = torch.from_numpy(pos).to(dev)
    q_d = torch.from_numpy(q).to(dev)
    t_d = torch.zeros(n, dtype=torch.int32, device=dev)
    f_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    flags = _lib.P3MX_DEVICE_PTRS | _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE

    def timed(h):
        def step():
            _lib.check(lib.p3mx_forces(h, n, _lib.dptr(pos_d), _lib.dptr(q_d), _lib.dptr(t_d),
                                       _lib.dptr(f_d), None, None, flags, sp), h)
        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    s.electrostatics.solver = act
    s._sync_pairs(act._handle, np.zeros(n, dtype=np.int32))
    t_p3m = timed(act._handle)
    elc = ELC(actor=act, maxPWerror=args.accuracy, gap_size=args.gap)
    s.electrostatics.solver = elc
    h = elc._handle
    s._sync_pairs(h, np.zeros(n, dtype=np.int32))
    with ClockSampler(0) as clk:
        t_elc = timed(h)
    names = (ctypes.c_char_p * 40)()
    ms = (ctypes.c_double * 40)()
    nst = ctypes.c_int()
    _lib.check(lib.p3mx_profile(h, 5, ms, names, 40, ctypes.byref(nst)), h)
    stages = {names[k].decode(): ms[k] for k in range(nst.value)}
    fcd = ctypes.c_double()
    nm = ctypes.c_int()
    _lib.check(lib.p3mx_get_elc(h, ctypes.byref(fcd), None, ctypes.byref(nm)), h)
    fc, nmodes = fcd.value, nm.value
    elc_ms = sum(v for k, v in stages.items() if k.startswith("elc_"))
    out = {
        "metric": "particle-steps/s", "impl": "ours", "workload": "elc",
        "value": n / (t_elc * 1e-3), "unit": "particle-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_elc,
        "ms_per_step_without_elc": t_p3m, "higher_is_better": True,
        "dtype": "f64" if args.fp64 else "f32-mixed (ELC f64)", "data": "synthetic",
        "stages_ms": stages,
        "elc": {"modes": nmodes, "far_cut": fc, "ms": elc_ms,
                "mode_particle_evals_per_s": 2.0 * nmodes * n / (elc_ms * 1e-3)},
        "clocks": clk.summary(),
        "config": {"workload": f"slab: {n} ions, density 0.5, box {box:g}^2 x {lz:g} "
                               f"(gap {args.gap:g}), LJ 2.5, P3M mesh {args.mesh}^2 x {mz}, "
                               f"cao {args.cao}, r_cut {args.r_cut}, accuracy {args.accuracy:g}, "
                               f"ELC maxPWerror {args.accuracy:g}",
                   "inputs": "resident in HBM, larger than L2"},
    }
    print(json.dumps(out))


def run_dipolar(args):
    """Point-dipole workload: N dipoles of unit moment, random orientations,
    on a jittered lattice at number density 0.5 (cubic box), dipolar P3M
    tuned for accuracy 1e-4 (DipolarTuningAlgorithm: mesh, cao, r_cut,
    alpha; outside the timed region), FP64 and FP32 paths (``fp32_mesh``:
    FP32 mesh, FFT and real-space pair terms, FP64 sums).  One step =
    one evaluation of forces and torques (k-space + real space) through
    p3mx_dp3m_compute with device pointers; e2e = the same through pinned
    host arrays (positions and moments in, forces and torques out).  Prints
    one JSON line."""
    line = dipolar_measure(args, int(args.dipoles), args.steps, args.warmup)
    if line is not None:
        print(json.dumps(line))


def dipolar_measure(args, n, steps, warmup):
    """The dipolar workload's measurement (see run_dipolar): the JSON line,
    or None under --profile-only."""
    import torch
    from espresso_b200 import _lib
    from espresso_b200.magnetostatics import DipolarP3M

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = (n / 0.5) ** (1.0 / 3.0)
    rng = np.random.default_rng(0)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    g = np.stack(np.meshgrid(*(np.arange(side),) * 3, indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = (g + 0.5 + rng.uniform(-0.2, 0.2, (n, 3))) * (L / side)
    dip = rng.normal(size=(n, 3))
    dip /= np.linalg.norm(dip, axis=1, keepdims=True)
    pos_d = torch.from_numpy(pos).to(dev)
    dip_d = torch.from_numpy(dip).to(dev)
    f_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    t_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    pos_h = torch.from_numpy(pos).pin_memory()
    dip_h = torch.from_numpy(dip).pin_memory()
    f_h = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    t_h = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    out = {}
    for label, sprec in (("fp64", False), ("fp32_mesh", True)):
        if args.profile_only:
            # the parameters the tuner chose for 2^17 dipoles in a plain run
            # (timings under a profiler would mislead the tuner)
            act = DipolarP3M(prefactor=1.0, accuracy=1e-4, single_precision=sprec, tune=False,
                             mesh=112, cao=7, r_cut=4.70, alpha=0.718)
        else:
            act = DipolarP3M(prefactor=1.0, accuracy=1e-4, single_precision=sprec, timings=2,
                             verbose=False)
        act._set_system([L] * 3, args.skin if args.skin is not None else 0.4, (True,) * 3)
        act._activate(pos, dip)
        h = act._handle
        flags = _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE
        if args.profile_only:
            # three evaluations inside a profiler range (ncu --profile-from-start
            # off captures them without the tuner's trial launches)
            torch.cuda.synchronize(dev)
            torch.cuda.profiler.start()
            for _ in range(3):
                _lib.check(lib.p3mx_dp3m_compute(h, n, _lib.dptr(pos_d), _lib.dptr(dip_d),
                                                 _lib.dptr(f_d), _lib.dptr(t_d), None,
                                                 flags | _lib.P3MX_DEVICE_PTRS, sp),
                           h, lib.p3mx_dp3m_last_error)
            torch.cuda.synchronize(dev)
            torch.cuda.profiler.stop()
            return None

        def step(device=True):
            if device:
                rc = lib.p3mx_dp3m_compute(h, n, _lib.dptr(pos_d), _lib.dptr(dip_d),
                                           _lib.dptr(f_d), _lib.dptr(t_d), None,
                                           flags | _lib.P3MX_DEVICE_PTRS, sp)
            else:
                rc = lib.p3mx_dp3m_compute(h, n, _lib.dptr(pos_h), _lib.dptr(dip_h),
                                           _lib.dptr(f_h), _lib.dptr(t_h), None, flags, sp)
            _lib.check(rc, h, lib.p3mx_dp3m_last_error)

        def timed(device):
            for _ in range(max(3, warmup)):
                step(device)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                step(device)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1) / steps

        l0 = ctypes.c_longlong()
        lib.p3mx_dp3m_launch_count(h, ctypes.byref(l0))
        with ClockSampler(0) as clk:
            ms = timed(True)
        l1 = ctypes.c_longlong()
        lib.p3mx_dp3m_launch_count(h, ctypes.byref(l1))
        ms_e2e = timed(False)
        names = (ctypes.c_char_p * 40)()
        sms = (ctypes.c_double * 40)()
        nst = ctypes.c_int()
        _lib.check(lib.p3mx_dp3m_profile(h, n, _lib.dptr(pos), _lib.dptr(dip), 5, sms, names, 40,
                                         ctypes.byref(nst)), h, lib.p3mx_dp3m_last_error)
        stages = {names[k].decode(): round(sms[k], 4) for k in range(min(40, nst.value))}
        p = act.get_params()
        out[label] = {"ms_per_step": ms, "value": n / (ms * 1e-3),
                      "e2e": {"value": n / (ms_e2e * 1e-3), "unit": "dipole-steps/s",
                              "ms_per_step": ms_e2e, "h2d_bytes_per_step": 48 * n,
                              "d2h_bytes_per_step": 48 * n},
                      "gpu_launches_per_step": (l1.value - l0.value) / max(1, steps),
                      "stages_ms": stages,
                      "tuned": {"mesh": p["mesh"][0], "cao": p["cao"], "r_cut": p["r_cut"],
                                "alpha": p["alpha"], "accuracy_estimate": p["accuracy"]},
                      "clocks": clk.summary()}
    line = {
        "metric": "dipole-steps/s (dipolar P3M forces + torques at accuracy 1e-4)",
        "impl": "ours", "workload": "dipolar", "value": out["fp64"]["value"],
        "unit": "dipole-steps/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": out["fp64"]["ms_per_step"], "higher_is_better": True, "dtype": "f64",
        "data": "synthetic", "e2e": out["fp64"]["e2e"], "variants": out,
        "config": {"workload": f"{n} unit point dipoles, random orientations, density 0.5, "
                               f"box {L:.4g}^3, dipolar P3M tuned for accuracy 1e-4",
                   "inputs": "resident in HBM, larger than L2 with the Verlet lists"},
    }
    return line


def main():
    args = parse()
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "elc":
        run_elc(args)
        return
    if args.workload == "melt":
        run_melt(args)
        return
    if args.workload == "pe_sweep":
        run_pe_sweep(args)
        return
    if args.workload == "dipolar":
        run_dipolar(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    import espresso_b200 as eb
    from espresso_b200 import _lib
    from espresso_b200.electrostatics import P3M, P3MGPU

    lib = _lib.load()
    pos, q, box = make_workload(seed=rank, box=args.box)
    n = len(q)
    cls = P3M if args.fp64 else P3MGPU
    if args.profile_only:
        # ncu captures: the alpha the tuner would pick (same error formula),
        # without the tuner's timed trials before the captured launches
        act = cls(prefactor=1.0, accuracy=args.accuracy, mesh=args.mesh, cao=args.cao,
                  r_cut=args.r_cut, alpha=tuned_alpha(args, n, float(np.sum(q * q)), box),
                  tune=False)
    else:
        act = cls(prefactor=1.0, accuracy=args.accuracy, mesh=args.mesh, cao=args.cao,
                  r_cut=args.r_cut, tune=True, timings=2, verbose=False)
    s = eb.System(box_l=[box] * 3)
    s.time_step = 0.01
    s.cell_system.skin = args.skin if args.skin is not None else 0.4
    s.part.add(pos=pos, q=q)
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5,
                                                      shift="auto")
    s.electrostatics.solver = act
    prm = act.get_params()
    h = act._handle
    types = np.zeros(n, dtype=np.int32)
    s._sync_pairs(h, types)
    dev = torch.device("cuda", local)
    pos_d = torch.from_numpy(pos).to(dev)
    q_d = torch.from_numpy(q).to(dev)
    t_d = torch.from_numpy(types).to(dev)
    f_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    flags = _lib.P3MX_DEVICE_PTRS | _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE

    def step():
        rc = lib.p3mx_forces(h, n, _lib.dptr(pos_d), _lib.dptr(q_d), _lib.dptr(t_d), _lib.dptr(f_d),
                             None, None, flags, sp)
        if rc:
            _lib.check(rc, h)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize(dev)
    if args.profile_only:
        for _ in range(2):
            step()
        torch.cuda.synchronize(dev)
        return
    # stage profile (CUDA events between stages, same stream as the launches)
    names = (ctypes.c_char_p * 32)()
    ms = (ctypes.c_double * 32)()
    nst = ctypes.c_int()
    _lib.check(lib.p3mx_profile(h, 5, ms, names, 32, ctypes.byref(nst)), h)
    stages = {names[k].decode(): ms[k] for k in range(nst.value)}
    # timed comparison (not used by the path): cuFFT through torch.fft on the
    # same mesh, one r2c and three c2r transforms as one force evaluation
    # needs, against the hand-written FFT stages above
    cufft_ms = None
    if rank == 0 and not args.fp64:
        M = args.mesh
        xr = torch.randn((M, M, M), dtype=torch.float32, device=dev)
        xc = torch.fft.rfftn(xr)
        for _ in range(3):
            torch.fft.rfftn(xr)
            torch.fft.irfftn(xc, s=(M, M, M))
        torch.cuda.synchronize(dev)
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record()
        for _ in range(5):
            torch.fft.rfftn(xr)
            for _ in range(3):
                torch.fft.irfftn(xc, s=(M, M, M))
        c1.record()
        torch.cuda.synchronize(dev)
        cufft_ms = c0.elapsed_time(c1) / 5
        del xr, xc
        torch.cuda.empty_cache()
    # rebuild cost: one evaluation with a forced Verlet rebuild
    lc0 = ctypes.c_longlong()
    lc1 = ctypes.c_longlong()
    # timed region
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    lib.p3mx_launch_count(h, ctypes.byref(lc0))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    lib.p3mx_launch_count(h, ctypes.byref(lc1))
    if dist is not None:
        dist.barrier()
    t_ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        tt = torch.tensor([t_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = n * world / (t_ms * 1e-3)

    # end to end through the C ABI with host buffers (pinned staging inside)
    pos_h = np.ascontiguousarray(pos)
    q_h = np.ascontiguousarray(q)
    f_h = np.zeros((n, 3))
    hflags = _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE

    def step_host():
        rc = lib.p3mx_forces(h, n, _lib.dptr(pos_h), _lib.dptr(q_h), _lib.dptr(types),
                             _lib.dptr(f_h), None, None, hflags, sp)
        if rc:
            _lib.check(rc, h)

    for _ in range(3):
        step_host()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    k_e2e = max(5, args.steps // 2)
    for _ in range(k_e2e):
        step_host()
    torch.cuda.synchronize(dev)
    t_e2e = (time.perf_counter() - t0) / k_e2e
    if dist is not None:
        tt = torch.tensor([t_e2e], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = n * world / t_e2e

    # Verlet rebuild at the headline size: a resort makes the next force
    # evaluation rebuild the cell and Verlet lists; the stage profile times
    # the rebuild between CUDA events (outside the timed region)
    _lib.check(lib.p3mx_resort(h), h)
    names_r = (ctypes.c_char_p * 32)()
    ms_r = (ctypes.c_double * 32)()
    nst_r = ctypes.c_int()
    _lib.check(lib.p3mx_profile(h, 1, ms_r, names_r, 32, ctypes.byref(nst_r)), h)
    prof_r = {names_r[k].decode(): ms_r[k] for k in range(nst_r.value)}
    verlet_rebuild_ms = prof_r.get("sr_rebuild")

    # FP32-mixed vs FP64 electrostatic forces (k-space + real-space Coulomb,
    # LJ switched off on both actors) on the same configuration
    fp_diff = None
    f_rms = None
    ewald_acc = None
    variants = {}
    if not args.fp64:
        zero_tab = (_lib.PairParams * 1)()
        ref_act = P3M(prefactor=1.0, accuracy=args.accuracy, mesh=args.mesh, cao=args.cao,
                      r_cut=args.r_cut, alpha=prm["alpha"], tune=False)
        s.electrostatics.clear()
        s.electrostatics.solver = ref_act
        res = []
        for hh in (h, ref_act._handle):
            _lib.check(lib.p3mx_set_pair_params(hh, 1, zero_tab), hh)
            ff = np.zeros((n, 3))
            _lib.check(lib.p3mx_forces(hh, n, _lib.dptr(pos_h), _lib.dptr(q_h), _lib.dptr(types),
                                       _lib.dptr(ff), None, None, hflags, None), hh)
            res.append(ff)
        fp_diff = float(np.sqrt(((res[0] - res[1]) ** 2).sum(1).mean()))
        f_rms = float(np.sqrt((res[1] ** 2).sum(1).mean()))
        if rank == 0 and not args.no_ewald:
            ewald_acc = ewald_accuracy(pos, q, box, prm["alpha"], args, res[0], res[1])
        if rank == 0 and not args.no_variants:
            # plain FP64 GPU path on the same workload (LJ back on)
            s._sync_pairs(ref_act._handle, types)
            s._sync_pairs(h, types)
            variants["fp64_single"] = time_single_variant(
                lib, ref_act._handle, n, pos_d, q_d, t_d, f_d, stream, sp, args)
        del ref_act

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    hbm, hbm_kind = peaks()
    # roofline of the dominant stage
    N = n
    M3 = float(args.mesh) ** 3
    K = args.mesh * args.mesh * (args.mesh // 2 + 1)
    c = args.cao
    rc_eff = args.r_cut + 0.4
    nb_full = 4.18879 * rc_eff ** 3 * 0.5
    bytes_alg = {
        "p3m_assign": 28 * N + 4 * M3,
        "p3m_interp": 28 * N + 12 * M3 + 24 * N,
        "fft_fwd_zy": 4 * M3 + 8 * K + 8 * K + 8 * K,
        "fft_x_kspace": 8 * K + 4 * K + 3 * 8 * K,
        "fft_inv_yz": 3 * (8 * K + 8 * K) + 3 * (8 * K + 4 * M3),
        "pair_forces": N * nb_full * 4 + 32 * N + 24 * N,
        "p3m_sort": 2 * (24 + 4 + 4) * N + 8 * M3,
        "p3m_weights": 24 * N + 8 * N + 3 * 4 * c * N,
    }
    dom = max(stages, key=stages.get)
    dom_ms = stages[dom]
    alg = bytes_alg.get(dom)
    achieved = alg / (dom_ms * 1e-3) / 1e9 if alg else None
    traffic = ncu_traffic().get(dom)
    flops_alg = {"p3m_assign": 2 * c ** 3 * N + 30 * c * N, "p3m_interp": 6 * c ** 3 * N,
                 "pair_forces": N * nb_full * 8 + N * 0.5 * 4.18879 * args.r_cut ** 3 * 25}
    fp32 = None
    if dom in flops_alg:
        tf = flops_alg[dom] / (dom_ms * 1e-3) / 1e12
        fp32 = {"achieved": tf, "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                "frac": tf / FP32_NOMINAL_TFLOPS, "peak_kind": "nominal 148 SM x 128 x 2 x 1965 MHz"}
    cpu = None
    if not args.no_cpu_baseline:
        ncores = os.cpu_count() or 1
        tab = lj_table_oracle()
        t_cpu = cpu_reference_step(pos, q, box, args.mesh, args.cao, prm["alpha"], args.r_cut, tab)
        cpu = {"value": n / t_cpu, "unit": "particle-steps/s", "cores": ncores, "kind": "port",
               "sample": "one full force evaluation of the same workload on the FP64 CPU "
                         "restatement of the reference path (OpenMP, all host cores)"}
    n_launch = lc1.value - lc0.value
    if not args.no_variants and not args.fp64 and world == 1:
        # the 512-replica batched step (config 4), after the single-system
        # engines' work is done
        del act
        s.electrostatics.clear()
        torch.cuda.synchronize(dev)
        try:
            b = batched_measure(args, max(args.variant_steps, 20), 3, cpu=False, clocks=True)
            variants["batched_f32_mixed"] = {
                k: b[k] for k in ("value", "unit", "ms_per_step", "steps", "stages_ms", "config",
                                  "clocks", "gpu_launches")}
            sb = b["stages_ms"]
            dom_b = max(sb, key=sb.get)
            variants["batched_f32_mixed"]["dominant_stage"] = {"kernel": dom_b, "ms": sb[dom_b]}
        except Exception as exc:  # reported, not hidden
            variants["batched_f32_mixed"] = {"error": str(exc)}
        # dipolar P3M (the magnetostatics actor on the same kernels): 2^17
        # unit dipoles, tuned for accuracy 1e-4, FP64 and FP32 mesh
        try:
            dl = dipolar_measure(args, 1 << 17, max(args.variant_steps, 10), 3)
            variants["dipolar_p3m"] = {
                "config": dl["config"]["workload"], "unit": "dipole-steps/s",
                **{k: {kk: v[kk] for kk in ("value", "ms_per_step", "tuned", "stages_ms",
                                            "gpu_launches_per_step")}
                   for k, v in dl["variants"].items()}}
        except Exception as exc:  # reported, not hidden
            variants["dipolar_p3m"] = {"error": str(exc)}
    out = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.fp64 else "f32-mixed (f64 positions/accumulators)",
        "data": "synthetic", "config": config_dict(args, n, prm["alpha"], world),
        "e2e": {"value": e2e, "unit": "particle-steps/s",
                # positions cross PCIe every step; charges and types are
                # compared with the staged copy of the previous call and sent
                # only when changed (they do not change here)
                "h2d_bytes_per_step": int(n * 24), "d2h_bytes_per_step": int(n * 24),
                "host_inputs_bytes_per_step": int(n * (24 + 8 + 4))},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                     "traffic": traffic, "peak_kind": hbm_kind,
                     "algorithmic_bytes": alg, "launch_ms": dom_ms, "fp32": fp32},
        "stages_ms": stages,
        "fft_comparison": None if cufft_ms is None else {
            "cufft_r2c_plus_3_c2r_ms": cufft_ms,
            "own_fft_stages_ms": stages.get("fft_fwd_zy", 0) + stages.get("fft_x_kspace", 0) +
                                 stages.get("fft_inv_yz", 0),
            "note": "own stages include the influence function, ik-differentiation, "
                    "energy/virial sums and the packed field-mesh output"},
        "accuracy": {"rms_force_err_estimate": prm["accuracy"],
                     "fp32_vs_fp64_rms_coulomb_force_diff": fp_diff,
                     "rms_coulomb_force": f_rms, **(ewald_acc or {})},
        "verlet_rebuild_ms": verlet_rebuild_ms,
        "variants": variants or None,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(n_launch),
    }
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
