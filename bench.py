"""Benchmark of the two-electron hot path on B200.

Workload: (H2O)_16 on the 2.9 A cubic lattice with seeded rotations,
6-31G* Cartesian basis (304 functions, 160 shells), Schwarz
threshold 1e-12.  One step = one direct FP64 J/K Fock build (fused MMD ERI +
J/K digestion, the plain kernel) from the core-guess density.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  ``value`` = Schwarz-surviving canonical shell quartets
per second (all ranks), device-timed with CUDA events, L2 flushed between
steps.  ``e2e`` = the same metric through the C ABI entry point with the
density in pinned host memory and J/K copied back every step.  ``roofline``
= the dominant class kernel's model FLOP rate against the FP64 FMA peak
measured in the same run.  ``cpu_baseline`` = the CPU oracle (a C
restatement of the reference algorithm) on a bounded random sample of the
same quartets, all host cores.  ``--impl reference`` times that CPU
implementation as the reference arm.  ``fock_gradient`` reports the
end-to-end SCF Fock-build seconds of the plain FP64 path against the chosen
(mixed-precision, incremental) path and the energy difference.

N > 1 runs (torchrun, one rank per GPU) are weak-scaling replicas: every
rank builds its own seeded cluster; there is no collective on the data path.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_WATERS = int(os.environ.get("JQC_BENCH_WATERS", "16"))
BASIS = "6-31g*"
SCHWARZ_TAU = 1e-12
# density-screening threshold of the chosen (mixed) path's gradient (the
# batched path's MIXED_GRAD_TAU): skipped quartets change the (H2O)16
# gradient by 3.0e-6 Eh/bohr, a 3x margin to the 1e-5 tolerance
CHOSEN_GRAD_TAU = 1e-9
METRIC = "ERI quartets/s (direct J/K Fock build, (H2O)16 6-31G*)"
WORKLOAD = (f"(H2O){N_WATERS} lattice 2.9A, 6-31G* Cartesian ({19 * N_WATERS} bf), "
            "FP64 direct J/K build")


def _dist():
    from jax_examples_b200.dist import env_ranks

    return env_ranks()


# ------------------------------------------------------------------- CPU leg
def cpu_sample(seed: int = 0, sample: int = 6000, mode: int = 0):
    """Time the oracle's J/K digestion of a random sample of surviving
    canonical quartets of the workload; returns (quartets/s, threads, desc)."""
    import oracle
    from jax_examples_b200 import basis as pb

    mol = pb.water_cluster(N_WATERS, seed=seed)
    bs = pb.build_basis_set(mol, BASIS)
    pk = oracle.Packed(bs)
    Q = oracle.schwarz(pk, mode=1)
    ns = pk.n_shell
    rng = np.random.default_rng(1234 + seed)
    iu = np.array([(i, j) for i in range(ns) for j in range(i + 1)], dtype=np.int64)
    qv = Q[iu[:, 0], iu[:, 1]]
    chunks, have = [], 0
    while have < sample:
        m = min(4 * sample, 1 << 21)
        a = rng.integers(0, len(iu), m)
        b = rng.integers(0, len(iu), m)
        keep = (a >= b) & (qv[a] * qv[b] >= SCHWARZ_TAU)
        chunks.append(np.concatenate([iu[a[keep]], iu[b[keep]]], axis=1))
        have += int(keep.sum())
    quart = np.ascontiguousarray(np.concatenate(chunks)[:sample], dtype=np.int32)
    n = pk.n
    D = np.eye(n) * 0.1
    t0 = time.perf_counter()
    oracle.jk_quartets(pk, D, quart, mode=mode)
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return sample / dt, threads, f"{sample} random Schwarz-surviving canonical quartets of the workload, {dt:.1f}s"


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    vals = []
    for _ in range(args.warmup):
        cpu_sample(sample=2000)
    for _ in range(args.steps):
        v, cores, desc = cpu_sample(sample=args.ref_sample)
        vals.append(v)
    value = float(np.mean(vals))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": "quartets/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ GPU leg
class Clocks:
    def __init__(self, path):
        self.path = path
        self.p = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            self.p.wait()
            self.f.close()

    def summary(self, gpu_index):
        try:
            rows = [r.split(", ") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [r for r in rows if len(r) >= 9 and r[0].strip() == str(gpu_index)]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


def batched_sweep(local: int, n_mol: int, seed: int = 2024):
    """Uneven-size geometry sweep: n_mol water clusters (1..12 waters,
    +-0.1 A Gaussian noise) through one batched, graph-replayed
    mixed-precision RHF (incremental builds, FP64 tail) + screened gradient,
    against the same molecules one at a time on the plain FP64 path (a full
    FP64 build every iteration, unscreened gradient: the reference's
    per-geometry loop shape).  Both paths' kernels are loaded by a warm-up
    on a few molecules first; gradients are timed on a second call (the
    first, also reported, builds the gradient work list on the host)."""
    import torch

    from jax_examples_b200 import CalcConfig, DirectERI, compute_integrals, run_scf
    from jax_examples_b200 import basis as pb
    from jax_examples_b200.batch import MIXED_GRAD_TAU, BatchedERI, MoleculeBatch, rhf_gradient_batch, run_rhf_batch
    from jax_examples_b200.grad import rhf_gradient

    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.integers(1, 13, n_mol)]
    mols = [pb.water_cluster(n, seed=seed + i, noise_angstrom=0.1) for i, n in enumerate(sizes)]
    cfg = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, incremental=False)
    chosen = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, precision="mixed", incremental=True)
    # warm-up of both paths on a few of the molecules: the kernels both use are
    # loaded before anything is timed
    wb = MoleculeBatch(mols[:4], BASIS)
    weng = BatchedERI(wb, schwarz_tau=SCHWARZ_TAU)
    wscf = run_rhf_batch(wb, chosen, engine=weng, use_graph=True, autotune=False)
    rhf_gradient_batch(wb, wscf, None, MIXED_GRAD_TAU)
    wscf.engine.close()
    weng2 = DirectERI(wb.bases[0], mols[0], device=local, schwarz_tau=SCHWARZ_TAU)
    wr = run_scf(mols[0], compute_integrals(mols[0], wb.bases[0], device=local, engine=weng2), cfg)
    rhf_gradient(mols[0], wr, engine=weng2)
    weng2.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = MoleculeBatch(mols, BASIS)
    t_ctx = time.perf_counter()
    beng = BatchedERI(batch, schwarz_tau=SCHWARZ_TAU)
    torch.cuda.synchronize()
    t_ctx = time.perf_counter() - t_ctx
    # untuned launch shapes: on this sweep the autotuner saves 2% of the Fock
    # seconds (0.605 against 0.617 s) for 1.6-5.2 s of tuning, which pays
    # back only over many sweeps through its cache file
    scf = run_rhf_batch(batch, chosen, engine=beng, use_graph=True, autotune=False)
    # the first gradient call also builds the gradient work list on the host;
    # the second is the kernel time (both sides are timed that way)
    first = {}
    rhf_gradient_batch(batch, scf, first, MIXED_GRAD_TAU)
    timing = {}
    grads = rhf_gradient_batch(batch, scf, timing, MIXED_GRAD_TAU)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    rec = scf.record
    scf.engine.close()
    fock_seq = grad_seq = grad_seq_first = 0.0
    e_err = g_err = 0.0
    iters = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m, mol in enumerate(mols):
        eng = DirectERI(batch.bases[m], mol, device=local, schwarz_tau=SCHWARZ_TAU)
        ints = compute_integrals(mol, batch.bases[m], device=local, engine=eng)
        r = run_scf(mol, ints, cfg)
        fock_seq += r.precision["jk_seconds"]
        iters.append(r.n_iterations)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g = rhf_gradient(mol, r, engine=eng)
        e1.record()
        e1.synchronize()
        grad_seq_first += e0.elapsed_time(e1) * 1e-3
        e0.record()
        g = rhf_gradient(mol, r, engine=eng)
        e1.record()
        e1.synchronize()
        grad_seq += e0.elapsed_time(e1) * 1e-3
        e_err = max(e_err, abs(r.energy - scf.results[m].energy))
        g_err = max(g_err, float((g - grads[m]).abs().max()))
        eng.close()
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    return {
        "workload": f"{n_mol} water clusters, 1..12 waters (seeded), +-0.1 A noise, {BASIS}",
        "n_basis_total": batch.n_basis, "waters_total": int(sum(sizes)),
        "batched_mixed": {"fock_s": round(rec["jk_seconds"], 4), "gradient_s": round(timing["grad_seconds"], 4),
                          "gradient_first_call_s": round(first["grad_seconds"], 4),
                          "fock_builds": rec["fock_builds"],
                          "builds": {k: rec[k] for k in ("builds_mixed", "builds_fp64", "incremental_builds")},
                          "gradient_dens_tau": MIXED_GRAD_TAU, "setup_s": round(rec["setup_seconds"], 3),
                          "setup_breakdown_s": dict({k: round(v, 3) for k, v in rec["prepare_breakdown"].items()},
                                                    context_pairs=round(t_ctx, 3)),
                          "wall_s": round(t_batch, 3), "graph": rec["graph"], "autotuned": rec["autotuned"]},
        "sequential_fp64": {"fock_s": round(fock_seq, 4), "gradient_s": round(grad_seq, 4),
                            "gradient_first_calls_s": round(grad_seq_first, 4),
                            "iterations_mean": float(np.mean(iters)), "wall_s": round(t_seq, 3)},
        "fock_plus_gradient_speedup": round((fock_seq + grad_seq) / max(1e-12, rec["jk_seconds"]
                                                                         + timing["grad_seconds"]), 3),
        "wall_speedup": round(t_seq / max(1e-12, t_batch), 3),
        "max_energy_diff_eh": e_err, "max_gradient_diff_eh_bohr": g_err,
    }


def config3_scf(local: int, split_tau: float = 1e-7):
    """(H2O)8 on the lattice, 6-31G* Cartesian (152 bf): RHF-DIIS to 1e-8 Eh
    with the plain FP64 build every iteration against the mixed build with
    the FP32/FP64 Schwarz split at ``split_tau`` (and the package's default
    split beside it); iterations, Fock seconds and the energy error against
    FP64.  The same FP64 SCF in 6-31G** (200 bf) gives that basis's size and
    time."""
    import torch

    from jax_examples_b200 import CalcConfig, compute_integrals, run_scf
    from jax_examples_b200 import basis as pb

    mol = pb.water_cluster(8, seed=0)
    out = {"workload": "(H2O)8 lattice 2.9A, RHF-DIIS to 1e-8 Eh, Schwarz 1e-12"}
    for basis in ("6-31g*", "6-31g**"):
        bs = pb.build_basis_set(mol, basis)
        ints = compute_integrals(mol, bs, device=local, schwarz_tau=SCHWARZ_TAU)
        runs = [("fp64", CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, incremental=False))]
        if basis == "6-31g*":
            runs += [(f"mixed_split_{split_tau:g}", CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU,
                                                             precision="mixed", mixed_tau=split_tau)),
                     ("mixed_default", CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, precision="mixed"))]
        rows = {}
        for name, cfg in runs:
            run_scf(mol, ints, cfg)  # warm-up: work lists built, kernels loaded
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = run_scf(mol, ints, cfg)
            torch.cuda.synchronize()
            rows[name] = {"energy": r.energy, "iterations": r.n_iterations, "converged": r.converged,
                          "fock_s": round(r.precision["jk_seconds"], 4), "scf_s": round(time.perf_counter() - t0, 4),
                          "mixed_tau": cfg.mixed_tau if cfg.precision == "mixed" else None}
        e64 = rows["fp64"]["energy"]
        for name, row in rows.items():
            if name != "fp64":
                row["energy_err_eh"] = abs(row["energy"] - e64)
                row["fock_speedup"] = round(rows["fp64"]["fock_s"] / max(1e-12, row["fock_s"]), 3)
        out[basis] = dict(rows, n_bf=bs.n_basis)
        ints.ERI.close()
    return out


def _sequential_bfgs(local, mols, max_steps):
    """The reference's loop shape on the device: one molecule at a time, every
    BFGS evaluation a new engine, a plain FP64 SCF (full build every
    iteration) and the unscreened analytic gradient
    (geomopt/optimizer.py:55-76 per trial geometry)."""
    from jax_examples_b200 import CalcConfig, DirectERI, compute_integrals, run_scf
    from jax_examples_b200 import basis as pb
    from jax_examples_b200.batch import _bfgs_walker
    from jax_examples_b200.core import make_molecule
    from jax_examples_b200.grad import rhf_gradient

    cfg = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, incremental=False, max_scf_iter=200)
    out, evals = [], 0
    for mol in mols:
        w = _bfgs_walker(mol, max_steps, 1e-4, 1e-6, 0.3)
        xyz = w.send(None)
        while True:
            m = make_molecule(mol.elements, xyz, mol.atomic_numbers, charge=mol.charge, spin=mol.spin)
            bs = pb.build_basis_set(m, BASIS)
            eng = DirectERI(bs, m, device=local, schwarz_tau=SCHWARZ_TAU)
            r = run_scf(m, compute_integrals(m, bs, device=local, engine=eng), cfg)
            g = rhf_gradient(m, r, engine=eng).cpu().numpy()
            eng.close()
            evals += 1
            try:
                xyz = w.send((r.energy, g))
            except StopIteration as stop:
                out.append(stop.value)
                break
    return out, evals


def batched_bfgs(local: int, n_mol: int, steps: int = 10, seed: int = 2024, seq_every: int = 4):
    """The sweep's molecules (n_mol water clusters, 1..12 waters, +-0.1 A
    noise) optimised for ``steps`` BFGS steps each on the batched path: one
    engine for the whole optimisation, geometry-only updates
    between rounds, mixed precision with incremental builds, screened
    gradient.  Per-molecule energy and gradient error against FP64 at the
    final geometries (one batched plain-FP64 evaluation there).  Every
    ``seq_every``-th molecule is also optimised on the reference's loop shape
    (one molecule and one new engine per evaluation, plain FP64) and on the
    batched path alone, for the wall-clock comparison on the same subset."""
    import torch

    from jax_examples_b200 import CalcConfig
    from jax_examples_b200 import basis as pb
    from jax_examples_b200.batch import _BatchEvaluator, optimize_bfgs_batch

    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.integers(1, 13, n_mol)]
    mols = [pb.water_cluster(n, seed=seed + i, noise_angstrom=0.1) for i, n in enumerate(sizes)]
    chosen = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, precision="mixed", incremental=True,
                        max_scf_iter=200)
    plain = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, incremental=False, max_scf_iter=200)

    def run_batched(ms):
        tm = {}
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = optimize_bfgs_batch(ms, BASIS, max_steps=steps, config=chosen, autotune=False, timing=tm)
        torch.cuda.synchronize()
        return res, tm, time.perf_counter() - t0

    res, tm, wall = run_batched(mols)
    # FP64 at the final geometries: one batched plain evaluation
    ev = _BatchEvaluator([r.molecule for r in res], BASIS, plain)
    try:
        ref = ev({i: np.asarray(r.molecule.coords) for i, r in enumerate(res)})
    finally:
        ev.close()
    e_err = [abs(r.energy - ref[i][0]) for i, r in enumerate(res)]
    g_err = [float(np.abs(np.asarray(r.gradient) - ref[i][1]).max()) for i, r in enumerate(res)]
    sub = mols[::seq_every]
    sub_res, sub_tm, sub_wall = run_batched(sub)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq_res, seq_evals = _sequential_bfgs(local, sub, steps)
    torch.cuda.synchronize()
    seq_wall = time.perf_counter() - t0
    traj_de = max(abs(a.energy - b.energy) for a, b in zip(sub_res, seq_res))
    return {
        "workload": f"{n_mol} water clusters, 1..12 waters (seeded), +-0.1 A noise, {BASIS}, {steps} BFGS steps each",
        "bfgs_steps": steps,
        "batched_mixed": {"wall_s": round(wall, 3), "rounds": tm.get("rounds"), "evaluations": tm.get("evaluations"),
                          "fock_s": round(tm.get("jk_seconds", 0.0), 3),
                          "gradient_s": round(tm.get("grad_seconds", 0.0), 3),
                          "fock_builds": tm.get("fock_builds"),
                          "setup_s": round(tm.get("setup_seconds", 0.0), 3),
                          "setup_breakdown_s": {k: round(v, 3) for k, v in tm.get("prepare_breakdown", {}).items()},
                          "geometry_update_s": round(tm.get("geometry_update_seconds", 0.0), 3),
                          "steps_taken": [r.n_steps for r in res], "converged": sum(bool(r.converged) for r in res)},
        "max_energy_err_vs_fp64_eh": max(e_err), "max_gradient_err_vs_fp64_eh_bohr": max(g_err),
        "per_molecule_energy_err_eh": [float("%.3g" % x) for x in e_err],
        "per_molecule_gradient_err_eh_bohr": [float("%.3g" % x) for x in g_err],
        "subset": {"molecules": len(sub), "every": seq_every,
                   "batched_wall_s": round(sub_wall, 3), "batched_evaluations": sub_tm.get("evaluations"),
                   "sequential_fp64_wall_s": round(seq_wall, 3), "sequential_evaluations": seq_evals,
                   "wall_speedup": round(seq_wall / max(1e-12, sub_wall), 3),
                   "max_final_energy_diff_eh": traj_de},
    }


def sharded_sweep(local: int, rank: int, world: int, n_mol: int, seed: int = 2024):
    """The uneven-size sweep (n_mol water clusters, 1..12 waters, +-0.1 A
    noise) sharded over the ranks: each rank takes a contiguous,
    cost-balanced share (``dist.sweep_shard``) and runs it as its own batch on
    the chosen path (batched, graph-replayed, mixed + incremental,
    screened gradient).  No data-path collective; the times are the maximum
    over the ranks, from a barrier to the last rank's synchronize."""
    import torch

    from jax_examples_b200 import CalcConfig
    from jax_examples_b200 import basis as pb
    from jax_examples_b200 import dist as jdist
    from jax_examples_b200.batch import MIXED_GRAD_TAU, BatchedERI, MoleculeBatch, rhf_gradient_batch, run_rhf_batch

    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.integers(1, 13, n_mol)]
    mine = jdist.sweep_shard(sizes, rank, world)
    chosen = CalcConfig(scf_conv=1e-8, schwarz_tau=SCHWARZ_TAU, precision="mixed", incremental=True)
    mols = [pb.water_cluster(sizes[i], seed=seed + i, noise_angstrom=0.1) for i in mine]
    if mols:  # kernels loaded before the timed region
        wb = MoleculeBatch(mols[:2], BASIS)
        w = run_rhf_batch(wb, chosen, engine=BatchedERI(wb, schwarz_tau=SCHWARZ_TAU), use_graph=True)
        rhf_gradient_batch(wb, w, None, MIXED_GRAD_TAU)
        w.engine.close()
    torch.cuda.synchronize()
    jdist.barrier()
    t0 = time.perf_counter()
    fock = grad = 0.0
    if mols:
        batch = MoleculeBatch(mols, BASIS)
        scf = run_rhf_batch(batch, chosen, engine=BatchedERI(batch, schwarz_tau=SCHWARZ_TAU), use_graph=True,
                            autotune=False)
        tm = {}
        rhf_gradient_batch(batch, scf, tm, MIXED_GRAD_TAU)
        fock, grad = scf.record["jk_seconds"], tm["grad_seconds"]
        scf.engine.close()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return {"workload": f"{n_mol} water clusters, 1..12 waters (seeded), +-0.1 A noise, {BASIS}, "
                        f"energies and gradients, sharded over {world} GPUs by cost",
            "molecules_this_rank": len(mine), "waters_this_rank": int(sum(sizes[i] for i in mine)),
            "wall_s_max_over_ranks": round(jdist.max_over_ranks(wall), 3),
            "fock_s_max_over_ranks": round(jdist.max_over_ranks(fock), 4),
            "gradient_s_max_over_ranks": round(jdist.max_over_ranks(grad), 4),
            "molecules_per_s": round(n_mol / max(1e-12, jdist.max_over_ranks(wall)), 3)}


def kernel_configs(local: int):
    """The kernel-level configurations beside the Fock build: Boys
    throughput (2^24 T, half U[0,30], half log-U[1e-8,1e3], m = 0..8, FP64
    and FP32; HBM bound), primitive-quartet blocks of four classes (2^20
    random quartets each, exponents log-U[0.1,100], centres in a 4 A cube)
    and the (H2O)8 J/K build in 6-31G* (FP64 and mixed) and 6-31G**."""
    import torch

    from jax_examples_b200 import DirectERI, boys, eri_prim_quartets
    from jax_examples_b200 import basis as pb

    dev = torch.device("cuda", local)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    rng = np.random.default_rng(1)
    n = 1 << 24
    T = torch.tensor(np.concatenate([rng.uniform(0, 30, n // 2), 10 ** rng.uniform(-8, 3, n // 2)]), device=dev)
    out = {}
    for fp32 in (False, True):
        sec = timed(lambda: boys(T, 8, fp32=fp32))
        nbytes = n * 8 + n * 9 * (4 if fp32 else 8)
        out["boys_fp32" if fp32 else "boys_fp64"] = {
            "values_per_s": n * 9 / sec, "ms": round(sec * 1e3, 3), "gbs": nbytes / sec / 1e9,
            "hbm_frac": nbytes / sec / 1e9 / hbm}
    del T
    from jax_examples_b200 import flops
    from jax_examples_b200.engine import fp_peak

    classes = {"(ss|ss)": (0, 0, 0, 0), "(pp|pp)": (1, 1, 1, 1), "(dd|dd)": (2, 2, 2, 2), "(ds|ps)": (2, 0, 1, 0)}
    nq = 1 << 20
    prim = {}
    peak64 = fp_peak(False)
    for name, cls in classes.items():
        ex = torch.tensor(10 ** rng.uniform(-1, 2, (nq, 4)), device=dev)
        ctr = torch.tensor(rng.uniform(0, 4.0 / 0.529177210903, (nq, 4, 3)), device=dev)
        sec = timed(lambda: eri_prim_quartets(cls, ex, ctr), reps=2)
        ne = 1
        for l in cls:
            ne *= (l + 1) * (l + 2) // 2
        nbytes = nq * (16 + ne) * 8  # 4 exponents + 12 centre coordinates in, the block out
        tf = nq * flops.prim_quartet_flops(*cls) / sec / 1e12
        prim[name] = {"prim_quartets_per_s": nq / sec, "ms": round(sec * 1e3, 3), "gbs": round(nbytes / sec / 1e9, 1),
                      "hbm_frac": round(nbytes / sec / 1e9 / hbm, 3), "model_tflops": round(tf, 2),
                      "fp64_frac": round(tf / peak64, 3)}
        del ex, ctr
        torch.cuda.empty_cache()
    out["prim_quartets"] = prim
    h2o8 = {}
    for basis in ("6-31g*", "6-31g**"):
        mol = pb.water_cluster(8, seed=0)
        bs = pb.build_basis_set(mol, basis)
        eng = DirectERI(bs, mol, device=local, schwarz_tau=SCHWARZ_TAU)
        D = torch.eye(bs.n_basis, dtype=torch.float64, device=dev) * 0.1
        row = {"n_bf": bs.n_basis, "quartets": eng.stats("fp64")["quartets_fp64"]}
        row["fp64_ms"] = round(timed(lambda: eng.jk(D)) * 1e3, 3)
        if basis == "6-31g*":
            eng.stats("mixed", 1e-7)
            row["mixed_ms"] = round(timed(lambda: eng.jk(D, precision="mixed", mixed_tau=1e-7)) * 1e3, 3)
        h2o8[basis] = row
        eng.close()
    out["h2o8_jk"] = h2o8
    return out


def gradient_only(args):
    """ERI-derivative adjoint alone (the profiling case of the gradient
    kernels): core-guess density of the workload, --warmup untimed and
    --steps timed jqc_grad2e calls; prints per-class kernel times."""
    import torch

    from jax_examples_b200 import DirectERI
    from jax_examples_b200 import basis as pb
    from jax_examples_b200.engine import QUARTET_CLASSES
    from jax_examples_b200.grad import grad_two_electron

    mol = pb.water_cluster(N_WATERS, seed=0)
    bs = pb.build_basis_set(mol, BASIS)
    eng = DirectERI(bs, mol, device=0, schwarz_tau=SCHWARZ_TAU)
    S, T, V = eng.one_electron()
    w, U = torch.linalg.eigh(S)
    X = (U * (1.0 / torch.sqrt(w))[None, :]) @ U.T
    _, Cp = torch.linalg.eigh(X.T @ (T + V) @ X)
    C = X @ Cp
    nocc = mol.n_electrons // 2
    D = (2.0 * C[:, :nocc] @ C[:, :nocc].T).contiguous()
    for _ in range(max(1, args.warmup)):
        grad_two_electron(eng, [D], 1.0, 0.5)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        grad_two_electron(eng, [D], 1.0, 0.5)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = []
    grad_two_electron(eng, [D], 1.0, 0.5, 0.0, ms)
    print(json.dumps({"workload": WORKLOAD.replace("J/K build", "ERI-derivative adjoint"),
                      "gradient_ms": float(np.mean(times)),
                      "classes_ms": {"(%d%d|%d%d)" % QUARTET_CLASSES[q]: round(ms[q], 3) for q in range(21) if ms[q]}}))


def run_ours(args):
    import torch

    from jax_examples_b200 import CalcConfig, DirectERI, _abi, compute_integrals, run_scf
    from jax_examples_b200 import basis as pb
    from jax_examples_b200 import dist as jdist
    from jax_examples_b200 import flops
    from jax_examples_b200.engine import QUARTET_CLASSES, fp_peak

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    mol = pb.water_cluster(N_WATERS, seed=rank)
    bs = pb.build_basis_set(mol, BASIS)
    eng = DirectERI(bs, mol, device=local, schwarz_tau=SCHWARZ_TAU)
    st = eng.stats("fp64")
    nq = st["quartets_fp64"]
    S, T, V = eng.one_electron()
    H = T + V
    w, U = torch.linalg.eigh(S)
    X = (U * (1.0 / torch.sqrt(w))[None, :]) @ U.T
    _, Cp = torch.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    nocc = mol.n_electrons // 2
    D = (2.0 * C[:, :nocc] @ C[:, :nocc].T).contiguous()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        eng.jk(D)
    barrier()
    # --- device-timed region: K steps, L2 flushed before each
    times = []
    clk = Clocks(args.clock_log.format(rank=rank) if args.clock_log else
                 os.path.join(tempfile.gettempdir(), f"jqc_clocks_{os.getpid()}_{rank}.csv"))
    with clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.jk(D)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    barrier()
    ms = float(np.sum(times)) / args.steps
    ms_max = jdist.max_over_ranks(ms)
    value = nq * world / (ms_max * 1e-3)

    # --- end to end through the C ABI with host buffers
    n = eng.packed.n_cart
    D_h = D.cpu().pin_memory()
    J_h = torch.empty((2, n, n), dtype=torch.float64).pin_memory()
    D_d = torch.empty_like(D)
    J_d = torch.empty((1, n, n), dtype=torch.float64, device=dev)
    K_d = torch.empty_like(J_d)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def e2e_step():
        D_d.copy_(D_h, non_blocking=True)
        _abi.call("jqc_jk", eng._ctx, 1, ctypes.c_void_p(D_d.data_ptr()), ctypes.c_void_p(J_d.data_ptr()),
                  ctypes.c_void_p(K_d.data_ptr()), 0, 0.0, 0.0, sp)
        J_h[0].copy_(J_d[0], non_blocking=True)
        J_h[1].copy_(K_d[0], non_blocking=True)

    for _ in range(3):
        e2e_step()
    barrier()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        e2e_step()
        e1.record()
        torch.cuda.synchronize()
        e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = float(np.mean(e2e_times))
    e2e_value = nq * world / (jdist.max_over_ranks(e2e_ms) * 1e-3)
    # N > 1: the uneven-size sweep sharded over the ranks (every rank takes
    # part, so the collectives of the timing stay in step)
    shard = None
    if world > 1 and args.batch_molecules > 0:
        shard = sharded_sweep(local, rank, world, args.batch_molecules)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    # --- roofline of the dominant class kernel (serialized, CUDA events)
    _, _, cls_ms = eng.jk_timed(D)
    cls_stats = eng.class_stats("fp64")
    best = None
    per_class = []
    for p, q, nquart, nprim, ntask in cls_stats:
        la, lb, lc, ld = QUARTET_CLASSES[q]
        f = nprim * flops.prim_quartet_flops(la, lb, lc, ld) + nquart * flops.digestion_flops(la, lb, lc, ld)
        msq = cls_ms[p * 21 + q]
        per_class.append({"class": f"({la}{lb}|{lc}{ld})", "ms": round(msq, 3), "quartets": nquart,
                          "prim_quartets": nprim, "model_gflop": round(f / 1e9, 3)})
        if best is None or msq > best[0]:
            best = (msq, f, (la, lb, lc, ld))
    peak64 = fp_peak(False)
    peak32 = fp_peak(True)
    achieved = best[1] / (best[0] * 1e-3) / 1e12
    total_model = sum(c["model_gflop"] for c in per_class)

    # --- Fock-build seconds in a full SCF: plain FP64 vs chosen path
    fg = None
    if args.scf:
        ints = compute_integrals(mol, bs, device=local, engine=eng)
        torch.cuda.synchronize()
        # both paths' work lists are built, and the kernels of both paths
        # loaded, before the timed SCF runs
        t_wl = time.perf_counter()
        chosen_tau = CalcConfig().mixed_tau
        eng.stats("mixed", chosen_tau)
        torch.cuda.synchronize()
        t_wl = time.perf_counter() - t_wl
        for prec, tau in (("mixed", 0.0), ("mixed", 1e-8), ("fp64", 1e-11)):
            eng.jk(D, precision=prec, mixed_tau=chosen_tau, dens_tau=tau)
        torch.cuda.synchronize()
        # plain: a full FP64 build every iteration (the reference's Fock build).
        # The two SCFs run alternately, twice each, and each keeps its faster
        # run, so a clock or power-cap change during the leg hits both sides.
        cfg = CalcConfig(scf_conv=1e-8, precision="mixed", incremental=True)
        r64 = rmx = None
        t64 = tmx = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            r = run_scf(mol, ints, CalcConfig(scf_conv=1e-8, incremental=False))
            torch.cuda.synchronize()
            t64 = min(t64, time.perf_counter() - t0)
            if r64 is None or r.precision["jk_seconds"] < r64.precision["jk_seconds"]:
                r64 = r
            t0 = time.perf_counter()
            r = run_scf(mol, ints, cfg)
            torch.cuda.synchronize()
            tmx = min(tmx, time.perf_counter() - t0)
            if rmx is None or r.precision["jk_seconds"] < rmx.precision["jk_seconds"]:
                rmx = r
        from jax_examples_b200.grad import rhf_gradient

        rhf_gradient(mol, r64, engine=eng)  # warm-up (builds the gradient work list)
        rhf_gradient(mol, rmx, engine=eng, dens_tau=CHOSEN_GRAD_TAU)
        torch.cuda.synchronize()
        ge0 = torch.cuda.Event(enable_timing=True)
        ge1 = torch.cuda.Event(enable_timing=True)
        tgrad = tgrad_mx = float("inf")
        for _ in range(2):  # alternately, the faster of two each
            ge0.record()
            g64 = rhf_gradient(mol, r64, engine=eng)
            ge1.record()
            torch.cuda.synchronize()
            tgrad = min(tgrad, ge0.elapsed_time(ge1) * 1e-3)
            ge0.record()
            gmx = rhf_gradient(mol, rmx, engine=eng, dens_tau=CHOSEN_GRAD_TAU)
            ge1.record()
            torch.cuda.synchronize()
            tgrad_mx = min(tgrad_mx, ge0.elapsed_time(ge1) * 1e-3)
        plain_total = r64.precision["jk_seconds"] + tgrad
        chosen_total = rmx.precision["jk_seconds"] + tgrad_mx
        fg = {"mixed_work_list_build_s": round(t_wl, 4),
              "plain_fp64_scf_s": round(t64, 4), "plain_fp64_fock_s": round(r64.precision["jk_seconds"], 4),
              "gradient_s": round(tgrad, 4), "chosen_gradient_s": round(tgrad_mx, 4),
              "chosen_gradient_dens_tau": CHOSEN_GRAD_TAU,
              "gradient_err_eh_bohr": float((g64 - gmx).abs().max()),
              "plain_fock_plus_gradient_s": round(plain_total, 4),
              "chosen_fock_plus_gradient_s": round(chosen_total, 4),
              "fock_plus_gradient_speedup": round(plain_total / max(1e-12, chosen_total), 3),
              "plain_iterations": r64.n_iterations, "chosen_scf_s": round(tmx, 4),
              "chosen_fock_s": round(rmx.precision["jk_seconds"], 4), "chosen_iterations": rmx.n_iterations,
              "chosen_builds": {k: rmx.precision[k] for k in ("builds_mixed", "builds_fp64", "incremental_builds")},
              "energy_fp64": r64.energy, "energy_chosen": rmx.energy,
              "energy_err_eh": abs(r64.energy - rmx.energy),
              "fock_speedup": round(r64.precision["jk_seconds"] / max(1e-12, rmx.precision["jk_seconds"]), 3)}

    sweep = None
    if world == 1 and args.batch_molecules > 0:
        sweep = batched_sweep(local, args.batch_molecules)
    bfgs = None
    if world == 1 and args.batch_molecules > 0 and args.bfgs_steps > 0:
        bfgs = batched_bfgs(local, args.batch_molecules, args.bfgs_steps)
    conf3 = config3_scf(local) if (world == 1 and args.scf) else None
    kconf = kernel_configs(local) if (world == 1 and args.kernel_configs) else None

    cpu = None
    if world == 1 and not args.no_cpu:
        v, cores, desc = cpu_sample(sample=args.cpu_sample)
        cpu = {"value": v, "unit": "quartets/s", "cores": cores, "kind": "port", "sample": desc}

    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_basis": n, "n_shell": eng.packed.n_shell, "schwarz_tau": SCHWARZ_TAU,
                   "quartets_per_step": nq, "prim_quartets_per_step": st["prim_quartets"], "parallelism": (
                       f"replicas{world}" if world > 1 else "single"), "l2": "flushed (256 MiB write) before each step"},
        "e2e": {"value": e2e_value, "unit": "quartets/s", "h2d_bytes_per_step": n * n * 8,
                "d2h_bytes_per_step": 2 * n * n * 8},
        "gpu_launches": st["launches_per_jk"] * args.steps,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64,
                     # DRAM bytes of one launch of the dominant kernel on this workload, from an ncu
                     # capture of dram__bytes_read.sum + dram__bytes_write.sum (7,585,280 + 0)
                     "traffic": 7515904 if best[2] == (1, 0, 0, 0) and N_WATERS == 16 else None,
                     "traffic_note": "L2-resident working set: the DRAM bytes are the compulsory reads of "
                                     "the pair data, the Boys table and D",
                     "kernel": "jk_kernel<double,%d,%d,%d,%d>" % best[2],
                     "peak_source": "FP64 FMA microbenchmark (jqc_fp_peak) measured in this run",
                     "fp32_peak": peak32,
                     "whole_build_tflops": total_model / 1e3 / (ms_max * 1e-3),
                     "whole_build_frac": total_model / 1e3 / (ms_max * 1e-3) / peak64},
        "classes": per_class,
        "clocks": clk.summary(local),
        "cpu_baseline": cpu,
        "fock_gradient": fg,
        "batched_sweep": sweep,
        "sharded_sweep": shard,
        "batched_bfgs": bfgs,
        "config3_scf": conf3,
        "kernel_configs": kconf,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=6_000_000)
    ap.add_argument("--ref-sample", type=int, default=1_000_000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-scf", dest="scf", action="store_false")
    ap.add_argument("--batch-molecules", type=int, default=64,
                    help="molecules in the batched uneven-size sweep (0 skips it)")
    ap.add_argument("--bfgs-steps", type=int, default=10,
                    help="BFGS steps per molecule of the batched sweep (0 skips the optimisation leg)")
    ap.add_argument("--waters", type=int, default=None, help="cluster size (default 16; profiling uses smaller)")
    ap.add_argument("--no-kernel-configs", dest="kernel_configs", action="store_false",
                    help="skip the Boys / primitive-quartet / (H2O)8 kernel sections")
    ap.add_argument("--clock-log", default=None,
                    help="CSV file for the nvidia-smi clock samples of the timed region ({rank} is replaced; "
                         "default: a temporary file)")
    ap.add_argument("--gradient-only", action="store_true",
                    help="time only the ERI-derivative adjoint (profiling case)")
    args = ap.parse_args()
    if args.waters is not None:
        global N_WATERS, WORKLOAD
        N_WATERS = args.waters
        WORKLOAD = WORKLOAD.replace("(H2O)16", f"(H2O){N_WATERS}").replace("(304 bf)", f"({19 * N_WATERS} bf)")
    if args.impl == "reference":
        run_reference(args)
    elif args.gradient_only:
        gradient_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
