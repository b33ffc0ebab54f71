"""Batched SCF energies, gradients and geometry optimisation for many
molecules of uneven size on one device.

The reference evaluates one geometry at a time: ``geomopt/optimizer.py:55-76``
(``_energy_and_gradient``) rebuilds the basis, integrals, SCF and gradient for
every call, and a sweep over geometries is a Python loop of such calls.  Here
a whole set of molecules (different sizes, different geometries) shares one
libjqc context.  ``jqc_batch_partition`` keeps shell pairs and quartets inside
each molecule, so the class-sorted work list of one J/K build covers every
molecule of the batch, and the build is one launch sequence, captured once
into a CUDA graph and replayed in every SCF iteration.  Matrices of a batch
are block-diagonal: molecule m owns rows and columns [off_m, off_m + n_m).

* :class:`MoleculeBatch`   -- the concatenated basis and nuclei, block offsets.
* :class:`BatchedERI`      -- the engine of a batch: J/K into fixed buffers,
  CUDA-graph capture and replay, autotuning, gradients.
* :func:`run_rhf_batch`    -- RHF of every molecule in lock step (per molecule
  exactly ``scf/rhf.py:95-169``: core guess, Loewdin X, DIIS, the same
  convergence test); a converged molecule leaves the loop and its density
  block is zeroed, so density screening skips all of its quartets.
* :func:`rhf_gradient_batch` -- analytic gradients of all molecules with one
  ``jqc_grad2e`` and one ``jqc_grad1e`` call.
* :func:`optimize_bfgs_batch` -- the BFGS of ``geomopt/optimizer.py:79-209``
  for every molecule, each round of energy + gradient evaluations batched.
"""

from __future__ import annotations

import concurrent.futures as cf
import ctypes
import os
import time
from typing import List, NamedTuple, Optional, Sequence

import numpy as np
import torch

from . import _abi
from .basis import build_basis_set, build_shell_indices
from .core import BasisSet, CalcConfig, SCFResult, SCFState, Shell, make_molecule
from .engine import DirectERI, _ptr, _stream
from .grad import energy_weighted_density, grad_one_electron, grad_two_electron, nuclear_repulsion_gradient
from .integrals import nuclear_repulsion_energy

# Density-screening threshold of the batched FP64 builds.  A quartet is
# skipped only when Q_ab Q_cd max|D| < 1e-30, i.e. when its density blocks are
# zero (the blocks of converged molecules) or its contribution is below
# 1e-30 Eh: the builds stay FP64-exact for every active molecule.
BATCH_DENS_TAU = 1e-30

# Density screening of the gradient on the mixed path: on (H2O)16 6-31G* the
# skipped quartets change the gradient by 3.0e-6 Eh/bohr (3e-10: 9.8e-7,
# 3e-9: 9.6e-6), a 3x margin to the 1e-5 tolerance, for 16.5 ms instead of
# 41.8 ms unscreened; the 64-cluster sweep's largest change is 2.5e-6.
MIXED_GRAD_TAU = 1e-9


class _Nuclei:
    """Nuclei of a batch in the form DirectERI reads (coords, charges)."""

    def __init__(self, coords, atomic_numbers):
        self.coords = coords
        self.atomic_numbers = atomic_numbers


class MoleculeBatch:
    """Molecules of uneven size concatenated into one basis and one set of
    nuclei, with the offsets of every molecule's atoms and basis functions.

    Args:
        mols: the molecules (Molecule records, coordinates in bohr).
        basis: basis name used to build every molecule's basis (ignored when
            ``bases`` is given).
        bases: optional per-molecule BasisSet list.
        spherical: layout of the built bases (all bases must agree).
    """

    def __init__(self, mols: Sequence, basis: str = "6-31g*", bases: Optional[Sequence] = None,
                 spherical: bool = False):
        self.mols = list(mols)
        if not self.mols:
            raise ValueError("a batch needs at least one molecule")
        if bases is None:
            bases = [build_basis_set(m, basis, spherical=spherical) for m in self.mols]
        if len(bases) != len(self.mols):
            raise ValueError("one basis per molecule is required")
        sph = {bool(getattr(b, "spherical", False)) for b in bases}
        if len(sph) != 1:
            raise ValueError("all bases of a batch must share the spherical/Cartesian layout")
        self.spherical = sph.pop()
        self.bases = list(bases)
        shells, coords, Z, mol_of_atom = [], [], [], []
        self.atom_off, self.n_atoms, self.bf_off, self.n_bf = [], [], [], []
        a0 = b0 = 0
        for m, (mol, bs) in enumerate(zip(self.mols, self.bases)):
            na = len(np.asarray(mol.atomic_numbers))
            for sh in bs.shells:
                shells.append(Shell(angular_momentum=int(sh.angular_momentum),
                                    exponents=np.asarray(sh.exponents, np.float64),
                                    coefficients=np.asarray(sh.coefficients, np.float64),
                                    center=np.asarray(sh.center, np.float64),
                                    atom_index=int(sh.atom_index) + a0))
            coords.append(np.asarray(mol.coords, np.float64))
            Z.append(np.asarray(mol.atomic_numbers))
            mol_of_atom += [m] * na
            self.atom_off.append(a0)
            self.n_atoms.append(na)
            self.bf_off.append(b0)
            self.n_bf.append(int(bs.n_basis))
            a0 += na
            b0 += int(bs.n_basis)
        s2b, b2a, n = build_shell_indices(shells, spherical=self.spherical)
        self.basis = BasisSet(shells=tuple(shells), n_basis=n, shell_to_basis=s2b, basis_to_atom=b2a,
                              name="batch", spherical=self.spherical)
        self.coords = np.concatenate(coords, axis=0)
        self.atomic_numbers = np.concatenate(Z)
        self.mol_of_atom = np.asarray(mol_of_atom, dtype=np.int32)
        self.n_basis = n

    def __len__(self) -> int:
        return len(self.mols)

    def update_geometry(self, moved: dict) -> None:
        """Replace molecule m by ``moved[m]`` (same atoms, new coordinates) for
        every m in ``moved``; the concatenated nuclei follow.  The engine of
        the batch is moved with :meth:`BatchedERI.update_geometry`."""
        for m, mol in moved.items():
            xyz = np.asarray(mol.coords, np.float64)
            if xyz.shape != (self.n_atoms[m], 3):
                raise ValueError(f"molecule {m}: expected {self.n_atoms[m]} atoms")
            self.mols[m] = mol
            o = self.atom_off[m]
            self.coords[o:o + self.n_atoms[m]] = xyz

    def nuclei(self) -> _Nuclei:
        return _Nuclei(self.coords, self.atomic_numbers)

    def block(self, M: torch.Tensor, m: int) -> torch.Tensor:
        """View of molecule m's block of a batch matrix (last two dims)."""
        o, k = self.bf_off[m], self.n_bf[m]
        return M[..., o:o + k, o:o + k]

    def atoms(self, g: torch.Tensor, m: int) -> torch.Tensor:
        """Rows of molecule m in a per-atom batch array."""
        o = self.atom_off[m]
        return g[o:o + self.n_atoms[m]]


class BatchedERI:
    """Two-electron engine of a :class:`MoleculeBatch` (one libjqc context).

    J/K builds write into fixed buffers so that a build can be captured into
    a CUDA graph (``jqc_graph_begin``/``jqc_graph_end``) and replayed.
    """

    def __init__(self, batch: MoleculeBatch, device=None, schwarz_tau: float = 1e-12, prim_tau: float = 1e-20):
        self.batch = batch
        self.engine = DirectERI(batch.basis, batch.nuclei(), device=device, schwarz_tau=schwarz_tau,
                                prim_tau=prim_tau, mol_of_atom=batch.mol_of_atom)
        self.device = self.engine.device
        self.cartesian = self.engine._C is None
        self._capture_stream = None
        self._graphs: List[int] = []

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        self.engine.close()

    def update_geometry(self, moved: dict, active: Optional[Sequence[bool]] = None) -> None:
        """Geometry-only update of the batch (``jqc_set_geometry``): molecules
        in ``moved`` take their new coordinates, shell pairs and Schwarz
        bounds are rebuilt in the same context, and the launch tuning (the
        autotuner's choice) is kept.  ``active`` (one flag per molecule)
        leaves the other molecules out of the next builds."""
        self.batch.update_geometry(moved)
        self.engine.set_geometry(self.batch.coords, None if active is None else [bool(a) for a in active])

    @property
    def n_basis(self) -> int:
        return self.engine.n_basis

    @property
    def n_cart(self) -> int:
        return self.engine.packed.n_cart

    def buffers(self, n_dens: int = 1):
        """Zeroed (D, J, K) stacks of the batch's Cartesian size."""
        nc = self.n_cart
        D = torch.zeros((n_dens, nc, nc), dtype=torch.float64, device=self.device)
        return D, torch.zeros_like(D), torch.zeros_like(D)

    # ------------------------------------------------------------------ J/K
    def jk_into(self, D, J, K, precision: str = "fp64", mixed_tau: float = 1e-7, dens_tau: float = 0.0,
                stream=None) -> None:
        """J/K of the stack D (Cartesian layout) into J, K (``jqc_jk``)."""
        for t in (D, J, K):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.shape == D.shape):
                raise ValueError("D, J, K must be contiguous float64 CUDA tensors of one shape")
        s = _stream(self.device) if stream is None else ctypes.c_void_p(stream.cuda_stream)
        with torch.cuda.device(self.device):
            _abi.call("jqc_jk", self.engine._ctx, D.shape[0], _ptr(D), _ptr(J), _ptr(K), _abi.PREC[precision],
                      float(mixed_tau), float(dens_tau), s)

    def capture_jk(self, D, J, K, precision: str = "fp64", mixed_tau: float = 1e-7,
                   dens_tau: float = BATCH_DENS_TAU) -> int:
        """Capture one J/K build of the buffers D -> J, K into a CUDA graph and
        return its id; replay with :meth:`launch`.  Runs one ordinary build
        first (it builds the work list and the screening scratch)."""
        if self._capture_stream is None:
            self._capture_stream = torch.cuda.Stream(self.device)
        s = self._capture_stream
        cur = torch.cuda.current_stream(self.device)
        s.wait_stream(cur)
        sp = ctypes.c_void_p(s.cuda_stream)
        lib = self.engine.lib
        with torch.cuda.device(self.device):
            self.jk_into(D, J, K, precision, mixed_tau, dens_tau, stream=s)
            _abi.call("jqc_graph_begin", self.engine._ctx, sp)
            gid = ctypes.c_int(-1)
            try:
                self.jk_into(D, J, K, precision, mixed_tau, dens_tau, stream=s)
            except Exception:
                if lib.jqc_graph_end(self.engine._ctx, sp, ctypes.byref(gid)) == 0:
                    lib.jqc_graph_destroy(self.engine._ctx, gid.value)
                raise
            _abi.call("jqc_graph_end", self.engine._ctx, sp, ctypes.byref(gid))
        cur.wait_stream(s)
        self._graphs.append(gid.value)
        return gid.value

    def launch(self, graph_id: int) -> None:
        """Replay a captured graph on the current stream."""
        with torch.cuda.device(self.device):
            _abi.call("jqc_graph_launch", self.engine._ctx, int(graph_id), _stream(self.device))

    def autotune(self, D, J, K, precision: str = "fp64", mixed_tau: float = 1e-7,
                 dens_tau: float = BATCH_DENS_TAU, cache_path: Optional[str] = None) -> bool:
        """Pick the launch shape of every quartet class for this workload
        (``jqc_autotune``); returns True when it came from the cache file."""
        hit = ctypes.c_int(0)
        path = cache_path.encode() if cache_path else None
        with torch.cuda.device(self.device):
            _abi.call("jqc_autotune", self.engine._ctx, D.shape[0], _ptr(D), _ptr(J), _ptr(K),
                      _abi.PREC[precision], float(mixed_tau), float(dens_tau), path, ctypes.byref(hit),
                      _stream(self.device))
        return bool(hit.value)

    def tuning(self) -> np.ndarray:
        """(21, 4) array of (threads, lane_prims, persistent, engine) per
        quartet class; engine 0 register kernels, 1 column engine, 2 warp
        engine."""
        out = np.zeros(84, dtype=np.int32)
        _abi.call("jqc_get_tuning", self.engine._ctx, out.ctypes.data_as(_abi._ip))
        return out.reshape(21, 4)

    def set_tuning(self, cfg) -> None:
        arr = np.ascontiguousarray(np.asarray(cfg, dtype=np.int32).reshape(84))
        _abi.call("jqc_set_tuning", self.engine._ctx, arr.ctypes.data_as(_abi._ip))


# ---------------------------------------------------------------------------
# lock-step RHF
# ---------------------------------------------------------------------------

class BatchSCF(NamedTuple):
    """Per-molecule SCF results of a batch and the batch's build record."""

    results: List[SCFResult]
    engine: BatchedERI
    record: dict


class _BatchFock:
    """J/K builds of a batch under the SCF precision policy of
    :class:`jax_examples_b200.fock.FockBuilder`, on fixed buffers replayed as
    CUDA graphs (one graph per build kind).

    * ``precision="fp64"``: a full FP64 build every iteration (screening only
      drops the quartets of converged molecules, whose density blocks are
      zero).
    * ``precision="mixed"`` with ``incremental``: the first build is a full
      mixed build (FP32 for Q_ij Q_kl < mixed_tau); then each build contracts
      the density change of the active molecules (J, K are linear in D) with
      density screening at ``mixed_dens_tau``, a full rebuild every
      ``rebuild_every`` builds of the mixed phase (full mixed builds screened
      at ``mixed_full_dens_tau``).  Once the largest DIIS error of the active
      molecules is below ``fp64_switch`` it switches to a full FP64 build
      (screened at ``fp64_switch_dens_tau``) and incremental FP64 builds
      screened at ``fp64_tail_dens_tau``; convergence is accepted only after
      ``fp64_tail_iters`` FP64 builds.
    """

    def __init__(self, eng: BatchedERI, batch: MoleculeBatch, config: CalcConfig, use_graph: bool,
                 rebuild_every: int = 8):
        self.eng, self.batch, self.config = eng, batch, config
        self.cart = eng.cartesian
        self.use_graph = use_graph and self.cart
        self.mixed = config.precision == "mixed"
        self.incremental = bool(config.incremental) and self.mixed
        self.mixed_tau = float(config.mixed_tau)
        self.tail_tau = max(float(config.fp64_tail_dens_tau), BATCH_DENS_TAU)
        self.phase = "mixed" if self.mixed else "fp64"
        self.rebuild_every = rebuild_every
        self.fp64_builds = 0
        self.since_full = 0
        self.prev = None  # densities of the last build, per molecule
        self.events = []
        self.kinds = []  # (kind, active molecules) of every build
        self.graphs = {}
        self.log = {"builds_mixed": 0, "builds_fp64": 0, "incremental_builds": 0}
        self.D, self.J, self.K = eng.buffers(1)
        self.Jacc = torch.zeros_like(self.J[0])
        self.Kacc = torch.zeros_like(self.K[0])
        self._flat_idx = {}  # molecule set -> flat indices of its blocks in D

        # molecules of the next build, read on the device by every build and
        # graph replay: the others are compacted out of the work lists
        self.n_mol = eng.engine.n_mol
        self.active = None
        if self.cart and self.n_mol > 1:
            self.active = torch.ones(self.n_mol, dtype=torch.int32, device=eng.device)
            self._active_host = np.ones(self.n_mol, dtype=np.int32)
            eng.engine.set_molecule_activity(self.active)

    def _scatter(self, dens: dict, prev: Optional[dict] = None) -> None:
        """D <- the blocks of ``dens`` (minus those of ``prev``), zero
        elsewhere: one gather of the values and one indexed copy, not one
        copy launch per molecule."""
        ms = tuple(dens)
        idx = self._flat_idx.get(ms)
        if idx is None:
            b, n = self.batch, self.D.shape[-1]
            parts = []
            for m in ms:
                r = torch.arange(b.bf_off[m], b.bf_off[m] + b.n_bf[m], device=self.D.device, dtype=torch.int64)
                parts.append((r[:, None] * n + r[None, :]).reshape(-1))
            idx = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.int64, device=self.D.device)
            self._flat_idx[ms] = idx
        self.D.zero_()
        if not ms:
            return
        vals = torch.cat([dens[m].reshape(-1) for m in ms])
        if prev is not None:
            vals = vals - torch.cat([prev[m].reshape(-1) for m in ms])
        self.D[0].view(-1).index_copy_(0, idx, vals)

    def _set_active(self, molecules) -> None:
        if self.active is None:
            return
        mask = np.zeros(self.n_mol, dtype=np.int32)
        mask[list(molecules)] = 1
        if not np.array_equal(mask, self._active_host):
            self._active_host = mask
            self.active.copy_(torch.from_numpy(mask))

    def _settings(self, incremental: bool, phase: Optional[str] = None):
        """(precision, density-screening threshold) of the next build."""
        phase = self.phase if phase is None else phase
        if phase == "mixed":
            tau = self.config.mixed_dens_tau if incremental else self.config.mixed_full_dens_tau
            return "mixed", max(float(tau), BATCH_DENS_TAU)
        if not self.mixed:
            return "fp64", BATCH_DENS_TAU  # plain FP64: unscreened apart from zero blocks
        if incremental:
            return "fp64", self.tail_tau
        return "fp64", max(float(self.config.fp64_switch_dens_tau), BATCH_DENS_TAU)

    def _launch(self, incremental: bool):
        prec, tau = self._settings(incremental)
        key = (prec, tau)
        if self.use_graph:
            if key not in self.graphs:
                self.graphs[key] = self.eng.capture_jk(self.D, self.J, self.K, prec, self.mixed_tau, tau)
            self.eng.launch(self.graphs[key])
        else:
            self.eng.jk_into(self.D, self.J, self.K, prec, self.mixed_tau, tau)
        self.log["builds_mixed" if prec == "mixed" else "builds_fp64"] += 1
        if prec == "fp64" and self.switched:
            self.fp64_builds += 1

    @property
    def switched(self) -> bool:
        return self.mixed and self.phase == "fp64"

    def prepare(self, dens: dict, autotune: bool, tune_cache: Optional[str]) -> None:
        """Work lists, autotuning and graph capture before the timed builds."""
        if not self.cart:
            return
        self._set_active(dens.keys())
        self._scatter(dens)
        prec, tau = self._settings(False)
        self.prep_times = {}
        if autotune:
            t0 = time.perf_counter()
            self.eng.autotune(self.D, self.J, self.K, prec, self.mixed_tau, tau, cache_path=tune_cache)
            self.prep_times["autotune"] = time.perf_counter() - t0
        if self.use_graph:
            kinds = [(prec, tau)]
            if self.mixed:
                kinds += [self._settings(False, "fp64")]
            if self.incremental:
                kinds += [self._settings(True, "mixed"), self._settings(True, "fp64")]
            t0 = time.perf_counter()
            for p_, t_ in kinds:
                self.graphs[(p_, t_)] = self.eng.capture_jk(self.D, self.J, self.K, p_, self.mixed_tau, t_)
            torch.cuda.synchronize()
            self.prep_times["capture"] = time.perf_counter() - t0

    def build(self, dens: dict) -> dict:
        """(J_m, K_m) of the molecules in dens."""
        b = self.batch
        if not self.cart:
            Dfull = torch.zeros((self.eng.n_basis, self.eng.n_basis), dtype=torch.float64, device=self.eng.device)
            for m, d in dens.items():
                b.block(Dfull, m).copy_(d)
            prec, tau = self._settings(False)
            J, K = self.eng.engine.jk(Dfull, precision=prec, mixed_tau=self.mixed_tau, dens_tau=tau)
            self.log["builds_mixed" if prec == "mixed" else "builds_fp64"] += 1
            if prec == "fp64" and self.switched:
                self.fp64_builds += 1
            return {m: (b.block(J, m), b.block(K, m)) for m in dens}
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        # the FP64 tail runs without periodic rebuilds: screened at 1e-11 it
        # accumulates little (64-cluster sweep: 3% fewer Fock seconds, the
        # same largest energy error)
        periodic = not self.switched and self.since_full >= self.rebuild_every
        inc = self.incremental and self.prev is not None and not periodic and set(dens) <= set(self.prev)
        self._set_active(dens.keys())
        if inc:
            self._scatter(dens, self.prev)
            self._launch(True)
            self.Jacc += self.J[0]
            self.Kacc += self.K[0]
            self.since_full += 1
            self.log["incremental_builds"] += 1
        else:
            self._scatter(dens)
            self._launch(False)
            self.Jacc.copy_(self.J[0])
            self.Kacc.copy_(self.K[0])
            self.since_full = 0
        if self.incremental:
            self.prev = dict(dens)
        e1.record()
        self.events.append((e0, e1))
        self.kinds.append(("%s-%s" % (self._settings(inc)[0], "inc" if inc else "full"), len(dens)))
        return {m: (b.block(self.Jacc, m), b.block(self.Kacc, m)) for m in dens}

    def observe(self, err_max: float) -> bool:
        """True when this call switched the batch from the mixed phase to FP64."""
        if self.phase == "mixed" and err_max < float(self.config.fp64_switch):
            self.phase = "fp64"
            self.prev = None  # next build: a full FP64 build
            return True
        return False

    def converged_ok(self) -> bool:
        return not self.mixed or (self.phase == "fp64" and self.fp64_builds >= int(self.config.fp64_tail_iters))

    def seconds(self) -> float:
        if not self.events:
            return 0.0
        self.events[-1][1].synchronize()
        return sum(a.elapsed_time(c) for a, c in self.events) * 1e-3

    def build_ms(self) -> list:
        """[kind, active molecules, milliseconds] of every build."""
        if not self.events:
            return []
        self.events[-1][1].synchronize()
        return [[k, n, round(a.elapsed_time(c), 3)] for (k, n), (a, c) in zip(self.kinds, self.events)]


_HOST_EIGH_MAX_N = 512
_EIGH_POOL: Optional[cf.ThreadPoolExecutor] = None


def _eigh_pool() -> cf.ThreadPoolExecutor:
    global _EIGH_POOL
    if _EIGH_POOL is None:
        n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        _EIGH_POOL = cf.ThreadPoolExecutor(max_workers=max(1, min(n, 32)), thread_name_prefix="jqc-eigh")
    return _EIGH_POOL


def _eigh_one(A: torch.Tensor):
    # One solver thread per matrix: torch.set_num_threads sets this worker's
    # OpenMP and MKL thread counts (both thread-local here), so the pool's
    # workers do not each start a team of their own.
    torch.set_num_threads(1)
    return torch.linalg.eigh(A)


def _diag_all(groups, Fs, active=None):
    """(eps, C) of X^T F X for every group.

    ``active`` (one host boolean array per group, or None for all) names the
    members whose orbitals are wanted; the others get eps = 0 and C = X, which
    the caller masks out.  The eigensolver runs on the host cores for matrices
    up to a few hundred rows, one matrix per worker thread with one solver
    thread each, largest first: a device eigh of that size is latency bound
    (~3 ms a call), and one batched host call per group leaves most cores idle
    on the small molecules (64 molecules of 19-228 rows: 94 ms batched per
    group against 17 ms pooled on 8 cores).  The products around it stay on
    the device, and the selected matrices cross to the host in one copy."""
    out = [None] * len(groups)
    host_jobs = []  # (group index, member rows on the device, their matrices)
    for k, (g, F) in enumerate(zip(groups, Fs)):
        G, n = F.shape[0], F.shape[-1]
        rows = np.arange(G) if active is None else np.flatnonzero(np.asarray(active[k], dtype=bool))
        if len(rows) == 0:
            out[k] = (torch.zeros((G, n), dtype=F.dtype, device=F.device), g.X.clone())
            continue
        X = g.X if len(rows) == G else g.X[torch.as_tensor(rows, device=F.device)]
        Fs_k = F if len(rows) == G else F[torch.as_tensor(rows, device=F.device)]
        A = X.transpose(1, 2) @ Fs_k @ X
        if n > _HOST_EIGH_MAX_N:
            e, V = torch.linalg.eigh(A)
            out[k] = (rows, e, X @ V)
        else:
            host_jobs.append((k, rows, A))
    if host_jobs:
        flat = torch.cat([A.reshape(-1) for _, _, A in host_jobs]).cpu()
        mats, pos = [], 0
        for k, rows, A in host_jobs:
            n = A.shape[-1]
            for _ in rows:
                mats.append(flat[pos:pos + n * n].view(n, n))
                pos += n * n
        order = sorted(range(len(mats)), key=lambda i: -mats[i].shape[0])
        n0 = torch.get_num_threads()
        try:
            solved = list(_eigh_pool().map(_eigh_one, [mats[i] for i in order]))
        finally:
            torch.set_num_threads(n0)
        res = [None] * len(mats)
        for i, r in zip(order, solved):
            res[i] = r
        j = 0
        for k, rows, A in host_jobs:
            e = torch.stack([res[j + i][0] for i in range(len(rows))]).to(A.device)
            V = torch.stack([res[j + i][1] for i in range(len(rows))]).to(A.device)
            j += len(rows)
            X = groups[k].X if len(rows) == groups[k].X.shape[0] else groups[k].X[torch.as_tensor(rows, device=A.device)]
            out[k] = (rows, e, X @ V)
    for k, (g, F) in enumerate(zip(groups, Fs)):
        if len(out[k]) == 2:
            continue
        rows, e, C = out[k]
        G = F.shape[0]
        if len(rows) == G:
            out[k] = (e, C)
            continue
        idx = torch.as_tensor(rows, device=F.device)
        eps = torch.zeros((G, F.shape[-1]), dtype=F.dtype, device=F.device)
        Cf = g.X.clone()
        eps[idx] = e
        Cf[idx] = C
        out[k] = (eps, Cf)
    return out


class _Group:
    """Molecules of one (basis size, occupied count): their SCF state as
    stacked (G, n, n) tensors, so every step of the iteration is one batched
    operation per group."""

    def __init__(self, members, S, H, n_occ):
        self.members = list(members)
        self.S, self.H = S, H
        self.n_occ = n_occ
        w, U = torch.linalg.eigh(S)
        self.X = (U * (1.0 / torch.sqrt(w))[:, None, :]) @ U.transpose(1, 2)  # S^-1/2 (orthogonalize.py:22-26)
        self.Fh, self.Eh = [], []  # DIIS history, oldest first

    def diag(self, F):
        """Orbital energies and coefficients of X^T F X (one group)."""
        return _diag_all([self], [F])[0]

    def density(self, C):
        Co = C[:, :, :self.n_occ]
        return 2.0 * Co @ Co.transpose(1, 2)

    def diis(self, F, err, size: int):
        """Pulay extrapolation of every member (diis.py:53-130): ring buffer of
        ``size`` pairs, B_ij = <e_i, e_j> bordered by -1, fallback to F when
        the system is singular or the history has fewer than two entries."""
        self.Fh.append(F)
        self.Eh.append(err)
        if len(self.Fh) > size:
            self.Fh.pop(0)
            self.Eh.pop(0)
        m = len(self.Fh)
        if m < 2:
            return F
        G = F.shape[0]
        E = torch.stack(self.Eh, 1).reshape(G, m, -1)
        B = torch.empty((G, m + 1, m + 1), dtype=F.dtype, device=F.device)
        B[:, :m, :m] = E @ E.transpose(1, 2)
        B[:, m, :m] = -1.0
        B[:, :m, m] = -1.0
        B[:, m, m] = 0.0
        rhs = torch.zeros((G, m + 1, 1), dtype=F.dtype, device=F.device)
        rhs[:, m, 0] = -1.0
        c, info = torch.linalg.solve_ex(B, rhs)
        Fx = torch.einsum("gi,gimn->gmn", c[:, :m, 0], torch.stack(self.Fh, 1))
        ok = (info == 0) & torch.isfinite(c[:, :m, 0]).all(dim=1)
        return torch.where(ok[:, None, None], Fx, F)


def run_rhf_batch(batch: MoleculeBatch, config: Optional[CalcConfig] = None, engine: Optional[BatchedERI] = None,
                  use_graph: bool = True, autotune: bool = False, tune_cache: Optional[str] = None,
                  molecules: Optional[Sequence[int]] = None) -> BatchSCF:
    """Closed-shell SCF of every molecule of the batch, in lock step.

    Per molecule the iteration is that of ``scf/rhf.py:95-169`` (and of
    :func:`jax_examples_b200.scf.run_rhf`): core-Hamiltonian guess, Loewdin
    X = S^-1/2, F0 from the guess density, DIIS, converged when
    dE < scf_conv and max|DIIS error| < max(scf_conv, 1e-6).  All molecules
    share each Fock build (one graph replay of the batch J/K, see
    :class:`_BatchFock` for the precision policy of ``config.precision``); the
    rest of an iteration (DIIS error, extrapolation, eigh, density, energy)
    runs as batched tensor operations per group of equal-size molecules with
    one host read per iteration.  A converged molecule keeps its state and
    leaves the builds.

    ``molecules`` restricts the SCF to those molecules of the batch (the
    others get ``None`` results); the engine's molecule mask should leave the
    rest out of the pair list (:meth:`BatchedERI.update_geometry`).
    """
    config = config or CalcConfig()
    M = len(batch)
    sel = list(range(M)) if molecules is None else sorted({int(m) for m in molecules})
    if not sel or sel[0] < 0 or sel[-1] >= M:
        raise ValueError("molecules must be a non-empty subset of the batch's molecule indices")
    for m in sel:
        mol = batch.mols[m]
        if mol.spin != 0 or mol.n_electrons % 2 != 0:
            raise ValueError("run_rhf_batch requires closed-shell molecules (spin 0, even electron count)")
    eng = engine or BatchedERI(batch, schwarz_tau=config.schwarz_tau)
    t_setup = time.perf_counter()
    S_all, T_all, V_all = eng.engine.one_electron()
    H_all = T_all + V_all
    n_occ = [mol.n_electrons // 2 for mol in batch.mols]
    E_nuc = [nuclear_repulsion_energy(mol) if m in sel else 0.0 for m, mol in enumerate(batch.mols)]
    keys = {}
    for m in sel:
        keys.setdefault((batch.n_bf[m], n_occ[m]), []).append(m)
    groups = []
    for (n, no), members in keys.items():
        S = torch.stack([batch.block(S_all, m) for m in members])
        H = torch.stack([batch.block(H_all, m) for m in members])
        groups.append(_Group(members, S, H, no))
    fb = _BatchFock(eng, batch, config, use_graph)

    if fb.cart:
        # flat indices of every group's blocks in the batch matrices: J and K
        # of a whole group are one gather each from the builder's accumulators
        N = batch.n_basis
        for g in groups:
            r = torch.stack([torch.arange(batch.bf_off[m], batch.bf_off[m] + batch.n_bf[m], device=g.H.device)
                             for m in g.members])
            g.flat = r[:, :, None] * N + r[:, None, :]

    def fock(g: _Group, jk: dict, fallback):
        if fb.cart:
            # members that left the builds keep their last J/K there; their
            # state is not updated any more (masked below)
            J = fb.Jacc.view(-1)[g.flat]
            K = fb.Kacc.view(-1)[g.flat]
        else:
            J = torch.stack([jk[m][0] if m in jk else fallback[i] * 0 for i, m in enumerate(g.members)])
            K = torch.stack([jk[m][1] if m in jk else fallback[i] * 0 for i, m in enumerate(g.members)])
        return g.H + J - 0.5 * K

    # core guess (rhf.py:111-121)
    for g, (_, C) in zip(groups, _diag_all(groups, [g.H for g in groups])):
        g.D = g.density(C)
    dens = {m: g.D[i] for g in groups for i, m in enumerate(g.members)}
    torch.cuda.synchronize()
    t_prep = time.perf_counter()
    fb.prepare(dens, autotune, tune_cache)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    prepare_s = time.perf_counter() - t_prep
    jk = fb.build(dens)
    for g in groups:
        g.F = fock(g, jk, g.D)
    for g, (eps, C) in zip(groups, _diag_all(groups, [g.F for g in groups])):
        g.eps, g.C = eps, C
    for g in groups:
        g.E = 0.5 * torch.sum(g.D * (g.H + g.F), dim=(1, 2))
        g.active = torch.ones(len(g.members), dtype=torch.bool, device=g.D.device)
        g.iters = torch.zeros(len(g.members), dtype=torch.int64, device=g.D.device)
    last = torch.cat([g.E for g in groups]).cpu().numpy()
    order = [m for g in groups for m in g.members]
    pos = {m: k for k, m in enumerate(order)}
    converged = np.ones(M, dtype=bool)
    converged[sel] = False
    for _ in range(config.max_scf_iter):
        if converged.all():
            break
        dens = {m: g.D[i] for g in groups for i, m in enumerate(g.members) if not converged[m]}
        jk = fb.build(dens)
        Es, emaxs = [], []
        errs, Fxs = [], []
        for g in groups:
            Fn = fock(g, jk, g.D)
            if config.damping > 0.0:
                Fn = (1.0 - config.damping) * Fn + config.damping * g.F
            err = g.X.transpose(1, 2) @ (Fn @ g.D @ g.S - g.S @ g.D @ Fn) @ g.X  # diis.py:53-59
            errs.append(err)
            Fxs.append(g.diis(Fn, err, config.diis_space))
        eigs = _diag_all(groups, Fxs, [~converged[g.members] for g in groups])
        for g, err, Fx, (eps, C) in zip(groups, errs, Fxs, eigs):
            act = g.active
            D = g.density(C)
            E = 0.5 * torch.sum(D * (g.H + Fx), dim=(1, 2))
            a3 = act[:, None, None]
            g.D = torch.where(a3, D, g.D)
            g.F = torch.where(a3, Fx, g.F)
            g.C = torch.where(a3, C, g.C)
            g.eps = torch.where(act[:, None], eps, g.eps)
            g.E = torch.where(act, E, g.E)
            g.iters = g.iters + act.to(torch.int64)
            Es.append(g.E)
            emaxs.append(torch.amax(torch.abs(err), dim=(1, 2)))
        host = torch.cat([torch.cat(Es), torch.cat(emaxs)]).cpu().numpy()
        E_now, emax = host[:len(order)], host[len(order):]
        act_host = ~converged[order]
        if fb.observe(float(emax[act_host].max()) if act_host.any() else 0.0) and config.diis_reset_at_switch:
            for g in groups:  # as FockBuilder's drivers: no mixed-phase Fock matrix in the FP64 extrapolation
                g.Fh.clear()
                g.Eh.clear()
        ok = fb.converged_ok()
        for k, m in enumerate(order):
            if converged[m]:
                continue
            dE = abs(E_now[k] - last[k])
            last[k] = E_now[k]
            if ok and dE < config.scf_conv and emax[k] < max(config.scf_conv, 1e-6):
                converged[m] = True
        for g in groups:
            g.active = torch.tensor([not converged[m] for m in g.members], device=g.D.device)
    record = dict(fb.log, fock_builds=sum(fb.log[k] for k in ("builds_mixed", "builds_fp64")),
                  jk_seconds=fb.seconds(), build_ms=fb.build_ms(), setup_seconds=setup_s, graph=bool(fb.graphs),
                  autotuned=bool(autotune),
                  n_molecules=M, n_basis=batch.n_basis, precision=config.precision,
                  incremental=fb.incremental, groups=len(groups), prepare_seconds=prepare_s, molecules=len(sel),
                  prepare_breakdown=getattr(fb, "prep_times", {}))
    results = [None] * M
    for g in groups:
        iters = g.iters.cpu().numpy()
        for i, m in enumerate(g.members):
            e = float(g.E[i])
            st = SCFState(density=g.D[i], fock=g.F[i], coefficients=g.C[i], orbital_energies=g.eps[i], energy=e,
                          iteration=int(iters[i]))
            results[m] = SCFResult(converged=bool(converged[m]), state=st, energy=e + E_nuc[m], E_elec=e,
                                   E_nuc=E_nuc[m], n_iterations=int(iters[i]), S=g.S[i], H_core=g.H[i], ERI=None,
                                   precision={"precision": config.precision, "batched": True})
    return BatchSCF(results=results, engine=eng, record=record)


def rhf_gradient_batch(batch: MoleculeBatch, scf: BatchSCF, timing: Optional[dict] = None,
                       dens_tau: float = 0.0) -> List[torch.Tensor]:
    """Analytic RHF gradients (n_atoms_m, 3) of every molecule of the batch:
    one ``jqc_grad2e`` and one ``jqc_grad1e`` call over the block-diagonal
    densities (the per-molecule expression of
    :func:`jax_examples_b200.grad.rhf_gradient`; dens_tau > 0 screens the
    two-electron quartets by their density-weighted bound)."""
    eng = scf.engine
    dev = eng.device
    n = eng.n_basis
    D = torch.zeros((n, n), dtype=torch.float64, device=dev)
    W = torch.zeros_like(D)
    for m, res in enumerate(scf.results):
        if res is None:
            continue
        st = res.state
        batch.block(D, m).copy_(st.density)
        batch.block(W, m).copy_(energy_weighted_density(st.coefficients, st.orbital_energies,
                                                        batch.mols[m].n_electrons // 2))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    g = grad_one_electron(eng.engine, D, W) + grad_two_electron(eng.engine, [D], 1.0, 0.5, dens_tau)
    e1.record()
    e1.synchronize()
    if timing is not None:
        timing["grad_seconds"] = timing.get("grad_seconds", 0.0) + e0.elapsed_time(e1) * 1e-3
    out = []
    for m, mol in enumerate(batch.mols):
        if scf.results[m] is None:
            out.append(None)
            continue
        gn = nuclear_repulsion_gradient(mol.coords, mol.atomic_numbers).to(dev)
        out.append(batch.atoms(g, m) + gn)
    return out


# ---------------------------------------------------------------------------
# batched BFGS
# ---------------------------------------------------------------------------

class OptResult(NamedTuple):
    """Result of a geometry optimisation (``geomopt/optimizer.py:36-52``)."""

    converged: bool
    molecule: object
    energy: float
    gradient: np.ndarray
    n_steps: int
    trajectory: list


def _bfgs_walker(mol, max_steps: int, grad_tol: float, step_tol: float, max_step_size: float):
    """BFGS of ``geomopt/optimizer.py:79-209`` for one molecule, written as a
    generator: it yields the coordinates it needs evaluated and receives
    (energy, gradient) back, so many walkers can share batched evaluations.
    Identity initial inverse Hessian, step clipped to max_step_size, Armijo
    backtracking (c1 = 1e-4, at most 10 halvings, the last trial accepted
    when none passes), BFGS update when s.y > 1e-10."""
    coords = np.asarray(mol.coords, dtype=np.float64).copy()
    n_atoms = coords.shape[0]
    n_dof = 3 * n_atoms
    energy, grad = yield coords
    g = np.asarray(grad, dtype=np.float64).reshape(-1)
    H_inv = np.eye(n_dof)
    trajectory = [(coords.copy(), energy)]
    converged = False
    for _step in range(1, max_steps + 1):
        g_max = float(np.max(np.abs(g)))
        if g_max < grad_tol:
            converged = True
            break
        direction = -H_inv @ g
        norm = float(np.linalg.norm(direction))
        if norm > max_step_size:
            direction = direction * (max_step_size / norm)
        alpha, c1 = 1.0, 1e-4
        e_old, g_old = energy, g.copy()
        for _ in range(10):
            new_coords = coords + alpha * direction.reshape(n_atoms, 3)
            e_new, g_new = yield new_coords
            if e_new <= e_old + c1 * alpha * float(np.dot(g_old, direction)):
                break
            alpha *= 0.5
        s = (alpha * direction).reshape(-1)
        coords = new_coords
        energy = e_new
        g_new = np.asarray(g_new, dtype=np.float64).reshape(-1)
        y = g_new - g_old
        s_max = float(np.max(np.abs(s)))
        if s_max < step_tol and g_max < grad_tol * 10:
            converged = True
            g = g_new
            trajectory.append((coords.copy(), energy))
            break
        sy = float(np.dot(s, y))
        if sy > 1e-10:
            rho = 1.0 / sy
            V = np.eye(n_dof) - rho * np.outer(s, y)
            H_inv = V @ H_inv @ V.T + rho * np.outer(s, s)
        g = g_new
        trajectory.append((coords.copy(), energy))
    final = make_molecule(mol.elements, coords, np.asarray(mol.atomic_numbers), charge=mol.charge, spin=mol.spin)
    return OptResult(converged=converged, molecule=final, energy=energy, gradient=g.reshape(n_atoms, 3),
                     n_steps=len(trajectory) - 1, trajectory=trajectory)


def energies_and_gradients(mols: Sequence, basis: str = "6-31g*", config: Optional[CalcConfig] = None,
                           use_graph: bool = True, autotune: bool = False, tune_cache: Optional[str] = None,
                           timing: Optional[dict] = None):
    """RHF energies and analytic gradients of many molecules in one batch:
    ``[(energy, gradient (n_atoms, 3) ndarray, SCFResult)]``."""
    batch = MoleculeBatch(mols, basis)
    config = config or CalcConfig()
    scf = run_rhf_batch(batch, config, use_graph=use_graph, autotune=autotune, tune_cache=tune_cache)
    grads = rhf_gradient_batch(batch, scf, timing, MIXED_GRAD_TAU if config.precision == "mixed" else 0.0)
    if timing is not None:
        timing["jk_seconds"] = timing.get("jk_seconds", 0.0) + scf.record["jk_seconds"]
        timing["fock_builds"] = timing.get("fock_builds", 0) + scf.record["fock_builds"]
        timing["evaluations"] = timing.get("evaluations", 0) + len(mols)
        timing["batches"] = timing.get("batches", 0) + 1
    out = [(r.energy, g.cpu().numpy(), r) for r, g in zip(scf.results, grads)]
    scf.engine.close()
    return out


class _BatchEvaluator:
    """Energies and analytic gradients of a changing subset of a fixed set of
    molecules, on one engine that lives as long as the evaluator.

    The first call builds the context (and, with ``autotune``, tunes the
    launches); every later call moves the nuclei in place
    (:meth:`BatchedERI.update_geometry`), rebuilds only the shell pairs and
    work lists, leaves the molecules not asked for out of the pair list, and
    keeps the tuning.  Each evaluation is a full SCF from the core guess, as
    ``_energy_and_gradient`` (``geomopt/optimizer.py:55-76``) does."""

    def __init__(self, mols: Sequence, basis: str, config: CalcConfig, use_graph: bool = True,
                 autotune: bool = False, tune_cache: Optional[str] = None, timing: Optional[dict] = None):
        self.mols = list(mols)
        self.batch = MoleculeBatch(self.mols, basis)
        self.config, self.use_graph, self.autotune, self.tune_cache = config, use_graph, autotune, tune_cache
        self.timing = timing
        self.gtau = MIXED_GRAD_TAU if config.precision == "mixed" else 0.0
        self.eng = None
        self.rounds = 0

    def __call__(self, coords: dict) -> dict:
        """{i: (energy, gradient (n_atoms, 3) ndarray)} for {i: coords}."""
        ids = sorted(coords)
        mols = self.mols
        moved = {i: make_molecule(mols[i].elements, coords[i], np.asarray(mols[i].atomic_numbers),
                                  charge=mols[i].charge, spin=mols[i].spin) for i in ids}
        t0 = time.perf_counter()
        mask = [m in moved for m in range(len(mols))]
        if self.eng is None:
            self.eng = BatchedERI(self.batch, schwarz_tau=self.config.schwarz_tau)
            same = all(np.array_equal(np.asarray(moved[i].coords, np.float64),
                                      np.asarray(mols[i].coords, np.float64)) for i in ids)
            if not (same and all(mask)):
                self.eng.update_geometry(moved, mask)
        else:
            self.eng.update_geometry(moved, mask)
        t_geom = time.perf_counter() - t0
        scf = run_rhf_batch(self.batch, self.config, engine=self.eng, use_graph=self.use_graph,
                            autotune=self.autotune and self.rounds == 0, tune_cache=self.tune_cache, molecules=ids)
        grads = rhf_gradient_batch(self.batch, scf, self.timing, self.gtau)
        tm = self.timing
        if tm is not None:
            rec = scf.record
            tm["jk_seconds"] = tm.get("jk_seconds", 0.0) + rec["jk_seconds"]
            tm["fock_builds"] = tm.get("fock_builds", 0) + rec["fock_builds"]
            tm["evaluations"] = tm.get("evaluations", 0) + len(ids)
            tm["batches"] = tm.get("batches", 0) + 1
            tm["geometry_update_seconds"] = tm.get("geometry_update_seconds", 0.0) + t_geom
            tm["setup_seconds"] = tm.get("setup_seconds", 0.0) + rec["setup_seconds"]
            br = tm.setdefault("prepare_breakdown", {})
            for k, v in rec.get("prepare_breakdown", {}).items():
                br[k] = br.get(k, 0.0) + v
        self.rounds += 1
        return {i: (scf.results[i].energy, grads[i].cpu().numpy()) for i in ids}

    def close(self) -> None:
        if self.eng is not None:
            self.eng.close()
            self.eng = None


def optimize_bfgs_batch(mols: Sequence, basis: str = "6-31g*", max_steps: int = 50, grad_tol: float = 1e-4,
                        step_tol: float = 1e-6, scf_conv: float = 1e-10, max_step_size: float = 0.3,
                        config: Optional[CalcConfig] = None, use_graph: bool = True, autotune: bool = False,
                        tune_cache: Optional[str] = None, timing: Optional[dict] = None) -> List[OptResult]:
    """BFGS geometry optimisation of every molecule (``optimize_bfgs`` of
    ``geomopt/optimizer.py:79-209`` per molecule, RHF).  Every round collects
    the geometry each unfinished optimisation needs next (a step or a
    line-search trial) and evaluates all of them in one batch, on one engine
    kept for the whole optimisation (geometry-only updates between rounds,
    tuning done once: :class:`_BatchEvaluator`)."""
    config = config or CalcConfig(scf_conv=scf_conv, max_scf_iter=200)
    walkers = [_bfgs_walker(m, max_steps, grad_tol, step_tol, max_step_size) for m in mols]
    pending = {i: w.send(None) for i, w in enumerate(walkers)}
    results: List[Optional[OptResult]] = [None] * len(mols)
    ev = _BatchEvaluator(mols, basis, config, use_graph, autotune, tune_cache, timing)
    try:
        while pending:
            out = ev(pending)
            nxt = {}
            for i in sorted(pending):
                try:
                    nxt[i] = walkers[i].send(out[i])
                except StopIteration as stop:
                    results[i] = stop.value
            pending = nxt
    finally:
        ev.close()
    if timing is not None:
        timing["rounds"] = ev.rounds
    return results


def optimize_bfgs(mol, basis_name: str = "6-31g*", method: str = "rhf", max_steps: int = 50,
                  grad_tol: float = 1e-4, step_tol: float = 1e-6, scf_conv: float = 1e-10,
                  max_step_size: float = 0.3, verbose: int = 0) -> OptResult:
    """Single-molecule ``optimize_bfgs`` (``geomopt/optimizer.py:79-209``)
    with the device SCF and the analytic gradient."""
    if method != "rhf":
        raise NotImplementedError("optimize_bfgs: only method='rhf' is implemented on the batched path")
    return optimize_bfgs_batch([mol], basis_name, max_steps, grad_tol, step_tol, scf_conv, max_step_size)[0]
