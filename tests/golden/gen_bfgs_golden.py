"""Golden BFGS trajectories from the REFERENCE optimizer.

Runs ``jax_qc.geomopt.optimizer.optimize_bfgs`` (through the NumPy shim in
tests/golden/shim, because JAX is not installed here) with its energy and
gradient evaluation (``_energy_and_gradient``, optimizer.py:55-76) replaced by
the analytic pair potential of :func:`model_energy_gradient`, so that the
trajectory depends only on the optimizer's own algorithm (identity initial
inverse Hessian, step clipping, Armijo backtracking, BFGS update,
convergence tests).  Writes tests/golden/bfgs_model.json.

Run from the repository root, with the reference checkout available:

    python tests/golden/gen_bfgs_golden.py /path/to/reference
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def model_energy_gradient(coords: np.ndarray, r0: np.ndarray, de: float = 0.2, a: float = 1.1):
    """Morse pair potential E = sum_{i<j} de (1 - exp(-a (r_ij - r0_ij)))^2
    and its gradient (n, 3)."""
    x = np.asarray(coords, dtype=np.float64)
    n = x.shape[0]
    e = 0.0
    g = np.zeros_like(x)
    for i in range(n):
        for j in range(i + 1, n):
            d = x[i] - x[j]
            r = float(np.linalg.norm(d))
            ex = np.exp(-a * (r - r0[i, j]))
            e += de * (1.0 - ex) ** 2
            dedr = 2.0 * de * (1.0 - ex) * a * ex
            g[i] += dedr * d / r
            g[j] -= dedr * d / r
    return e, g


def cases():
    """Three starting geometries (bohr) and their reference pair lengths."""
    from jax_examples_b200 import basis as pb

    out = []
    for n_w, seed, stretch in [(1, 3, 1.08), (2, 4, 0.95), (3, 5, 1.04)]:
        mol = pb.water_cluster(n_w, seed=seed, noise_angstrom=0.05)
        x = np.asarray(mol.coords, dtype=np.float64)
        r0 = np.linalg.norm(x[:, None, :] - x[None, :, :], axis=-1) * stretch
        out.append((mol, r0))
    return out


def main(ref_root: str) -> None:
    sys.path.insert(0, os.path.join(HERE, "shim"))
    sys.path.insert(0, ref_root)
    sys.path.insert(0, REPO)
    from jax_qc.core.types import make_molecule
    from jax_qc.geomopt import optimizer as ropt

    records = []
    for mol, r0 in cases():
        def fake(coords, m, basis_name, config, r0=r0):
            e, g = model_energy_gradient(np.asarray(coords), r0)
            nm = make_molecule(elements=m.elements, coords=np.asarray(coords), atomic_numbers=m.atomic_numbers,
                               charge=m.charge, spin=m.spin)
            return e, g, nm

        ropt._energy_and_gradient = fake
        rmol = make_molecule(elements=mol.elements, coords=np.asarray(mol.coords),
                             atomic_numbers=np.asarray(mol.atomic_numbers), charge=0, spin=0)
        res = ropt.optimize_bfgs(rmol, basis_name="model", max_steps=25, grad_tol=1e-5, verbose=0)
        records.append({
            "elements": list(mol.elements),
            "coords": np.asarray(mol.coords).tolist(),
            "Z": np.asarray(mol.atomic_numbers).tolist(),
            "r0": r0.tolist(),
            "max_steps": 25,
            "grad_tol": 1e-5,
            "converged": bool(res.converged),
            "n_steps": int(res.n_steps),
            "energy": float(res.energy),
            "trajectory_energies": [float(e) for _, e in res.trajectory],
            "final_coords": np.asarray(res.molecule.coords).tolist(),
            "final_gradient": np.asarray(res.gradient).tolist(),
        })
    out = {
        "source": "jax_qc/geomopt/optimizer.py:79-209 (optimize_bfgs), energy/gradient replaced by "
                  "gen_bfgs_golden.model_energy_gradient",
        "cases": records,
    }
    with open(os.path.join(HERE, "bfgs_model.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "bfgs_model.json"), [(r["n_steps"], r["converged"]) for r in records])


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("JQC_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: gen_bfgs_golden.py REFERENCE_ROOT (or set JQC_REFERENCE_ROOT)")
    main(root)
