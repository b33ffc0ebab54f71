"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
jax_qc FP64 code (through the NumPy shim in tests/golden/shim, because JAX,
chex and basis_set_exchange are not installed here).

Run from the repository root, with the reference checkout available:

    python tests/golden/gen_golden.py /path/to/reference [core|real|all]

(or set ``JQC_REFERENCE_ROOT``).  ``core`` writes the fixtures of the
synthetic bases and the MMD primitives, ``real`` those of the published bases
(STO-3G, 6-31G, 6-31G*, 6-31G**) including the spherical path; the default is
both.

Everything it writes is produced by the reference functions named in each
fixture's ``source`` entry; the accurate Boys values come from mpmath
quadrature.  The bases are the ones ``jax_examples_b200.basis`` defines (the
published STO-3G / 6-31G family and the synthetic STO-3G- / 6-31G*-shaped
sets), registered with the shim's basis registry so that the reference parses
and normalizes them itself.
"""

from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref_root: str, sections=("core", "real")) -> None:
    sys.path.insert(0, os.path.join(HERE, "shim"))
    sys.path.insert(0, ref_root)
    sys.path.insert(0, REPO)
    import basis_set_exchange as bse_shim
    import mpmath

    import jax_qc
    import jax_qc.integrals.mcmurchie_davidson as mmd
    from jax_qc.core.types import CalcConfig, make_molecule
    from jax_qc.integrals import boys as rboys
    from jax_qc.integrals.eri import compute_eri_tensor
    from jax_qc.integrals.obara_saika import contracted_eri_block, primitive_eri_block
    from jax_qc.integrals.screening import compute_shell_pair_bounds
    from jax_qc.scf import diis as rdiis
    from jax_qc.scf.fock import build_fock_rhf, build_fock_uhf
    from jax_qc.grad.rhf_grad import rhf_gradient

    from jax_examples_b200 import basis as pb

    # NumPy arrays have no .at[].set: restate diis._push (diis.py:62-78).
    def _push(history, F, e):
        if history.size < history.max_size:
            fl = np.array(history.fock_list)
            el = np.array(history.error_list)
            fl[history.size] = F
            el[history.size] = e
            return history.replace(fock_list=fl, error_list=el, size=history.size + 1)
        fl = np.concatenate([history.fock_list[1:], F[None]], axis=0)
        el = np.concatenate([history.error_list[1:], e[None]], axis=0)
        return history.replace(fock_list=fl, error_list=el)

    rdiis._push = _push
    for name in ("sto-3g", "6-31g", "6-31g*", "6-31g**", "syn-sto-3g", "syn-6-31g*", "syn-6-31g**"):
        bse_shim.register(name, pb.get_basis_dict(name))

    mpmath.mp.dps = 40
    rng = np.random.default_rng(20261203)

    def boys_true(n, t):
        return float(mpmath.quad(lambda u: u ** (2 * n) * mpmath.exp(-t * u * u), [0, 1]))

    if "core" in sections:
        # ---------------------------------------------------------------- Boys
        T = np.concatenate([
            [0.0, 1e-12, 1e-8, 1e-4, 5e-3, 0.00999, 0.01, 0.01001, 0.02, 0.05, 0.1, 0.3, 0.5],
            rng.uniform(0, 30, 48), 10 ** rng.uniform(-8, 3, 48), [29.99, 30.0, 36.0, 40.0, 50.0, 117.0, 1000.0],
        ])
        nmax = 10
        ref = np.array([[float(rboys.boys_fn(n, t)) for n in range(nmax + 1)] for t in T])
        true = np.array([[boys_true(n, t) for n in range(nmax + 1)] for t in T])
        np.savez_compressed(os.path.join(HERE, "boys.npz"), T=T, ref=ref, true=true,
                            source="jax_qc/integrals/boys.py:86-109 boys_fn; true = mpmath quadrature (dps 40)")
        print("boys: max |ref-true| =", np.max(np.abs(ref - true)))

        # Accurate-Boys variant of the reference MMD (the reference code with its
        # boys_fn replaced by the quadrature; same recursion / contraction).
        def accurate_boys(n, t):
            return boys_true(n, float(t))

        # ------------------------------------------------- MMD primitives
        he_cases, he_out = [], []
        for la in range(4):
            for lb in range(4):
                xpa, xpb, p = rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.2, 20)
                he_cases.append((la, lb, xpa, xpb, p))
                he_out.append(mmd.hermite_e(la, lb, xpa, xpb, p).ravel())
        hr_cases, hr_out = [], []
        for L in range(0, 10):
            p = 10 ** rng.uniform(-1, 1.5)
            PC = rng.uniform(-1.5, 1.5, 3)
            hr_cases.append((L, p, *PC))
            hr_out.append(mmd.hermite_r_aux(L, L, L, 0, p, PC)[..., 0].ravel())

        classes = [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 1, 1), (2, 0, 1, 0), (2, 2, 2, 2), (2, 1, 1, 0),
                   (1, 1, 0, 0), (2, 2, 1, 1), (0, 1, 2, 0), (2, 1, 2, 1)]
        pe_cases, pe_ref, pe_acc = [], [], []
        t0 = time.time()
        for cls in classes:
            for rep in range(3 if sum(cls) < 8 else 1):
                ex = 10 ** rng.uniform(-1, 2, 4)
                ctr = rng.uniform(0, 4.0 / 0.529177210903, (4, 3))
                args = []
                for k in range(4):
                    args += [float(ex[k]), ctr[k], cls[k]]
                pe_cases.append(np.concatenate([[*cls], ex, ctr.ravel()]))
                pe_ref.append(primitive_eri_block(*args).ravel())
                old = mmd.boys_fn
                mmd.boys_fn = accurate_boys
                try:
                    pe_acc.append(primitive_eri_block(*args).ravel())
                finally:
                    mmd.boys_fn = old
        print("primitive eri cases", len(pe_cases), "in %.1fs" % (time.time() - t0))
        np.savez_compressed(
            os.path.join(HERE, "mmd_primitives.npz"),
            he_cases=np.array(he_cases), he_out=np.array(he_out, dtype=object),
            hr_cases=np.array(hr_cases), hr_out=np.array(hr_out, dtype=object),
            pe_cases=np.array(pe_cases), pe_ref=np.array(pe_ref, dtype=object), pe_acc=np.array(pe_acc, dtype=object),
            source="mcmurchie_davidson.py:60-172 hermite_e/hermite_r_aux; obara_saika.py:227-332 primitive_eri_block "
                   "(pe_acc: same code with boys_fn replaced by mpmath quadrature)",
        )

    # ------------------------------------------------- molecules
    def ref_mol(m):
        return make_molecule(elements=m.elements, coords=np.asarray(m.coords), atomic_numbers=np.asarray(m.atomic_numbers),
                             charge=m.charge, spin=m.spin)

    def shells_record(basis):
        return {
            "l": [int(s.angular_momentum) for s in basis.shells],
            "exps": [np.asarray(s.exponents).tolist() for s in basis.shells],
            "coefs": [np.asarray(s.coefficients).tolist() for s in basis.shells],
            "centers": [np.asarray(s.center).tolist() for s in basis.shells],
            "atoms": [int(s.atom_index) for s in basis.shells],
        }

    def run_system(tag, mol, bname, full_tensor, n_sample=0, grad=False, uhf=False, spherical=False, rng=rng):
        rm = ref_mol(mol)
        basis = jax_qc.build_basis_set(rm, bname, use_cache=False, spherical=spherical)
        t0 = time.time()
        ints = jax_qc.compute_integrals(rm, basis)
        t_int = time.time() - t0
        eri = np.asarray(ints.ERI)
        n = eri.shape[0]
        rec = {"tag": tag, "basis": bname, "spherical": bool(spherical), "n": n, "elements": list(mol.elements),
               "coords": np.asarray(mol.coords).tolist(), "Z": np.asarray(mol.atomic_numbers).tolist(),
               "charge": mol.charge, "spin": mol.spin, "shells": shells_record(basis),
               "t_integrals_s": t_int, "E_nuc": float(ints.E_nuc)}
        arrays = {"S": np.asarray(ints.S), "T": np.asarray(ints.T), "V": np.asarray(ints.V)}
        if full_tensor:
            arrays["eri"] = eri
        if n_sample:
            idx = rng.integers(0, n, (n_sample, 4))
            arrays["eri_idx"] = idx
            arrays["eri_val"] = eri[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
        Dr = rng.standard_normal((n, n)) * 0.1
        Dr = Dr + Dr.T
        arrays["D_rand"] = Dr
        arrays["F_rand"] = np.asarray(build_fock_rhf(np.zeros((n, n)), Dr, eri))
        Db = rng.standard_normal((n, n)) * 0.1
        Db = Db + Db.T
        Fa, Fb = build_fock_uhf(np.zeros((n, n)), Dr, Db, eri)
        arrays["D_rand_b"] = Db
        arrays["Fa_rand"] = np.asarray(Fa)
        arrays["Fb_rand"] = np.asarray(Fb)
        arrays["Q"] = compute_shell_pair_bounds(basis)
        cfg = CalcConfig(method="uhf" if uhf else "rhf", basis=bname, scf_conv=1e-10)
        t0 = time.time()
        res = jax_qc.run_scf(rm, ints, cfg)
        rec["t_scf_s"] = time.time() - t0
        rec["energy"] = float(res.energy)
        rec["converged"] = bool(res.converged)
        rec["n_iterations"] = int(res.n_iterations)
        arrays["D_scf"] = np.asarray(res.state.density)
        if grad:
            t0 = time.time()
            g = np.asarray(rhf_gradient(rm, res, basis_name=bname, step_size=1e-4))
            rec["t_grad_s"] = time.time() - t0
            arrays["grad"] = g
        with open(os.path.join(HERE, f"{tag}.json"), "w") as f:
            json.dump(rec, f, indent=1)
        np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), **arrays)
        print(tag, "n=%d E=%.10f conv=%s its=%d t_int=%.1fs" % (n, rec["energy"], rec["converged"],
                                                               rec["n_iterations"], t_int))

    from jax_examples_b200.core import make_molecule as pmake

    if "core" in sections:
        water = pmake(("O", "H", "H"), pb.water_monomer_bohr(), np.array([8, 1, 1]))
        run_system("water_synsto3g", water, "syn-sto-3g", full_tensor=True, grad=True)
        cation = pmake(("O", "H", "H"), pb.water_monomer_bohr(), np.array([8, 1, 1]), charge=1, spin=1)
        run_system("water_cation_synsto3g_uhf", cation, "syn-sto-3g", full_tensor=False, uhf=True)
        run_system("water_syn631gs", water, "syn-6-31g*", full_tensor=False, n_sample=20000)

        # Tier-1 molecules (examples/07_rhf_scf.py:31-36 golden energies), STO-3G from
        # the reference's own parameter table.
        r = 1.65
        tier1 = {
            "H2": (("H", "H"), [[0, 0, 0], [0, 0, 1.4]], [1, 1], 0, -1.1167143251),
            "He": (("He",), [[0, 0, 0]], [2], 0, -2.8077839575),
            "HeH+": (("He", "H"), [[0, 0, 0], [0, 0, 1.4632]], [2, 1], 1, -2.8418364993),
            "H3+": (("H", "H", "H"), [[0, 0, 0], [r, 0, 0], [r / 2, r * np.sqrt(3) / 2, 0]], [1, 1, 1], 1, -1.2375476999),
        }
        out = {}
        for name, (el, xyz, Z, q, golden) in tier1.items():
            rm = make_molecule(elements=el, coords=np.array(xyz, dtype=float), atomic_numbers=np.array(Z), charge=q)
            basis = jax_qc.build_basis_set(rm, "sto-3g", use_cache=False, spherical=False)
            ints = jax_qc.compute_integrals(rm, basis)
            res = jax_qc.run_scf(rm, ints, CalcConfig(method="rhf", basis="sto-3g", scf_conv=1e-10))
            out[name] = {"elements": list(el), "coords": xyz, "Z": Z, "charge": q,
                         "reference_energy": float(res.energy), "golden_pyscf": golden,
                         "golden_source": "examples/07_rhf_scf.py:31-36"}
            print(name, float(res.energy), golden, float(res.energy) - golden)
        with open(os.path.join(HERE, "tier1_sto3g.json"), "w") as f:
            json.dump(out, f, indent=1)

    if "real" in sections:
        real_fixtures(run_system, ref_mol, pmake, jax_qc, CalcConfig, make_molecule)


def real_fixtures(run_system, ref_mol, pmake, jax_qc, CalcConfig, make_molecule) -> None:
    """Fixtures of the published bases: config-1 water (STO-3G, full tensor,
    FD gradient), its UHF cation, the 6-31G* (Cartesian) and 6-31G**
    (spherical, the reference default) water, and the example-08 energies."""
    from jax_examples_b200 import basis as pb

    rng = np.random.default_rng(20261204)
    water = pmake(("O", "H", "H"), pb.water_monomer_bohr(), np.array([8, 1, 1]))
    cation = pmake(("O", "H", "H"), pb.water_monomer_bohr(), np.array([8, 1, 1]), charge=1, spin=1)
    run_system("water_sto3g", water, "sto-3g", full_tensor=True, grad=True, rng=rng)
    run_system("water_cation_sto3g_uhf", cation, "sto-3g", full_tensor=False, uhf=True, rng=rng)
    run_system("water_631gs", water, "6-31g*", full_tensor=False, n_sample=20000, rng=rng)
    run_system("water_631gss_sph", water, "6-31g**", full_tensor=False, n_sample=20000, spherical=True, rng=rng)

    # examples/08_rhf_tier2.py:33-41: PySCF energies (spherical basis, bohr).
    rn, th = 1.913, np.deg2rad(106.7)
    sn, cs = np.sin(th / 2.0), np.cos(th / 2.0)
    rc = 2.052 / np.sqrt(3.0)
    mols = {
        "H2O": (("O", "H", "H"), [[0.0, 0.0, 0.117], [0.0, 0.757, -0.469], [0.0, -0.757, -0.469]], [8, 1, 1]),
        "HF": (("F", "H"), [[0.0, 0.0, 0.0], [0.0, 0.0, 1.7325]], [9, 1]),
        "CH4": (("C", "H", "H", "H", "H"), [[0, 0, 0], [rc, rc, rc], [rc, -rc, -rc], [-rc, rc, -rc], [-rc, -rc, rc]],
                [6, 1, 1, 1, 1]),
        "NH3": (("N", "H", "H", "H"), [[0, 0, 0], [rn * sn, 0, -rn * cs],
                                       [-rn * sn / 2, rn * sn * np.sqrt(3) / 2, -rn * cs],
                                       [-rn * sn / 2, -rn * sn * np.sqrt(3) / 2, -rn * cs]], [7, 1, 1, 1]),
    }
    pyscf = {("H2O", "sto-3g"): -73.2144728363, ("H2O", "6-31g"): -74.4943924164, ("H2O", "6-31g**"): -74.5428909110,
             ("HF", "sto-3g"): -98.5708712083, ("CH4", "sto-3g"): -39.7268589862, ("NH3", "sto-3g"): -55.4540090032}
    out = {}
    for (name, bname), golden in pyscf.items():
        el, xyz, Z = mols[name]
        rm = make_molecule(elements=el, coords=np.array(xyz, dtype=float), atomic_numbers=np.array(Z))
        basis = jax_qc.build_basis_set(rm, bname, use_cache=False, spherical=True)
        t0 = time.time()
        ints = jax_qc.compute_integrals(rm, basis)
        res = jax_qc.run_scf(rm, ints, CalcConfig(method="rhf", basis=bname, scf_conv=1e-10))
        out[f"{name}/{bname}"] = {"elements": list(el), "coords": np.asarray(xyz, dtype=float).tolist(), "Z": Z,
                                  "basis": bname, "spherical": True, "n_basis": int(basis.n_basis),
                                  "reference_energy": float(res.energy), "golden_pyscf": golden,
                                  "golden_source": "examples/08_rhf_tier2.py:33-41", "t_s": time.time() - t0}
        print(name, bname, float(res.energy), golden, float(res.energy) - golden)
    with open(os.path.join(HERE, "tier2_pyscf.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("JQC_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: gen_golden.py REFERENCE_ROOT [core|real|all] (or set JQC_REFERENCE_ROOT)")
    which = sys.argv[2] if len(sys.argv) > 2 else "all"
    main(root, ("core", "real") if which == "all" else (which,))
