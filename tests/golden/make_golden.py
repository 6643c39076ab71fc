"""Generates the golden fixtures tests/golden/<case>.npz by running the reference's own CPU
assembly (oracle/_ref, built from the reference sources by oracle/Makefile) on the cases of
tests/golden/cases.py.  Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, case_arrays, cohesive_state, spec_kwargs  # noqa: E402
from oracle import ref  # noqa: E402


def effective_openings(c, U, R):
    """The effective opening of every cohesive point under U.  Laws that write their maximum
    opening report it as the trial internal variable of the assembly R just ran; the plain
    trilinear laws never write it, so an Ortiz-Pandolfi twin of the same mesh (one internal
    variable per point, set to the effective opening on first loading) measures it."""
    if c["coh_law"] not in (9, 11):
        return R.get("isv_trial")
    twin = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(dict(c, coh_law=5, coh=(50.0, 2e-4, 1.0, 0.0)))))
    try:
        twin.assemble(U, np.zeros(len(R.get("isv_trial"))), 1.0)
        return twin.get("isv_trial")
    finally:
        twin.close()


def generate(name):
    """The fixture arrays of one case, computed by the reference's own CPU assembly."""
    c = CASES[name]
    R = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(c)))
    try:
        n_isv = int(R.get("isv_off")[-1])
        if c["coh_law"]:
            U = cohesive_state(c, R.get("node_dofs"), R.n_free, R.n_const, R.get("elem_node_off"), R.get("elem_nodes"),
                               R.get("elem_cut"), R.get("elem_coh_off"), R.get("coh_struct"), R.get("coh_struct_off"),
                               R.get("coh_qp_off"), R.get("coh_qp_R"))
            isv = np.zeros(n_isv)
            if c["isv_scale"] > 0 and n_isv:
                # committed maxima around the current openings: about half the points unload
                R.assemble(U, isv, 1.0)
                rng = np.random.default_rng(c["seed"] + 1000)
                isv = effective_openings(c, U, R) * rng.uniform(0.5, 1.5, n_isv)
        else:
            U, isv = case_arrays(c, R.n_free, R.n_const, n_isv)
        t_frac = 1.0
        R.assemble(U, isv, t_frac)
        out = dict(U_dof=U, isv_committed=isv, t_frac=np.array([t_frac]), node_dofs=R.get("node_dofs"), isv_off=R.get("isv_off"),
                   isv_elem_qp_off=R.get("isv_elem_qp_off"), P_f=R.get("P_f"), P_p=R.get("P_p"),
                   isv_trial=R.get("isv_trial"), coh_zone=R.get("coh_zone"),
                   node_coords=R.get("node_coords"), enrich_coords=R.get("enrich_coords"))
        for b in ("K_ff", "K_fp", "K_pf", "K_pp"):
            rp, ci, v, sh = R.csr(b)
            out[b + "_rowptr"], out[b + "_cols"], out[b + "_vals"] = rp, ci, v
        out = {k: np.array(v, copy=True) for k, v in out.items()}
        return out, (R.n_free, R.n_const, n_isv)
    finally:
        R.close()


def main(names=None):
    for name in CASES:
        if names and name not in names:
            continue
        out, (n_free, n_const, n_isv) = generate(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "free", n_free, "const", n_const, "nnz_ff", len(out["K_ff_vals"]), "isv", n_isv)


if __name__ == "__main__":
    main(sys.argv[1:])
