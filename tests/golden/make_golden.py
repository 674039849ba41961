"""Generate tests/golden/ fixtures by running the unmodified reference.

Needs the reference harness (oracle/_ref/libowtk_ref.so, built by
`make -C oracle ref` from the read-only reference sources).  The fixtures pin
the C restatement in oracle/ and the device results without the reference.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "owt-krylov_b200"), os.path.join(REPO, "tests")]

import oracle  # noqa: E402
import cases  # noqa: E402
from owtk_b200 import problems  # noqa: E402


def solver_options(**kw):
    return oracle.default_options(**kw)


def main():
    ref = oracle.Reference()
    out = {}
    # --------------------------------------------------------- kernels
    for name in cases.SPMV_CASES:
        c = cases.build(name)
        n, g, bs = c["owned"], c["ghost"], c["bs"]
        m = ref.matrix("bsr", n, g, bs, c["rowptr"], c["cols"], c["vals"])
        out[f"{name}/x"] = c["x"]
        out[f"{name}/spmv"] = m.apply(c["x"])[: n * bs]
        out[f"{name}/jacobi"] = ref.pc("jacobi", m).apply(c["x"])[: n * bs]
        for om in (1.0, 1.3):
            out[f"{name}/ssor{om}"] = ref.pc("ssor", m, om).apply(c["x"])[: n * bs]
        orp, oci, diag, off = cases.split_of(c)
        sm = ref.matrix("split", n, g, bs, orp, oci, diag=diag, off=off)
        out[f"{name}/split_spmv"] = sm.apply(c["x"])[: n * bs]
        for om in (1.0, 1.4):
            out[f"{name}/split_ssor{om}"] = ref.pc("split_ssor", sm, om).apply(c["x"])[: n * bs]
        if name in cases.ILU_CASES:
            for k in (0, 1, 2):
                p = ref.pc("ilu", m, k)
                rp, ci, v, inv = p.ilu_factors()
                out[f"{name}/ilu{k}_rowptr"] = rp
                out[f"{name}/ilu{k}_cols"] = ci
                out[f"{name}/ilu{k}_vals"] = v
                out[f"{name}/ilu{k}_inv"] = inv
                out[f"{name}/ilu{k}_apply"] = p.apply(c["x"])[: n * bs]
    for name, kw in cases.DENSE_CASES.items():
        c = cases.dense_case(**kw)
        m = ref.matrix("dense", c["owned"], 0, c["bs"], c["rowptr"], c["cols"], c["vals"])
        out[f"{name}/x"] = c["x"]
        out[f"{name}/spmv"] = m.apply(c["x"])
    # --------------------------------------------------------- orderings
    c0 = problems.config0()
    out["cfg0/rcm"] = ref.rcm(c0.owned, c0.rowptr, c0.cols).astype(np.int32)
    out["cfg0/hilbert"] = ref.hilbert(c0.xy).astype(np.int32)
    lat = cases.build("lattice8_bs3")
    out["lattice8_bs3/rcm"] = ref.rcm(lat["owned"], lat["rowptr"], lat["cols"])
    out["lattice8_bs3/hilbert"] = ref.hilbert(lat["xy"])
    # --------------------------------------------------------- solves
    solves = {}
    small = cases.lattice_case(side=24, bs=3, seed=21)
    out["solve24/rhs"] = small["rhs"]
    bench = dict(maximum_iterations=1000, convergence_check_interval=1, residual_replacement_interval=50)
    specs = [
        ("bicgstab_jacobi", "bicgstab", "jacobi", 0.0, dict(bench)),
        ("bicgstab_ilu", "bicgstab", "ilu", 0.0, dict(bench)),
        ("gmres_ilu", "gmres", "ilu", 0.0, dict(restart=30)),
        ("gmres_jacobi_cgs2", "gmres", "jacobi", 0.0, dict(restart=40, **bench)),
        ("gmres_jacobi_onesync", "gmres", "jacobi", 0.0, dict(restart=40, gmres_orthogonalization=2, **bench)),
        ("gmres_jacobi_adaptive", "gmres", "jacobi", 0.0, dict(restart=10, gmres_orthogonalization=1)),
        ("pipelined_jacobi", "pipelined_bicgstab", "jacobi", 0.0, dict(bench)),
        ("commhiding_jacobi", "comm_hiding_bicgstab", "jacobi", 0.0, dict(bench)),
        ("idrs4_jacobi", "idrs", "jacobi", 0.0, dict(bench)),
        ("idrs2_ssor", "idrs", "ssor", 1.0, dict(idr_shadow_space=2)),
        ("gmres_identity_restart5", "gmres", "identity", 0.0, dict(restart=5, maximum_iterations=40)),
    ]
    for case_name, sysm in (("solve24", small), ("cfg0", None)):
        if sysm is None:
            sysm = dict(owned=c0.owned, ghost=0, bs=c0.bs, rowptr=c0.rowptr, cols=c0.cols, vals=c0.vals,
                        rhs=c0.rhs)
        m = ref.matrix("bsr", sysm["owned"], 0, sysm["bs"], sysm["rowptr"], sysm["cols"], sysm["vals"])
        for key, solver, pck, par, kw in specs:
            p = ref.pc(pck, m, par)
            r, x = ref.solve(solver, m, p, solver_options(**kw), sysm["rhs"], np.zeros_like(sysm["rhs"]))
            d = {k: v for k, v in r.as_dict().items() if k != "solve_seconds"}
            d["x_norm"] = float(np.linalg.norm(x))
            d["options"] = kw
            d["solver"], d["pc"], d["parameter"] = solver, pck, par
            solves[f"{case_name}/{key}"] = d
            if case_name == "solve24":
                out[f"solve24/{key}/x"] = x
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"), **out)
    with open(os.path.join(HERE, "reference_solves.json"), "w") as f:
        json.dump(solves, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} arrays and {len(solves)} solves")


if __name__ == "__main__":
    main()
