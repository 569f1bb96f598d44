"""Generate the golden fixtures in this folder from the REFERENCE's own code.

Runs the reference's hot-path templates, compiled from its source tree into
oracle/_ref/libqsref.so (oracle/Makefile, oracle/ref_entry.cpp), on small
seeded inputs and stores the outputs.  Inputs are regenerated from the seeds
by the tests (numpy PCG64), and each fixture stores input checksums so RNG
drift is detected.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

from cases import CASES, SCF_C0, scf_inputs  # noqa: E402
import scf_oracle as S  # noqa: E402


def main(only=None):
    """All fixtures, or only the named cases (python make_golden.py NAME ...)."""
    assert O.ref_available(), "build oracle/_ref first: make -C oracle ref"
    for name, case in CASES.items():
        if only and name not in only:
            continue
        inp = case["inputs"]()
        out = case["reference"](inp)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), out=out,
                            checksum=np.array([float(np.sum(v)) for v in inp["checked"]]))
        print(name, out.shape, float(np.linalg.norm(out)))
    if not only or "scf_kpt" in only:
        # k-point SCF: the oracle loop with the reference's Eigen_z_multi_mpi per k-point
        from cases import SCF_KPT, scf_kpt_inputs
        inp = scf_kpt_inputs()
        r = S.scf_kpoints(inp["grid"], inp["pos"], inp["sp"], SCF_KPT["nb"], SCF_KPT["n_el"], inp["Xs"], inp["kvecs"],
                          inp["weights"], **SCF_KPT["params"])
        np.savez_compressed(os.path.join(HERE, "scf_kpt.npz"), energies=r["energies"], rq=r["rq"], occ=r["occ"],
                            rho=r["rho"], checksum=np.array([float(np.sum(v)) for v in inp["checked"]]))
        print("scf_kpt", r["steps"], r["energies"][-1])
    if not only or "scf_c0_pbe" in only:
        # the same SCF with the GGA-PBE (restated, pinned to the reference's
        # mSetPotentialVxc by the gga_pbe case)
        inp = scf_inputs()
        r = S.scf(inp["grid"], inp["pos"], inp["sp"], SCF_C0["nb"], SCF_C0["n_el"], inp["X"], xc="pbe",
                  **SCF_C0["params"])
        np.savez_compressed(os.path.join(HERE, "scf_c0_pbe.npz"), energies=r["energies"], rq=r["rq"], occ=r["occ"],
                            rho=r["rho"], converged=np.array(r["converged"]),
                            checksum=np.array([float(np.sum(v)) for v in inp["checked"]]))
        print("scf_c0_pbe", r["steps"], r["energies"][-1])
    if only and "scf_c0" not in only:
        return
    # SCF of config 0: the oracle loop (reference LOBPCG + restated SCF pieces)
    inp = scf_inputs()
    r = S.scf(inp["grid"], inp["pos"], inp["sp"], SCF_C0["nb"], SCF_C0["n_el"], inp["X"], **SCF_C0["params"])
    np.savez_compressed(os.path.join(HERE, "scf_c0.npz"), energies=r["energies"], rq=r["rq"], occ=r["occ"],
                        rho=r["rho"], vloc=r["vloc"], converged=np.array(r["converged"]),
                        checksum=np.array([float(np.sum(v)) for v in inp["checked"]]))
    print("scf_c0", r["steps"], r["energies"][-1])


if __name__ == "__main__":
    main(sys.argv[1:] or None)
