"""Regenerates the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

The fixtures pin (a) the analytic known answers of the reference's
generate_matrix / cg (nnz = (3nx-2)(3ny-2)(3nz-2), b = A*1, Initial Residual
= ||b||, x -> 1) and (b) the oracle's FP64 residual histories, so GPU runs can
be checked without rebuilding the oracle and a change to the oracle shows up
as a fixture diff; (c) the multi-rank halo plans (make_local_matrix in the MPI
and CAF-V2 forms) and multi-rank CG histories of a few small communicators.
The reference itself (Fortran 90) cannot be run here.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402

CG_CASES = [(16, 16, 16, 150), (32, 32, 32, 150), (3, 5, 7, 150), (2, 2, 2, 150), (1, 1, 1, 150),
            (7, 1, 3, 150)]
CSR_CASES = [(3, 5, 7), (4, 4, 4), (1, 2, 3), (2, 1, 1)]
# multi-rank halo plans: (nx, ny, nz per rank, ranks); both the MPI and the CAF-V2 form
SLAB_CASES = [(4, 3, 2, 2), (4, 3, 2, 3), (3, 3, 1, 3)]
SLAB_FIELDS = ("colindex", "externals", "external_owners", "neighbors", "recv_length", "recv_length_literal",
               "send_length", "elements_to_send", "blocks", "remote_index")


def main():
    known = {"nnz": {}, "iters_to_1e-8": {}, "initial_residual": {}}
    for nx, ny, nz in CSR_CASES:
        A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
        np.savez_compressed(os.path.join(HERE, f"csr_{nx}x{ny}x{nz}.npz"), rowindex=A.rowindex,
                            colindex=A.colindex, values=A.values, b=b)
    for nx, ny, nz, it in CG_CASES:
        A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
        xs, niters, normr, hist = oracle.cg(A, b, x, it, 0.0)
        key = f"{nx}x{ny}x{nz}"
        known["nnz"][key] = A.nnz
        known["initial_residual"][key] = float(np.sqrt(np.dot(b, b)))
        below = np.nonzero(hist / hist[0] <= 1e-8)[0]
        known["iters_to_1e-8"][key] = int(below[0]) if len(below) else None
        np.savez_compressed(os.path.join(HERE, f"cg_{key}.npz"), hist=hist, niters=niters, normr=normr,
                            x=xs if A.nrow <= 4096 else np.empty(0), max_err=np.abs(xs - 1).max())
    for nx, ny, nz, P in SLAB_CASES:
        G, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
        for mode, tag in ((oracle.HALO_MPI, "mpi"), (oracle.HALO_GET, "get")):
            plan = oracle.SlabPlan(nx, ny, nz, P, mode)
            arrays = {f"r{r}_{k}": plan.get(r, k) for r in range(P) for k in SLAB_FIELDS}
            _, it, _, hist = plan.cg(bg, x0, 30, 0.0)
            np.savez_compressed(os.path.join(HERE, f"slab_{nx}x{ny}x{nz}x{P}_{tag}.npz"), hist=hist, **arrays)
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
