#!/usr/bin/env python3
"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own C (oracle/_ref/libparatt_ref.so, built by
`make -C oracle` from the reference sources) on seeded inputs and stores
inputs and outputs as .npz; also stores the values of one initial-condition
core file shipped with the reference (gaussian_dim_20/core_1.cr) and a .cr
folder written by the reference's pattac_write_tt_folder.  Needs the
reference checkout ($PARATT_REFERENCE, else a folder named `reference` beside
this repository); the fixtures are what the
tests read, so the tests themselves never need the reference.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("PARATT_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))

from oracle import ref_lib as R  # noqa: E402
from oracle import tt_oracle as O  # noqa: E402


def pack(prefix, cores):
    out = {f"{prefix}_ranks": np.array(O.ranks_of(cores)), f"{prefix}_dims": np.array(O.dims_of(cores))}
    for k, c in enumerate(cores):
        out[f"{prefix}_{k}"] = c.ravel(order="F")
    return out


def main():
    # rounding cases (tol is absolute on the RMS norm, as paratt_truncate takes it)
    cases = [
        ([6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1], 1, 1e-1, 10),
        ([6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1], 2, 1e-6, 10),
        ([8, 8, 8, 8], [1, 6, 9, 6, 1], 3, 1e-3, 4),
        ([4] * 7, [1, 3, 5, 6, 6, 5, 3, 1], 4, 1e-8, 64),
    ]
    for i, (dims, ranks, seed, rtol, mr) in enumerate(cases):
        x = O.random_tt(dims, ranks, seed)
        z = O.axpby(1.0, x, 0.5, O.random_tt(dims, ranks, seed + 100))
        tol = rtol * O.norm(z)
        out = R.ref_truncate(z, tol, mr)
        np.savez(os.path.join(HERE, f"round_{i}.npz"), tol=tol, maxrank=mr, **pack("in", z), **pack("out", out))
    # formal ops and contractions
    x = O.random_tt([6, 5, 7, 4], [1, 3, 4, 2, 1], 11)
    y = O.random_tt([6, 5, 7, 4], [1, 2, 3, 3, 1], 12)
    d = {}
    d.update(pack("x", x))
    d.update(pack("y", y))
    d.update(pack("axpby", R.ref_axpby(0.75, x, -1.5, y)))
    d.update(pack("had", R.ref_hadamard(x, y)))
    for m in range(4):
        d.update(pack(f"sten{m}", R.ref_stencil(x, m, [1.0, -2.0, 1.0])))
    d["norm"] = R.ref_norm(x)
    d["dot"] = R.ref_dot(x, y)
    d["entry_idx"] = np.array([5, 4, 6, 3])
    d["entry"] = R.ref_entry(x, [5, 4, 6, 3])
    np.savez(os.path.join(HERE, "ops.npz"), **d)
    # the reference's initial-condition core file (values only)
    fn = os.path.join(REF, "gaussian_dim_20", "core_1.cr")
    with open(fn) as f:
        head = f.readline().strip()
        vals = np.array([float(l) for l in f if l.strip()])
    np.savez(os.path.join(HERE, "ic_core.npz"), header=np.array([int(t) for t in head.split(",")]), values=vals)
    # a .cr folder written by the reference's pattac_write_tt_folder
    folder = os.path.join(HERE, "cr_written_by_reference")
    shutil.rmtree(folder, ignore_errors=True)
    t = R.RefTT(O.random_tt([3, 4, 2], [1, 2, 3, 1], 21))
    R.lib().pattac_write_tt_folder(folder.encode(), t.p)
    np.savez(os.path.join(HERE, "cr_values.npz"), **pack("x", t.cores()))
    t.free()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
