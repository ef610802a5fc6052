"""The reference's own driver program on the drop-in library.

The Burgers-Hopf CDF driver of the reference
(mpi_pattac_rxn_burgers_rank_max_read_file.c: a TT initial condition read
from a `.cr` folder, marginal trapezoid sums, then time steps of
attac_tt_axpby, paratt_truncate and the CDF stencil right-hand side, with
marginal CDFs and TT folders written every 0.001 time units) is compiled
unmodified from the reference tree by oracle/Makefile twice: linked against
the compiled reference library (CPU, the checker) and against
libparatt_b200.so (every call on the GPU through the reference API's host
mirrors).  Both run the same 100 steps (dt 1e-5 fixed in the driver, rank
cap 5, d = 6, n = 64) from the same seeded initial condition, each in its own
directory; everything the driver writes must agree: the printed TT ranks,
the 1-D and 2-D marginal CDFs (`.m` files, relative difference <= 1e-9 of
their largest value) and the TT folders at t = 0 and t = 0.001 (equal ranks,
relative difference as tensors <= 1e-9).  The measured differences and the
two run times (the driver's own timing log) are printed."""
import glob
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "..", "oracle", "_ref", "cdf_driver_ref")
B200_BIN = os.path.join(HERE, "..", "oracle", "_ref", "cdf_driver_b200")
D, N, RMAX = 6, 64, 5

needs = pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(B200_BIN)),
                           reason="driver binaries not built (make -C oracle)")


def write_ic(folder):
    """Seeded Gaussians per mode, one `1,64,1` core each, in the reference's
    `.cr` text format (header r_l,N,r_r, values %+1.16e)."""
    os.makedirs(folder)
    x = np.linspace(-1.3, 1.3, N)
    for k in range(D):
        v = np.exp(-(x - 0.1 * k) ** 2 / (2 * 0.3 ** 2)) / (0.3 * np.sqrt(2 * np.pi))
        with open(os.path.join(folder, f"core_{k + 1}.cr"), "w") as f:
            f.write(f"1,{N},1\n")
            f.writelines("%+1.16e\n" % a for a in v)


def run(binary, wd):
    write_ic(os.path.join(wd, "ic6"))
    out = subprocess.run([os.path.abspath(binary), "ic%d", str(D), str(RMAX), "1e-5", "0.0", "0.001", "0"],
                         cwd=wd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    ranks = re.findall(r"tt rank:\n([\d\t ]+)\n", out.stdout)
    log = open(glob.glob(os.path.join(wd, "kse_cdf_timing_nprocs=*.log"))[0]).read().split()
    return ranks, float(log[-1])


def read_m(path):
    """Every value of a matlabTensorPrint file (%+1.16e numbers, 1-D or 2-D)."""
    return np.array([float(v) for v in re.findall(r"[-+]\d\.\d+e[-+]\d+", open(path).read())])


def read_cr_folder(folder):
    cores = []
    for k in range(D):
        with open(os.path.join(folder, f"core_{k + 1}.cr")) as f:
            rl, n, rr = (int(v) for v in f.readline().split(","))
            vals = np.array([float(v) for v in f.read().split()])
        cores.append(vals.reshape((rl, n, rr), order="F"))
    return cores


@needs
def test_reference_driver_on_the_drop_in_library(tmp_path):
    wr, wg = str(tmp_path / "ref"), str(tmp_path / "b200")
    os.makedirs(wr)
    os.makedirs(wg)
    ranks_r, t_r = run(REF_BIN, wr)
    ranks_g, t_g = run(B200_BIN, wg)
    assert len(ranks_r) == 2 and ranks_g == ranks_r
    files = sorted(os.path.relpath(p, wr) for p in glob.glob(os.path.join(wr, "data", "**", "*"), recursive=True)
                   if os.path.isfile(p))
    files_g = sorted(os.path.relpath(p, wg) for p in glob.glob(os.path.join(wg, "data", "**", "*"), recursive=True)
                     if os.path.isfile(p))
    assert files == files_g and files
    worst_m = 0.0
    for f in files:
        if f.endswith(".m"):
            a, b = read_m(os.path.join(wr, f)), read_m(os.path.join(wg, f))
            assert a.shape == b.shape and a.size > 0
            worst_m = max(worst_m, float(np.max(np.abs(a - b)) / max(np.max(np.abs(a)), 1e-300)))
    worst_tt = 0.0
    for folder in sorted({os.path.dirname(f) for f in files if f.endswith(".cr")}):
        a, b = read_cr_folder(os.path.join(wr, folder)), read_cr_folder(os.path.join(wg, folder))
        assert O.ranks_of(a) == O.ranks_of(b)
        worst_tt = max(worst_tt, O.rel_diff_exact(b, a))
    print(f"driver: ranks {ranks_g[-1].split()}, marginals {worst_m:.2e}, TT folders {worst_tt:.2e}; "
          f"reference C {t_r:.2f} s, libparatt_b200 {t_g:.2f} s")
    assert worst_m <= 1e-9, worst_m
    assert worst_tt <= 1e-9, worst_tt
    shutil.rmtree(str(tmp_path), ignore_errors=True)
