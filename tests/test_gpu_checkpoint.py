"""Checkpoint / resume of device trains in the reference's .cr core file
format (pattac_write_tt_folder / pattac_load_tt_folder, paratt.c:1621-1892):
the files hold the snapshot taken when the checkpoint started, in the
reference's exact text format, and loading them back restores the train bit
for bit."""
import os

import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu


def _expected_text(core):
    rl, n, rr = core.shape
    return f"{rl},{n},{rr}\n" + "".join(f"{v:+1.16e}\n" for v in core.ravel(order="F"))


def test_checkpoint_write_behind_and_resume(ctx, tmp_path):
    dims, ranks = [7, 5, 9, 4], [1, 3, 6, 2, 1]
    x = O.random_tt(dims, ranks, 21)
    X = P.TT.from_cores(ctx, x)
    folder = str(tmp_path / "ck")
    cp = X.checkpoint(folder)
    X.scale(2.0)  # queued after the snapshot: not in the files
    cp.wait()
    for k, core in enumerate(x):
        with open(os.path.join(folder, f"core_{k + 1}.cr")) as f:
            assert f.read() == _expected_text(core)
    for a, b in zip(X.get(), O.scale(2.0, x)):
        np.testing.assert_array_equal(a, b)
    Y = P.TT(ctx, dims, [1] * (len(dims) + 1))
    Y.load_folder(folder)
    for a, b in zip(Y.get(), x):
        np.testing.assert_array_equal(a, b)
    Y.close()
    X.close()


def test_resume_rejects_mismatched_folder(ctx, tmp_path):
    x = O.random_tt([4, 4, 4], [1, 2, 2, 1], 22)
    X = P.TT.from_cores(ctx, x)
    folder = str(tmp_path / "ck2")
    X.checkpoint(folder).wait()
    Y = P.TT(ctx, [4, 5, 4], [1, 1, 1, 1])  # mode 1 differs
    with pytest.raises(P.PttError):
        Y.load_folder(folder)
    Y.close()
    X.close()
