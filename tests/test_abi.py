"""The C ABI library: it loads without a GPU, exports every function the
headers declare, and fails loudly (no CPU fallback) when no GPU is present."""
import os
import re

import pytest

import paratt_b200 as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = ["paratt.h", "paratt_ode.h", "paratt_b200.h"]


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^\s*(?:PTT_API\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M):
        name = m.group(1)
        if name not in ("if", "defined", "sizeof"):
            names.add(name)
    return names


@pytest.mark.parametrize("header", HEADERS)
def test_library_exports_every_declared_function(header):
    lib = P.lib()
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_no_gpu_fails_loudly():
    import ctypes as C

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(P.PttError) as e:
        P.Context(0)
    assert e.value.code == P.PTT_ERR_NOGPU
    assert b"no CPU" in P.lib().ptt_last_error_message() or b"CUDA" in P.lib().ptt_last_error_message()


def test_checkpoint_argument_errors():
    """The checkpoint and resume entry points reject null trains and paths
    before touching a device (no GPU needed)."""
    import paratt_b200 as P
    L = P.lib()
    assert not L.ptt_checkpoint_begin(None, b"/tmp/x")
    assert L.ptt_checkpoint_wait(None) != 0
    assert L.ptt_tt_load_folder(None, b"/tmp/x") != 0
