"""The C-ABI library loads, exports every entry point include/petch_b200.h declares, and rejects
bad arguments with PETCH_E_INVALID before touching the device.  CPU only (no kernel runs)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from petch_b200 import _lib

HEADER = os.path.join(ROOT, "include", "petch_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(petch_\w+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    so = _lib.lib()
    names = declared()
    assert len(names) >= 4
    for n in names:
        assert hasattr(so, n), f"{n} declared in the header but not exported"
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_abi_version():
    assert _lib.lib().petch_abi_version() >= 1


@pytest.mark.parametrize("name,args", [
    ("petch_advect", [None, None, None, None, None, 4, 4, 4, 1.0, 0.1, 1, None]),
    ("petch_reinit_eik", [None, None, None, None, 4, 4, 4, 0.25, 1.0, 1.0, 3, 0, None]),
    ("petch_seed_level_set", [None, None, 4, 4, 4, 0.25, 1.0, 1.0, 0.5, 0.2, 0.4, 1, None]),
    ("petch_plan", [None, None, 1, None, None]),
    ("petch_step", [None, None]),
    ("petch_plan_status", [None, None, None]),
    ("petch_plan_seek", [None, 0]),
])
def test_null_pointers_rejected(name, args):
    rc = getattr(_lib.lib(), name)(*args)
    assert rc == 1  # PETCH_E_INVALID
    assert "null" in _lib.last_error()


def test_plan_rejects_bad_configuration_before_touching_the_device():
    """petch_plan checks the configuration first: a bad grid or ray count is PETCH_E_INVALID with
    a message, and nothing is allocated (no GPU needed)."""
    c = _lib.StepConfig()
    c.nx, c.ny, c.nz, c.dx, c.dt, c.max_tris = 0, 4, 4, 0.25, 0.1, 1024
    h = ctypes.c_void_p()
    phi = ctypes.c_float(0.0)
    rc = _lib.lib().petch_plan(ctypes.byref(c), ctypes.addressof(phi), 1, ctypes.byref(h), None)
    assert rc == 1 and "bad grid" in _lib.last_error() and not h.value
    c.nx, c.n_neu = 4, 1 << 29
    rc = _lib.lib().petch_plan(ctypes.byref(c), ctypes.addressof(phi), 1, ctypes.byref(h), None)
    assert rc == 1 and "ray counts" in _lib.last_error()
    assert _lib.lib().petch_destroy(None) == 0
