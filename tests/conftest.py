"""Test configuration: puts the package and the oracle on sys.path and registers the `gpu` mark.

`-m "not gpu"` runs here (no GPU): the oracle against the golden fixtures, host-side logic, and the
C-ABI library's load/export/argument checks.  `-m gpu` runs on a B200 and compares the CUDA path,
called through the C ABI, with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "plasma-etching-code_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


@pytest.hookimpl(hookwrapper=True)
def pytest_runtest_call(item):
    """Print a failing test's exception at once, before the report is formatted: after a CUDA
    fault the context is unusable, and freeing a device tensor while the report is built can
    abort the process before the message is shown."""
    outcome = yield
    exc = outcome.excinfo
    if exc is not None and not isinstance(exc[1], (AssertionError, pytest.skip.Exception)):
        sys.stderr.write(f"\n[{item.nodeid}] {exc[0].__name__}: {exc[1]}\n")
        sys.stderr.flush()
