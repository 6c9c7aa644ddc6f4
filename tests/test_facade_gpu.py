"""The C++ drop-in facade (include/physxcoopa_b200.hpp) driven by physxcoopa's own code: the
reference's builders, solve_cloth and solve_strands on one copy, the facade on the device on the
other, equal particle for particle (tests/facade/facade_check.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "facade", "_build", "facade_check")


@pytest.mark.gpu
def test_cpp_facade_equals_reference_solvers():
    assert os.path.exists(BIN), "facade_check was not built (run __graft_entry__.build())"
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "facade ok" in r.stdout
