"""The integration examples (laph_eigsys_b200/host/integration_examples.cpp:
the binding code that goes into the reference's ev_ts / tune_hyp, each block
inside a function that declares the variables the reference has in scope
there) compile against the shipped headers (include/laph_gpu.h,
include/laph_matshell.h over include/petsc_shim.h), so the examples cannot
drift from the ABI."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXAMPLES = os.path.join(ROOT, "laph_eigsys_b200", "host", "integration_examples.cpp")


def test_integration_examples_compile():
    src = open(EXAMPLES).read()
    assert len(re.findall(r"^int example_\d+\(\)", src, re.M)) >= 4
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                        "-I" + os.path.join(ROOT, "include"), EXAMPLES], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
