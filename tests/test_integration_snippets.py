"""The C++ snippets of INTEGRATION.md compile against the shipped headers
(include/laph_gpu.h, include/laph_matshell.h over include/petsc_shim.h), each
inside a function that declares the surrounding variables of the reference's
ev_ts / tune_hyp loop -- so the integration guide cannot drift from the ABI."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PREAMBLE = r"""
#include <cstdio>
#include <vector>
#include "laph_matshell.h"
struct ref_io { double get_float(const char*); int get_int(const char*); };  // the reference's IO singleton
"""

# variables the reference's ev_ts / tune_hyp have in scope where each snippet goes
SCOPE = r"""
  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;
"""


def snippets():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, re.S)


def test_integration_snippets_compile(tmp_path):
    blocks = snippets()
    assert len(blocks) >= 4
    src = [PREAMBLE]
    for i, b in enumerate(blocks):
        b = b.replace("#define LAPH_USE_REAL_PETSC", "// (real PETSc in the guide; the shim here)")
        b = "\n".join(ln for ln in b.splitlines() if not ln.startswith("#include"))
        # the snippets that use a solver handle without creating it get one from the scope
        needs_s = "laph_solver* s;" not in b and re.search(r"\bs\b", b)
        src.append(f"int snippet_{i}() {{\n{SCOPE}\n" + ("  laph_solver* s = nullptr;\n" if needs_s else "")
                   + b + "\n  return 0;\n}\n")
    f = tmp_path / "snippets.cpp"
    f.write_text("".join(src))
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                        "-I" + os.path.join(ROOT, "include"), str(f)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
