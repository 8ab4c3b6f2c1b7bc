"""The reference-side bindings shown in the repository's integration guide
compile against the reference's own headers (CPU only; needs the reference
sources, so it is skipped where they are absent).

The dense driver shim (section 1), the complex shim (section 2) and the
sparse driver shim (section 2b) are cut out of the guide as a maintainer
would paste them, put in one translation unit after the
reference's headers (CommonFiles/Permanent.h, Structures/SparseMatrix.h,
CommonFiles/Helpers.h, Algorithms/Complex/gpuComputeComplex.cuh) and
include/superman_b200.h, with the driver templates instantiated for the
reference's <double, double> and <double, float> (Algorithms/GPU/
GPUKernelWrappers.cu:398-428), and compiled with g++ -fsyntax-only.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_tree():
    """The reference source tree: $SPB_REFERENCE_TREE, else the REF default
    of oracle/Makefile (the recipe that builds the reference's CPU program)."""
    if os.environ.get("SPB_REFERENCE_TREE"):
        return os.environ["SPB_REFERENCE_TREE"]
    m = re.search(r"^REF \?= (\S+)", open(os.path.join(ROOT, "oracle", "Makefile")).read(), re.M)
    return m.group(1) if m else ""


REF = _reference_tree()


def _section_block(text, heading):
    start = text.index(heading)
    m = re.search(r"```cpp\n(.*?)```", text[start:], re.S)
    assert m, heading
    return m.group(1)


def test_integration_shims_compile_against_the_reference_headers(tmp_path):
    if not os.path.exists(os.path.join(REF, "CommonFiles", "Permanent.h")):
        pytest.skip("reference sources not present on this machine")
    gxx = shutil.which("g++") or "/usr/bin/g++"
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    dense = _section_block(doc, "## 1. Dense real path")
    cplx = _section_block(doc, "## 2. Complex path")
    sparse = _section_block(doc, "## 2b. Sparse path")
    unit = "\n".join([
        "#include <complex>", "#include <iomanip>", "#include <sstream>",
        '#include "Permanent.h"', '#include "SparseMatrix.h"', '#include "Helpers.h"',
        '#include "gpuComputeComplex.cuh"', '#include "superman_b200.h"',
        "// globals the reference's main.cpp defines (CommonFiles/Settings.h:30-34)",
        "double avgN = 0; double avgNNZ = 0; unsigned count = 0; bool printing = true; bool sparse = false;",
        dense, cplx, sparse,
        "template class spbSingleGPU<double, double>;",
        "template class spbSingleGPU<double, float>;",
        "template class spbSparseSingleGPU<double, double>;",
        "template class spbSparseSingleGPU<double, float>;",
    ])
    src = tmp_path / "shims.cpp"
    src.write_text(unit)
    inc = [os.path.join(REF, d) for d in ("Structures", "CommonFiles", "IO", "Algorithms",
                                           "Algorithms/Complex", "Algorithms/CPU/Dense",
                                           "Algorithms/CPU/Sparse")]
    cmd = [gxx, "-std=c++17", "-fsyntax-only", "-fopenmp", "-I", os.path.join(ROOT, "include")]
    for d in inc:
        cmd += ["-I", d]
    cmd.append(str(src))
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
