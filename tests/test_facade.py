"""The C++ facade (include/pdlpgpu.hpp) as the reference's callers would use
it: a program written against the reference's own headers and types calls
`pdlp::PdlpSolver::solve` and `pdlpgpu::PdlpSolver::solve` on the same
`pdlp::CompiledLp` and `pdlp::PdlpOptions`. The cases are the ones decided
before any device work (invalid problems and options), so the test needs no
GPU; it needs the reference's headers and the oracle library built from the
reference's sources, and is skipped where they are absent.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref")
OUR_LIB = os.path.join(ROOT, "optimisation_solver_b200", "_lib")

PROGRAM = r"""
#include "pdlpgpu.hpp"
#include "pdlp/pdlp_solver.h"

#include <cmath>
#include <cstdio>
#include <functional>
#include <vector>

static pdlp::CompiledLp base() {
    std::vector<pdlp::MatrixTriplet> t = {{0, 0, 1.0}, {0, 1, 2.0}, {1, 2, -1.0}, {1, 0, 0.5}};
    pdlp::CompiledLp lp;
    lp.matrix = pdlp::SparseMatrix::fromTriplets(2, 3, t);
    lp.objective = {1.0, 1.0, 1.0};
    lp.variableLower = {0.0, 0.0, 0.0};
    lp.variableUpper = {1.0, 1.0, 1.0};
    lp.rowLower = {0.0, -1.0};
    lp.rowUpper = {1.0, 1.0};
    return lp;
}

int main() {
    std::vector<std::function<void(pdlp::CompiledLp&, pdlp::PdlpOptions&)>> cases = {
        [](pdlp::CompiledLp& lp, pdlp::PdlpOptions&) { lp.rowLower[1] = 2.0; },
        [](pdlp::CompiledLp& lp, pdlp::PdlpOptions&) { lp.variableLower[2] = 3.0; },
        [](pdlp::CompiledLp& lp, pdlp::PdlpOptions&) { lp.objective[0] = std::nan(""); },
        [](pdlp::CompiledLp& lp, pdlp::PdlpOptions&) { lp.objectiveOffset = INFINITY; },
        [](pdlp::CompiledLp& lp, pdlp::PdlpOptions&) { lp.rowUpper.pop_back(); },
        [](pdlp::CompiledLp&, pdlp::PdlpOptions& o) { o.terminationCheckFrequency = 0; },
        [](pdlp::CompiledLp&, pdlp::PdlpOptions& o) { o.primalTolerance = -1.0; },
    };
    for (auto& edit : cases) {
        pdlp::CompiledLp lp = base();
        pdlp::PdlpOptions o;
        edit(lp, o);
        const pdlp::PdlpResult a = pdlp::PdlpSolver().solve(lp, o);
        const pdlp::PdlpResult b = pdlpgpu::PdlpSolver().solve(lp, o);
        std::printf("%d|%s|%s|%d|%s|%s\n", static_cast<int>(a.status), pdlp::toString(a.status),
                    a.statusMessage.c_str(), static_cast<int>(b.status), pdlp::toString(b.status),
                    b.statusMessage.c_str());
    }
    return 0;
}
"""


def _reference_include():
    import __graft_entry__
    inc = os.path.join(__graft_entry__.REFERENCE_SOURCES, "include")
    return inc if os.path.isdir(os.path.join(inc, "pdlp")) else None


def test_facade_matches_reference_on_rejected_inputs(tmp_path):
    inc = _reference_include()
    if inc is None or not os.path.exists(os.path.join(REF_LIB, "libpdlp_ref.so")):
        pytest.skip("the reference's headers or the oracle library are not available here")
    if not os.path.exists(os.path.join(OUR_LIB, "libpdlpgpu.so")) or shutil.which("g++") is None:
        pytest.skip("libpdlpgpu.so or g++ missing")
    src = tmp_path / "facade.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "facade"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", inc, str(src),
           "-o", str(exe), "-L", REF_LIB, "-lpdlp_ref", "-L", OUR_LIB, "-lpdlpgpu",
           f"-Wl,-rpath,{REF_LIB}", f"-Wl,-rpath,{OUR_LIB}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 7
    for line in lines:
        a_status, a_name, a_msg, b_status, b_name, b_msg = line.split("|")
        assert a_status == b_status and a_name == b_name == "invalid_problem", line
        assert a_msg == b_msg and a_msg, line
