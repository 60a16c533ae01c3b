"""The fast MPS reader and writer (include/pdlpgpu_mps.h) against the
reference reader, mps::MpsReader (src/mps/mps_reader.cpp), compiled from its
sources into oracle/_ref/libpipeline_ref.so.

Every MPS file the reference ships for its reader, its known-answer LPs, its
Netlib file and its CLI tests is read by both: files the reference refuses
must be refused with the same message; the others must give the same model --
name, variable and row names, types, bounds, objective constant and sense,
objective terms, per-row terms (as sets: the reference's order is its hash
map's), quadratic terms, warnings. Also: the adapter's CompiledLp of every
LP, written files read back bit for bit, features and refusals on files
written here, and the time of both readers on a 600,000-nonzero file.
"""
import os
import time

import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200 import mps
from oracle.pipeline import Pipeline, available

ROOT_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(not available("ref"),
                                reason="reference pipeline not built (make -C oracle pipeline)")


def _reference_root():
    import __graft_entry__
    return __graft_entry__.REFERENCE_ROOT


def reference_files():
    root = _reference_root()
    dirs = [os.path.join(root, "tests", "mps", "test_cases"),
            os.path.join(root, "benchmarks", "instances", "known"),
            os.path.join(root, "benchmarks", "instances", "netlib"),
            os.path.join(root, "tests", "cli")]
    out = []
    for d in dirs:
        if os.path.isdir(d):
            out += sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(".mps"))
    return out


@pytest.fixture(scope="module")
def ref():
    return Pipeline("ref")


def _rows_as_sets(start, index, value):
    out = []
    for i in range(len(start) - 1):
        pairs = sorted(zip(index[start[i]:start[i + 1]].tolist(), value[start[i]:start[i + 1]].tolist()))
        out.append(pairs)
    return out


def assert_same_model(ours: mps.MpsModel, theirs):
    a = theirs.export(allow_quadratic=True)
    names = theirs.names()
    assert ours.name == names["name"]
    assert ours.variable_names == names["variables"]
    assert ours.row_names == names["rows"]
    assert ours.warnings == names["warnings"]
    assert ours.sense == a["sense"] and ours.offset == a["offset"]
    for f in ("var_type", "var_lower", "var_upper", "row_lower", "row_upper"):
        assert np.array_equal(getattr(ours, f), a[f]), f
    assert sorted(zip(ours.objective_index.tolist(), ours.objective_value.tolist())) == \
        sorted(zip(a["objective_index"].tolist(), a["objective_value"].tolist()))
    assert _rows_as_sets(ours.row_start, ours.row_index, ours.row_value) == \
        _rows_as_sets(a["row_start"], a["row_index"], a["row_value"])
    qi, qj, qv = theirs.quadratic()
    assert list(zip(ours.quadratic_i.tolist(), ours.quadratic_j.tolist(), ours.quadratic_value.tolist())) \
        == list(zip(qi.tolist(), qj.tolist(), qv.tolist()))


def _read_both(ref, path):
    try:
        theirs = ref.read_mps(path)
        their_error = None
    except ValueError as e:
        theirs, their_error = None, str(e)
    try:
        ours = mps.read_mps(path)
        our_error = None
    except ValueError as e:
        ours, our_error = None, str(e)
    return ours, our_error, theirs, their_error


def test_reference_files_read_the_same(ref):
    files = reference_files()
    if not files:
        pytest.skip("the reference's MPS files are not available here")
    refused = 0
    for path in files:
        ours, our_error, theirs, their_error = _read_both(ref, path)
        assert our_error == their_error, (path, our_error, their_error)
        if their_error is not None:
            refused += 1
            continue
        assert_same_model(ours, theirs)
    assert refused >= 2   # the reference ships files it must refuse


def test_compiled_lp_matches_the_adapter(ref):
    files = reference_files()
    if not files:
        pytest.skip("the reference's MPS files are not available here")
    compiled = 0
    for path in files:
        ours, our_error, theirs, their_error = _read_both(ref, path)
        if their_error is not None:
            continue
        try:
            want = theirs.compile()
            want_error = None
        except ValueError as e:
            want, want_error = None, str(e)
        try:
            got, negated = ours.compiled_lp()
            got_error = None
        except ValueError as e:
            got, got_error = None, str(e)
        assert got_error == want_error, (path, got_error, want_error)
        if want is None:
            continue
        compiled += 1
        assert negated == (ours.sense == 1)
        for f in ("row_start", "col_index", "values", "objective", "row_lower", "row_upper",
                  "var_lower", "var_upper"):
            assert np.array_equal(getattr(got, f), getattr(want, f)), (path, f)
        assert got.objective_offset == want.objective_offset
    assert compiled >= 5


# A file exercising the reader's conventions, written for this test: OBJSENSE
# on the following line, an objective constant, integer markers, a repeated
# (row, column) pair, an explicit zero, a coefficient on a free row and on an
# unknown row, RHS records with and without a set name and a second RHS
# vector, RANGES on L, G and E rows of both signs, every bound type, the
# negative-UP rule, a column first seen in BOUNDS, comments and blank lines.
FEATURES = """* conventions test
NAME          features
OBJSENSE
    MAX
ROWS
 N  profit
 L  cap1
 G  need1
 E  bal1
 E  bal2
 N  spare
 L  cap2
COLUMNS
    x1        profit    3.5   cap1   2
    x1        need1     1     spare  9
    x2        profit    -1.25e+0
    x2        cap1      1     cap1   0.5
    x2        bal1      4     ghost  1
    MARKER    'MARKER'  'INTORG'
    y1        profit    2     bal2   1
    y2        bal2      0     cap2   1.0e-3
    MARKER    'MARKER'  'INTEND'
    x3        need1     .5    bal1   -2
    x3        bal2      7
RHS
    RHS       profit    -12.5
    RHS       cap1      10    need1  2
    ALT       cap1      99
    bal1      3   bal2  -1
    cap2      4.25
RANGES
    RNG       cap1      4     need1  -3
    RNG       bal1      2     bal2   -1.5
BOUNDS
 UP BND       x1        8
 LO BND       x2        -2
 UP BND       x3        -4
 MI BND       y1
 UP BND       y1        5
 BV BND       y2
 FR BND       z9
 LI BND       x2        -2
 UI BND       x1        6
 PL BND       x2
 FX BND       w1        1.5
ENDATA
"""


def test_features_read_the_same(tmp_path, ref):
    for name, text in (("lf", FEATURES), ("crlf", FEATURES.replace("\n", "\r\n"))):
        path = tmp_path / f"features_{name}.mps"
        path.write_bytes(text.encode())
        ours, our_error, theirs, their_error = _read_both(ref, str(path))
        assert our_error is None and their_error is None, (our_error, their_error)
        assert_same_model(ours, theirs)
        assert ours.warnings, "the file triggers warnings"


REFUSED = {
    "unknown_section": "NAME a\nROWS\n N obj\nFOO\nENDATA\n",
    "sos": "NAME a\nROWS\n N obj\nSOS\nENDATA\n",
    "row_sense": "NAME a\nROWS\n N obj\n Q r1\nENDATA\n",
    "duplicate_row": "NAME a\nROWS\n N obj\n L r1\n G r1\nENDATA\n",
    "missing_row_name": "NAME a\nROWS\n L\nENDATA\n",
    "no_coefficient": "NAME a\nROWS\n N obj\n L r1\nCOLUMNS\n x obj 1 r1\nENDATA\n",
    "bad_coefficient": "NAME a\nROWS\n N obj\n L r1\nCOLUMNS\n x obj one\nENDATA\n",
    "rhs_value": "NAME a\nROWS\n N obj\n L r1\nRHS\n rhs r1 1.5.2\nENDATA\n",
    "bound_type": "NAME a\nROWS\n N obj\nBOUNDS\n XX bnd x 1\nENDATA\n",
    "bound_value": "NAME a\nROWS\n N obj\nBOUNDS\n UP bnd x\nENDATA\n",
    "bound_column": "NAME a\nROWS\n N obj\nBOUNDS\n UP bnd\nENDATA\n",
    "fractional_li": "NAME a\nROWS\n N obj\nBOUNDS\n LI bnd x 1.5\nENDATA\n",
    "objsense": "NAME a\nOBJSENSE\n SIDEWAYS\nENDATA\n",
    "overflow": "NAME a\nROWS\n N obj\n L r1\nRHS\n rhs r1 1e999\nENDATA\n",
}


@pytest.mark.parametrize("case", sorted(REFUSED))
def test_refusals_match(tmp_path, ref, case):
    path = tmp_path / f"{case}.mps"
    path.write_text(REFUSED[case])
    ours, our_error, theirs, their_error = _read_both(ref, str(path))
    assert their_error is not None and our_error == their_error, (our_error, their_error)


def test_missing_file(ref):
    ours, our_error, theirs, their_error = _read_both(ref, "/nonexistent/x.mps")
    assert our_error == their_error and "Unable to open file" in our_error


def test_written_lp_reads_back_exactly(tmp_path, ref):
    """The planted 1000 x 2000 LP and a stress-family LP (free variables,
    ranged rows, rescaled magnitudes) written by pdlpgpu_mps_write: both
    readers give back the LP bit for bit."""
    for name, lp in (("planted", g.reference_lp(0).lp), ("stress", g.stress_lp(1, m=600, n=1200).lp)):
        path = str(tmp_path / f"{name}.mps")
        mps.write_mps(lp, path, name)
        ours, _ = mps.read_mps(path).compiled_lp()
        theirs = ref.read_mps(path).compile()
        for back in (ours, theirs):
            for f in ("row_start", "col_index", "values", "objective", "row_lower", "row_upper",
                      "var_lower", "var_upper"):
                assert np.array_equal(getattr(back, f), getattr(lp, f)), (name, f)
            assert back.objective_offset == lp.objective_offset


def test_reader_is_faster_than_the_reference(tmp_path, ref):
    """About 600,000 nonzeros (the large-LP family at 40,000 x 80,000). Both
    readers' models must agree, and this one must take less time."""
    lp = g.large_lp(2, m=40_000, n=80_000).lp
    path = str(tmp_path / "large.mps")
    mps.write_mps(lp, path, "large")
    t0 = time.perf_counter()
    ours = mps.read_mps(path)
    t1 = time.perf_counter()
    theirs = ref.read_mps(path)
    t2 = time.perf_counter()
    assert_same_model(ours, theirs)
    print(f"MPS read, {lp.nnz} nonzeros, {os.path.getsize(path) / 1e6:.1f} MB: "
          f"this reader {t1 - t0:.3f} s, reference {t2 - t1:.3f} s ({(t2 - t1) / (t1 - t0):.1f}x)")
    assert t1 - t0 < t2 - t1


FACADE_PROGRAM = r"""
#include "mps/mps_reader.h"
#include "pdlpgpu_mps.hpp"

#include <algorithm>
#include <cstdio>
#include <string>
#include <tuple>
#include <vector>

using Terms = std::vector<std::pair<int, double>>;

static Terms sorted(const std::vector<model::LinearTerm>& t) {
    Terms out;
    for (const auto& x : t) out.emplace_back(x.variableIndex, x.value);
    std::sort(out.begin(), out.end());
    return out;
}

static bool same(const model::Model& a, const model::Model& b) {
    if (a.name != b.name || a.objective.sense != b.objective.sense ||
        a.objective.offset != b.objective.offset || a.variables.size() != b.variables.size() ||
        a.constraints.size() != b.constraints.size() ||
        sorted(a.objective.linearTerms) != sorted(b.objective.linearTerms) ||
        a.objective.quadraticTerms.size() != b.objective.quadraticTerms.size())
        return false;
    for (size_t k = 0; k < a.objective.quadraticTerms.size(); ++k) {
        const auto& p = a.objective.quadraticTerms[k];
        const auto& q = b.objective.quadraticTerms[k];
        if (p.variableIndex1 != q.variableIndex1 || p.variableIndex2 != q.variableIndex2 || p.value != q.value)
            return false;
    }
    for (size_t j = 0; j < a.variables.size(); ++j) {
        const auto& p = a.variables[j];
        const auto& q = b.variables[j];
        if (p.name != q.name || p.type != q.type || p.lowerBound != q.lowerBound || p.upperBound != q.upperBound)
            return false;
    }
    for (size_t i = 0; i < a.constraints.size(); ++i) {
        const auto& p = a.constraints[i];
        const auto& q = b.constraints[i];
        if (p.name != q.name || p.lowerBound != q.lowerBound || p.upperBound != q.upperBound ||
            sorted(p.linearTerms) != sorted(q.linearTerms))
            return false;
    }
    return true;
}

int main(int argc, char** argv) {
    for (int f = 1; f < argc; ++f) {
        mps::MpsReader ref;
        pdlpgpu::MpsReader ours;
        model::Model a, b;
        std::string ea, eb;
        try { a = ref.read(argv[f]); } catch (const std::exception& e) { ea = e.what(); }
        try { b = ours.read(argv[f]); } catch (const std::exception& e) { eb = e.what(); }
        const bool ok = ea == eb && (!ea.empty() || (same(a, b) && ref.warnings() == ours.warnings()));
        std::printf("%s %s\n", ok ? "SAME" : "DIFFERENT", argv[f]);
    }
    return 0;
}
"""


def test_cpp_facade_reads_like_the_reference(tmp_path):
    """include/pdlpgpu_mps.hpp against mps::MpsReader in one C++ program built
    from the reference's headers and reader sources: the same model::Model,
    warnings and errors for every MPS file the reference ships."""
    import shutil
    import subprocess
    root = _reference_root()
    files = reference_files()
    if not files or shutil.which("g++") is None:
        pytest.skip("the reference's sources or g++ are not available here")
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(repo, "optimisation_solver_b200", "_lib")
    src = tmp_path / "mps_facade.cpp"
    src.write_text(FACADE_PROGRAM)
    exe = tmp_path / "mps_facade"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(repo, "include"),
           "-I", os.path.join(root, "include"), str(src),
           os.path.join(root, "src", "mps", "mps_reader.cpp"), os.path.join(root, "src", "model", "model.cpp"),
           "-o", str(exe), "-L", lib_dir, "-lpdlpgpu", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), *files], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == len(files)
    assert all(line.startswith("SAME ") for line in lines), [l for l in lines if not l.startswith("SAME")]


def _big_columns_text(m=2000, n=120_000, error_at=None):
    """An MPS text whose COLUMNS section is larger than the size from which
    the reader parses it on several threads (8 MiB): integer markers toggled
    every 5,000 columns, a term on an undeclared row every 1,000 columns (a
    warning), a repeated (row, column) pair every 777 columns, a record
    without coefficients every 4,321 columns, each column's terms on two lines
    (so chunk boundaries fall inside columns). `error_at`: the column whose
    second line loses its coefficient."""
    rng = np.random.default_rng(11)
    rows = rng.integers(0, m, size=(n, 3))
    vals = np.round(rng.standard_normal((n, 3)), 6)
    out = ["NAME big", "ROWS", " N obj"] + [f" L r{i}" for i in range(m)] + ["COLUMNS"]
    marker = False
    for j in range(n):
        if j % 5000 == 0 and j:
            marker = not marker
            out.append(f"    M{j}  'MARKER'  '{'INTORG' if marker else 'INTEND'}'")
        a, b, c = rows[j]
        out.append(f"    x{j}  obj  {vals[j, 0]}  r{a}  {vals[j, 1]}")
        second = f"    x{j}  r{b}  {vals[j, 2]}  r{c}  {vals[j, 0]}"
        if j == error_at:
            second = f"    x{j}  r{b}  {vals[j, 2]}  r{c}"
        out.append(second)
        if j % 1000 == 7:
            out.append(f"    x{j}  ghost  1.5")
        if j % 777 == 3:
            out.append(f"    x{j}  r{a}  0.25")
        if j % 4321 == 5:
            out.append(f"    x{j}")
    out += ["RHS", "    rhs  r0  1", "BOUNDS", " UP bnd x0 4", "ENDATA"]
    return "\n".join(out) + "\n"


def test_parallel_columns_section_reads_the_same(tmp_path, ref):
    text = _big_columns_text()
    assert len(text) > 9 << 20
    path = tmp_path / "big.mps"
    path.write_text(text)
    ours, our_error, theirs, their_error = _read_both(ref, str(path))
    assert our_error is None and their_error is None, (our_error, their_error)
    assert_same_model(ours, theirs)
    assert any("ghost" in w for w in ours.warnings)
    assert (ours.var_type == 1).any() and (ours.var_type == 0).any()
    # An error deep in the section: the same message and line number.
    bad = tmp_path / "bad.mps"
    bad.write_text(_big_columns_text(error_at=97_531))
    ours, our_error, theirs, their_error = _read_both(ref, str(bad))
    assert their_error is not None and our_error == their_error, (our_error, their_error)


def test_reference_mps_reader_tests_pass_with_fast_reader():
    """The reference's own MPS parser tests (tests/mps/mps_reader_tests.cpp),
    built with its reader and with the fast reader linked in place of
    src/mps/mps_reader.cpp (oracle/mps_override.cpp): both pass, with the same
    output. They read their fixtures relative to the reference root."""
    import subprocess
    root = _reference_root()
    progs = os.path.join(ROOT_DIR, "oracle", "_ref", "presolve_tests")
    ref_prog = os.path.join(progs, "test_mps_reader_ref")
    fast_prog = os.path.join(progs, "test_mps_reader_fast")
    if not (os.path.isdir(os.path.join(root, "tests", "mps")) and os.path.exists(fast_prog)):
        pytest.skip("reference tree or test programs absent (make -C oracle presolve)")
    ref = subprocess.run([ref_prog], cwd=root, capture_output=True, text=True, timeout=300)
    fast = subprocess.run([fast_prog], cwd=root, capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stdout + ref.stderr
    assert fast.returncode == 0, fast.stdout + fast.stderr
    assert fast.stdout == ref.stdout
