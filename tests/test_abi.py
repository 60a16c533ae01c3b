"""The C-ABI library loads on a host without a GPU and exports every symbol
the public headers declare; host-only entry points work without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from optimisation_solver_b200 import native
from tests import cases

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_symbols():
    names = set()
    for f in os.listdir(INCLUDE):
        if f.endswith(".h"):
            text = open(os.path.join(INCLUDE, f)).read()
            names |= set(re.findall(r"\b(pdlpgpu_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    names = declared_symbols()
    assert names, "no declarations found"
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert declared_symbols() <= set(native.SIGNATURES)


def test_status_strings_match_reference():
    lib = native.lib()
    names = ["optimal", "infeasible", "unbounded", "iteration_limit", "time_limit",
             "numerical_failure", "invalid_problem"]
    for code, name in enumerate(names):
        assert lib.pdlpgpu_status_string(code).decode() == name
    assert lib.pdlpgpu_status_string(99).decode() == "unknown"


def test_default_options_match_reference(port_oracle):
    o = native.options_struct(None)
    ref = port_oracle.default_options()
    for name, _ in native.Options._fields_:
        assert getattr(o, name) == ref[name], name


def test_device_count_without_gpu_is_safe():
    assert native.lib().pdlpgpu_device_count() >= 0


def test_invalid_problem_needs_no_device():
    from optimisation_solver_b200.pdlp import PdlpSolver
    from optimisation_solver_b200.lp import PdlpStatus
    r = PdlpSolver().solve(cases.crossed_row_bounds(), cases.strict_options())
    assert r.status == PdlpStatus.INVALID_PROBLEM
    assert r.status_message == "Invalid row bounds"
    assert r.primal.size == 0 and np.isnan(r.primal_objective)


def test_mis_sized_vectors_are_rejected_not_read():
    """A CompiledLp whose vectors or CSR arrays do not match its dimensions
    gets the reference's message (compiled_lp.h:32-45), decided on the host;
    the library is never handed an array shorter than it would read."""
    import dataclasses

    from optimisation_solver_b200.lp import PdlpStatus, SparseMatrix
    from optimisation_solver_b200.pdlp import PdlpSolver
    base = cases.infeasible_rows()
    solver = PdlpSolver()
    expect = {
        "objective": "CompiledLp column vector dimensions do not match A",
        "var_upper": "CompiledLp column vector dimensions do not match A",
        "row_lower": "CompiledLp row vector dimensions do not match A",
        "row_upper": "CompiledLp row vector dimensions do not match A",
    }
    for field, message in expect.items():
        lp = dataclasses.replace(base, **{field: np.asarray(getattr(base, field))[:-1]})
        r = solver.solve(lp, cases.strict_options())
        assert r.status == PdlpStatus.INVALID_PROBLEM and r.status_message == message, field
    m = base.matrix
    short = SparseMatrix(m.rows, m.columns, m.row_start, m.col_index[:-1], m.values[:-1])
    r = solver.solve(dataclasses.replace(base, matrix=short), cases.strict_options())
    assert r.status == PdlpStatus.INVALID_PROBLEM
    assert r.status_message == "CompiledLp contains an invalid sparse matrix"


def test_session_refuses_short_inputs_before_any_device_work():
    """Per-instance inputs shorter than the instances x length the library
    would read are refused by the Python session before the C call."""
    import pytest

    from optimisation_solver_b200.session import _check_sizes
    n, m = 5, 3
    ok = [np.zeros((4, n)), np.zeros((4, m)), None, None, None, None, None, np.zeros(4)]
    _check_sizes(ok, 4, n, m)
    _check_sizes([np.zeros((6, n))] + [None] * 7, 4, n, m)   # extra rows are not read
    with pytest.raises(ValueError, match="row_lower"):
        _check_sizes([None, np.zeros((3, m))] + [None] * 6, 4, n, m)
    with pytest.raises(ValueError, match="warm_weight"):
        _check_sizes([None] * 7 + [np.zeros(3)], 4, n, m)


def test_session_refuses_mistyped_and_short_buffers():
    """Buffers the library uses in place (device inputs, every output) must be
    contiguous float64 storage of at least the size it reads or writes; host
    memory passed as a device buffer is refused too. All checked before any
    C call, so this runs without a GPU."""
    import pytest
    import torch

    from optimisation_solver_b200.session import _check_output, _check_sizes
    n, m = 5, 3
    _check_output(np.zeros((4, n)), "primal", 4 * n, False)
    with pytest.raises(ValueError, match="float64"):
        _check_output(np.zeros((4, n), np.float32), "primal", 4 * n, False)
    with pytest.raises(ValueError, match="at least 20"):
        _check_output(np.zeros((3, n)), "primal", 4 * n, False)
    with pytest.raises(ValueError, match="C-contiguous"):
        _check_output(np.zeros((n, 8))[:, :4].T, "primal", 4 * n, False)
    with pytest.raises(ValueError, match="float64"):
        _check_output(torch.zeros(4 * n, dtype=torch.float32), "primal", 4 * n, False)
    # host memory where the call expects device memory
    with pytest.raises(ValueError, match="device buffer"):
        _check_sizes([np.zeros((4, n))] + [None] * 7, 4, n, m, on_device=True)
    with pytest.raises(ValueError, match="CUDA tensor"):
        _check_sizes([torch.zeros(4 * n, dtype=torch.float64)] + [None] * 7, 4, n, m,
                     on_device=True)
    # host inputs are copied to float64, so their dtype does not matter
    _check_sizes([np.zeros((4, n), np.float32)] + [None] * 7, 4, n, m)


def test_noalloc_trial_rejects_null_pointers_before_any_launch():
    """pdlpgpu_trial_noalloc refuses NULL device pointers on the side that has
    lines (and a NULL reductions pointer) with -1 before it touches a device,
    so this runs on a host without a GPU."""
    lib = native.lib()
    one = (C.c_double * 4)()
    fake = C.cast(one, C.c_void_p)   # never dereferenced: the call fails first
    # reductions NULL
    rc = lib.pdlpgpu_trial_noalloc(2, 3, *([fake] * 18), 1.0, 1.0, fake, fake, fake, None, None)
    assert rc == -1 and "reductions is NULL" in native.last_error()
    # a column-side pointer NULL with columns present (the objective, argument 9)
    args = [fake] * 18
    args[6] = None
    rc = lib.pdlpgpu_trial_noalloc(2, 3, *args, 1.0, 1.0, fake, fake, fake, fake, None)
    assert rc == -1 and "column-side" in native.last_error()
    # a row-side pointer NULL with rows present (y)
    args = [fake] * 18
    args[16] = None
    rc = lib.pdlpgpu_trial_noalloc(2, 3, *args, 1.0, 1.0, fake, fake, fake, fake, None)
    assert rc == -1 and "row-side" in native.last_error()
    # x_out NULL with columns present
    rc = lib.pdlpgpu_trial_noalloc(2, 3, *([fake] * 18), 1.0, 1.0, None, fake, fake, fake, None)
    assert rc == -1 and "column-side" in native.last_error()


def test_public_c_headers_compile_as_c99(tmp_path):
    """Every include/*.h is a C header: a C99 translation unit including all
    of them compiles with warnings as errors, as an FFI binding's would."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    headers = sorted(f for f in os.listdir(INCLUDE) if f.endswith(".h"))
    src = tmp_path / "all_headers.c"
    src.write_text("".join(f'#include "{h}"\n' for h in headers) + "int main(void) { return 0; }\n")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", INCLUDE,
                        "-c", str(src), "-o", str(tmp_path / "all_headers.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_presolve_refuses_null_arrays_and_bad_counts():
    """pdlpgpu_presolve checks its arguments before reading them: NULL arrays
    with positive counts and negative counts return -1 with a message, and
    nothing is allocated."""
    lib = native.lib()
    lower = np.zeros(2)
    upper = np.ones(2)
    types = np.zeros(2, np.int8)
    start = np.array([0], np.int64)

    def call(**kw):
        f = dict(num_variables=2, num_constraints=0, var_lower=native.ptr(lower),
                 var_upper=native.ptr(upper), var_type=native.ptr(types, C.c_int8),
                 row_start=native.ptr(start, C.c_int64))
        f.update(kw)
        m = native.PresolveModel(**f)
        out = C.POINTER(native.PresolveResult)()
        rc = lib.pdlpgpu_presolve(C.byref(m), C.byref(out))
        if rc == 0:
            lib.pdlpgpu_presolve_free(out)
        return rc, native.last_error()

    assert call()[0] == 0
    assert call(var_lower=None) == (-1, "presolve: NULL variable array")
    assert call(row_start=None) == (-1, "presolve: NULL row_start")
    assert call(num_constraints=1)[0] == -1            # row bounds NULL
    assert call(num_variables=-1) == (-1, "presolve: negative count")
    assert call(num_objective_terms=3) == (-1, "presolve: NULL objective array")
    assert call(num_quadratic_terms=1) == (-1, "presolve: NULL quadratic array")
    assert lib.pdlpgpu_presolve(None, None) == -1
