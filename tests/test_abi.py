"""The C ABI library: it loads without a GPU and exports every symbol that
include/sirocco_solve.h declares (no compute calls here)."""
import re
import subprocess
from pathlib import Path

import pytest

from oracle import oracle
from python_b200 import build, engine

HEADER = Path(__file__).resolve().parent.parent / "include" / "sirocco_solve.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    text = re.sub(r"\btypedef\b[^;]*;", "", text)   # callback types are not functions
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)) - {"if", "sizeof", "defined"})


@pytest.fixture(scope="module")
def lib():
    build.build_engine()
    return engine.load()


def test_header_declares_reference_interface():
    names = declared_functions()
    for ref_name in ("solve_matrix", "invert_matrix", "get_matrix_error_string", "cusolver_create",
                     "cusolver_destroy", "cusolver_get_error_string", "gpu_solve_matrix", "gpu_invert_matrix"):
        assert ref_name in names
    assert set(names) == set(engine.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(engine.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    for f in declared_functions():
        assert hasattr(lib, f)


def test_error_strings_without_gpu(lib):
    for code in (2, 3, 4, 0, 99):
        assert engine.error_string(code) == oracle.error_string(code)
    assert lib.cusolver_get_error_string(0).decode() == "The operation completed successfully"


def test_destroy_without_create_is_noop(lib):
    assert lib.cusolver_destroy() == 0
