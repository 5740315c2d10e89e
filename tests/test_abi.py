"""CPU tests of the boundary: libcad_td.so builds for sm_100a, loads without a
GPU, exports every symbol include/cad_td.h declares, and the host mirror keeps
the reference's argument checks (no compute call is made here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cad_td.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|double|void\*|const char\*)\s+(cad_\w+)\(", text, re.M)))


def test_header_matches_binding_list():
    from cutanddisplacejulia_b200 import _lib
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(cad):
    from cutanddisplacejulia_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_library_version_string(cad):
    from cutanddisplacejulia_b200 import _lib
    assert b"sm_100a" in _lib.load().cad_version()


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    from cutanddisplacejulia_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(_lib.CadError, match="not built"):
        _lib.load()


def test_dims_error_before_any_device_call(cad):
    P = np.zeros((2, 3))
    with pytest.raises(cad.CadError, match="Element size inputs must be the same dimensions"):
        cad.TD([0.0], [0.0], [-1.0], P, P, P, [1.0], [1.0, 1.0], [1.0, 1.0], 0.25, 1.0, 1, 1, 0)


def test_header_cites_reference_interfaces():
    text = open(os.path.join(ROOT, "include", "cad_td.h")).read()
    for cite in ("src/TD.jl:146-214", "src/TD_sum.jl:1-41", "src/CalculateInfluenceMatrices3D.jl",
                 "src/SlipCalculator3D.jl"):
        assert cite in text
