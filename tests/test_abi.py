"""The C-ABI library loads, exports every entry point include/bugdef.h declares, and the
ctypes structure mirrors have the layout a C compiler gives the header (no GPU needed)."""
import ctypes
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "bugdef.h"


def declared():
    return re.findall(r"BD_API\s+\w+\s+(bd_\w+)\s*\(", HEADER.read_text())


@pytest.fixture(scope="module")
def lib():
    from bug_defense_b200 import build, _lib
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    from bug_defense_b200 import _lib
    names = declared()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (bd_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    extra = sorted(exported - set(names))
    assert not extra, f"exported but not declared: {extra}"
    assert set(_lib.declared_symbols()) == set(names)
    for n in names:
        assert getattr(lib, n) is not None


def test_version_and_errors_without_gpu(lib):
    from bug_defense_b200 import _lib
    assert lib.bd_abi_version() == 1
    # argument validation happens before any device work
    rc = lib.bd_thermal_advance(None, None, None, 1, None, None, None, None)
    assert rc == _lib.BD_ERR_INVALID_ARG
    assert "params is NULL" in _lib.last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)
    n = ctypes.c_int(-1)
    assert lib.bd_device_count(ctypes.byref(n)) == 0
    assert n.value >= 0


STRUCTS = ["BdMcParams", "BdThermalParams", "BdAblationParams", "BdPlumeParams", "BdGridRef", "BdPhaseDesc",
           "BdEngineDesc", "BdEpochDiag", "BdConvCall", "BdRecordSpec", "BdRecordHead"]
PY = {"BdMcParams": "McParams", "BdThermalParams": "ThermalParams", "BdAblationParams": "AblationParams",
      "BdPlumeParams": "PlumeParams", "BdGridRef": "GridRef", "BdPhaseDesc": "PhaseDesc",
      "BdEngineDesc": "EngineDesc", "BdEpochDiag": "EpochDiag", "BdConvCall": "ConvCall",
      "BdRecordSpec": "RecordSpec", "BdRecordHead": "RecordHead"}


def test_struct_layouts_match_header():
    from bug_defense_b200 import _lib
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for s in STRUCTS:
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for fname, _ in getattr(_lib, PY[s])._fields_:
            lines.append(f'printf("{s}.{fname} %zu\\n", offsetof({s}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "layout.c"
        src.write_text("\n".join(lines))
        exe = Path(d) / "layout"
        subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for s in STRUCTS:
        cls = getattr(_lib, PY[s])
        assert int(got[s]) == ctypes.sizeof(cls), s
        for fname, _ in cls._fields_:
            assert int(got[f"{s}.{fname}"]) == getattr(cls, fname).offset, f"{s}.{fname}"
