"""CPU checks of the drop-in boundary: the CUDA library builds for sm_100a,
loads, and exports exactly the entry points include/flosic_sic.h declares
(no compute calls: this environment has no GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "publicrelease_2020_b200", "libflosic_sic_b200.so")
HDR = os.path.join(ROOT, "include", "flosic_sic.h")


def declared_symbols():
    text = open(HDR).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(flosic_sic_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "publicrelease_2020_b200")], check=True)
    return ctypes.CDLL(LIB)


def test_header_declares_reference_entry_points():
    syms = declared_symbols()
    for name in ["apotnl_sic", "coupot_sic", "getvlxc", "siclagm", "frmorb2_force", "frmorb2_fmat", "frmiorb",
                 "gorbdrv"]:
        assert f"flosic_sic_{name}" in syms


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_python_binding_matches_header():
    from publicrelease_2020_b200 import sic
    assert sorted(sic.EXPORTS) == declared_symbols()


def test_library_built_for_sm100a(lib):
    out = subprocess.run(["cuobjdump", "--list-elf", LIB], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_missing_library_fails_loudly(tmp_path):
    from publicrelease_2020_b200 import sic
    with pytest.raises(FileNotFoundError):
        sic.load_library.__wrapped__(str(tmp_path / "nope.so")) if hasattr(sic.load_library, "__wrapped__") else \
            _load_fresh(sic, str(tmp_path / "nope.so"))


def _load_fresh(sic, path):
    saved = sic._lib
    try:
        sic._lib = None
        sic.load_library(path)
    finally:
        sic._lib = saved


def test_no_oracle_in_product_sources():
    pkg = os.path.join(ROOT, "publicrelease_2020_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.lower().replace("oracle/", ""), f
