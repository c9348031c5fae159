"""The C ABI: libblsgpu.so loads and exports every function include/blsgpu.h declares (no device calls)."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bls_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(bls):
    lib = C.CDLL(str(ROOT / "blocklinearsystems.jl_b200" / "libblsgpu.so"))
    names = declared(ROOT / "include" / "blsgpu.h")
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_string(bls):
    L = bls._lib.gpu()
    assert L.bls_version() >= 1
    assert isinstance(L.bls_last_error(), bytes)


def test_plan_rejects_bad_sizes_without_a_device(bls):
    """Argument checks of the host side need no GPU: a description error surfaces as ArgumentError."""
    import pytest
    with pytest.raises(bls.ArgumentError):
        bls.SchurStructure([6, 3], [[0, 1, 1]], eliminated=[False, True])
