"""The C-ABI library loads and exports every entry point include/*.h declares (CPU only; no
device calls)."""
import ctypes
import re
from pathlib import Path

from pct_reconstruction_b200 import _abi

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(pct_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"pct_create", "pct_drop_full_tx_iteration", "pct_mlp_paths"} <= names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_abi.LIB_PATH))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_every_declared_symbol():
    bound = {n for n, _, _ in _abi.SIGNATURES}
    assert declared_functions() <= bound, declared_functions() - bound


def test_config_struct_layout_matches():
    lib = _abi.load_library()
    assert lib.pct_config_size() == ctypes.sizeof(_abi.pct_config)


def test_exact_fast_points_key():
    import pytest
    from pct_reconstruction_b200 import Config, PCTError
    assert Config().EXACT_FAST_POINTS == 1
    assert Config(EXACT_FAST_POINTS=0).EXACT_FAST_POINTS == 0
    with pytest.raises(PCTError):
        Config(EXACT_FAST_POINTS=2)
