"""The C-ABI library loads and exports every entry point include/*.h declares (CPU only: no
compute call is made)."""
import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
LIB = REPO / "3fold-field-engine_b200" / "libfield_b200.so"


def declared_functions():
    names = []
    for header in sorted((REPO / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", text, flags=re.M):
            names.append(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert "edt_squared_large" in names and "fb_field_build_device" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    if not LIB.exists():
        pytest.skip("library not built")
    lib = ctypes.CDLL(str(LIB))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_record_layouts_match_python():
    import field_b200.expr as X
    import field_b200.build as B
    assert X.PRIM.itemsize == 216
    assert X.INSN.itemsize == 16
    assert ctypes.sizeof(B.FbGeom) == 64
    import field_b200.batch as BT
    assert ctypes.sizeof(BT._Item) == 96  # fb_batch_item


def test_product_fails_loudly_without_gpu(monkeypatch):
    import torch
    import field_b200._lib as L
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.lib()
