"""The C-ABI library loads and exports every entry point declared in include/dgb.h (no GPU)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    txt = (ROOT / "include" / "dgb.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dgb_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "dgb_residual" in names and "dgb_advance" in names and len(names) >= 25


def test_library_exports_every_declared_symbol():
    from dg_b200 import _ffi
    lib = _ffi.lib()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_ffi.EXPORTS) == declared()
    assert lib.dgb_abi_version() == 1


def test_device_calls_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import dg_b200 as dgb
    p = dgb.Problem.structured(2, 2, 4, 4, flux="rusanov", limiter="m2l")
    with pytest.raises(dgb.DGBError) as e:
        dgb.DGSolver(p)
    assert e.value.code == 9  # DGB_ERR_NO_DEVICE


def test_error_codes_for_bad_input(tmp_path):
    import dg_b200 as dgb
    with pytest.raises(dgb.DGBError) as e:
        dgb.Problem.from_deck(tmp_path / "missing.inp")
    assert e.value.code == 2  # DGB_ERR_IO
    (tmp_path / "deck.inp").write_text("#Code options\n#order\n2\n")
    with pytest.raises(dgb.DGBError) as e:
        dgb.Problem.from_deck(tmp_path / "deck.inp")
    assert e.value.code in (2, 4)
