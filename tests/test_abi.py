"""C-ABI checks that need no GPU: the library loads, exports every entry point declared
in include/dvr3d_b200.h, and the ctypes mirrors match the C struct layouts."""
from __future__ import annotations

import ctypes as C
import subprocess
import tempfile
from pathlib import Path

import pytest

from dvr3d_b200 import _abi

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_every_header_symbol():
    lib = _abi.load_library()
    names = _abi.header_entry_points()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def _c_layout(struct: str, fields: list[str]) -> dict:
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/dvr3d_b200.h"',
           'int main(void) {', f'  printf("size %zu\\n", sizeof({struct}));']
    for f in fields:
        src.append(f'  printf("{f} %zu\\n", offsetof({struct}, {f}));')
    src.append("  return 0; }")
    with tempfile.TemporaryDirectory() as td:
        c = Path(td) / "l.c"
        c.write_text("\n".join(src))
        exe = Path(td) / "l"
        subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.parametrize("py,cname", [(_abi.Deck, "dvr3d_deck"), (_abi.Options, "dvr3d_options"),
                                      (_abi.Result, "dvr3d_result")])
def test_struct_layouts_match_header(py, cname):
    fields = [f[0] for f in py._fields_]
    lay = _c_layout(cname, fields)
    assert lay["size"] == C.sizeof(py)
    for f in fields:
        assert lay[f] == getattr(py, f).offset, f


def test_strerror_and_parse_errors():
    lib = _abi.load_library()
    assert lib.dvr3d_b200_strerror(0) == b"ok"
    assert b"emax2" in lib.dvr3d_b200_strerror(-3)
    d = _abi.Deck()
    assert lib.dvr3d_b200_parse_deck(b"no namelist here\n", C.byref(d)) == _abi.DVR3D_ERR_DECK
    assert lib.dvr3d_b200_parse_deck(b" &PRT ZFOO=.TRUE. /\n    3\n", C.byref(d)) == _abi.DVR3D_ERR_DECK


def test_init_without_device_reports_no_device():
    """On a host without a GPU the library must refuse (no CPU fallback)."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    lib = _abi.load_library()
    h = C.c_void_p()
    assert lib.dvr3d_b200_init(0, C.byref(h)) == _abi.DVR3D_ERR_NO_DEVICE
