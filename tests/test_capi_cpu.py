"""C-ABI checks that need no GPU: the library loads, exports every entry
point declared in include/yrt_b200.h, and its host-only geometry calls match
the oracle bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "yrt_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(yrtb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "yrtb_forward" in syms and "yrtb_em_step" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from pyyrtpet_b200 import _lib
    L = _lib.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s
    # every declared symbol also has a ctypes signature in the binding
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_regular_lut_matches_oracle_bitexact():
    import pyyrtpet_b200 as yrt
    for args in [(64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1),
                 (256, 3.2, 3.2, 20, 410, 672, 80, 1, 79, 2, 1),
                 (25, 5, 3, 10, 300, 256, 5, 1, 4, 2, 8),
                 (60, 5, 5, 10, 200, 48, 12, 2, 11, 1, 4)]:
        sc = yrt.Scanner("t", *args)
        ref = po.scanner_lut(po.Scanner(*args))
        got = sc.createLUT()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_histogram_dims_match_oracle():
    import pyyrtpet_b200 as yrt
    for args in [(64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1),
                 (256, 3.2, 3.2, 20, 410, 672, 80, 1, 79, 2, 1),
                 (60, 5, 5, 10, 200, 48, 12, 2, 11, 1, 4)]:
        h = yrt.Histogram3D(yrt.Scanner("t", *args))
        assert (h.numZBin, h.numPhi, h.numR) == po.histo3d_dims(po.Scanner(*args))


def test_invalid_scanner_rejected_like_reference():
    import pyyrtpet_b200 as yrt
    with pytest.raises(RuntimeError, match="Maximum Ring difference"):
        yrt.Scanner("bad", 64, 4, 4, 10, 300, 256, 16, 1, 79, 2, 1)
    from pyyrtpet_b200 import _lib
    s = _lib.yrtb_scanner(64, 4, 4, 10, 300, 256, 16, 1, 16, 2, 1)
    out = np.zeros((4096, 6), np.float32)
    rc = _lib.lib().yrtb_scanner_regular_lut(ctypes.byref(s), out.ctypes.data)
    assert rc == _lib.YRTB_ERR_ARGUMENT
    assert b"Maximum Ring difference" in _lib.lib().yrtb_last_error()


def test_no_cpu_fallback_when_library_missing(monkeypatch, tmp_path):
    from pyyrtpet_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="libyrtb.so not found"):
        _lib.lib()


def test_ctypes_structs_match_the_c_header_layout(tmp_path):
    """Every struct the Python binding passes through the C ABI has the size
    and field offsets the C compiler gives it from include/yrt_b200.h."""
    import shutil
    import subprocess
    from pyyrtpet_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    structs = {
        "yrtb_scanner": _lib.yrtb_scanner, "yrtb_image_params": _lib.yrtb_image_params,
        "yrtb_projector_params": _lib.yrtb_projector_params,
        "yrtb_events": _lib.yrtb_events, "yrtb_range": _lib.yrtb_range,
        "yrtb_launch_config": _lib.yrtb_launch_config,
        "yrtb_tune_report": _lib.yrtb_tune_report,
        "yrtb_osem_params": _lib.yrtb_osem_params,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "yrt_b200.h"',
             "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        name, what, value = line.split()
        cls = structs[name]
        if what == "size":
            assert ctypes.sizeof(cls) == int(value), name
        else:
            assert getattr(cls, what).offset == int(value), (name, what)
