"""The C ABI: libwema_cuda loads (no GPU needed), exports every function the
headers in include/ declare, and the public structs have the reference's
layout byte for byte (fixture from the reference's own headers)."""
import ctypes
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(INC):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INC, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"static inline[^{]*\{[^}]*\}", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            if not m.group(0).lstrip().startswith(("typedef", "#")):
                names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    from wema_b200 import _build
    path = _build.cuda_lib_path()
    if not os.path.exists(path):
        _build.build_cuda()
    return ctypes.CDLL(path)


def test_exports_every_declared_function(lib):
    names = declared_functions()
    assert {"dwt_forward", "iir_temporal_process", "temporal_filter_apply", "coeff_amplify",
            "wema_process_frame", "wema_batch_process", "wema_cuda_process_u8",
            "wema_cuda_threshold_flat_noalloc"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_struct_layouts_match_reference(tmp_path):
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", INC, os.path.join(ROOT, "tests", "c", "abi_layout.c"),
                    "-o", str(exe)], check=True)
    ours = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "abi_layout.json")))
    assert ours == ref


def test_last_error_without_gpu_work(lib):
    lib.wema_cuda_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.wema_cuda_last_error(), bytes)
