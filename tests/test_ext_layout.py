"""The extension structs of include/wema_cuda.h (config, session status,
serve stats) have the same layout in C and in the Python binding, and a C11
caller of the extension API (tests/c/serve_client.c) compiles with -Wall
-Werror and links against libwema_cuda; on a GPU it runs and checks its frames."""
import ctypes as C
import subprocess

import pytest

from wema_b200 import cuda as wc

INCLUDE = __import__("os").path.join(__import__("os").path.dirname(__file__), "..", "include")

STRUCTS = {
    "wema_cuda_config": wc.Config,
    "wema_cuda_session_status": wc.SessionStatus,
    "wema_cuda_serve_stats": wc.ServeStats,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("layout")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wema_cuda.h"', "int main(void) {"]
    for name, py in STRUCTS.items():
        lines.append(f'printf("{name} size %zu\\n", sizeof({name}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines))
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    res = {}
    for line in out.splitlines():
        name, field, val = line.split()
        res[(name, field)] = int(val)
    return res


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_layout_matches(c_layout, name):
    py = STRUCTS[name]
    assert c_layout[(name, "size")] == C.sizeof(py)
    for f, _ in py._fields_:
        assert c_layout[(name, f)] == getattr(py, f).offset, f


def _client(tmp_path):
    from wema_b200 import _build
    lib = _build.build_cuda()
    exe = tmp_path / "serve_client"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", INCLUDE,
                    __import__("os").path.join(__import__("os").path.dirname(__file__), "c", "serve_client.c"),
                    "-o", str(exe), "-L", __import__("os").path.dirname(lib), "-lwema_cuda",
                    "-Wl,-rpath," + __import__("os").path.dirname(lib)], check=True)
    return exe


def test_c_client_builds(tmp_path):
    assert _client(tmp_path).exists()


@pytest.mark.gpu
def test_c_client_runs(tmp_path):
    r = subprocess.run([str(_client(tmp_path))], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
