"""Records the reference headers' struct layouts (sizeof / offsetof) into
tests/golden/abi_layout.json; tests/test_abi.py checks include/ against it.

    WEMA_REF_DIR=<reference checkout> python tests/golden/make_abi_layout.py

The reference checkout defaults to a directory named `reference` beside this
repository.
"""
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.path.dirname(HERE), "c", "abi_layout.c")
REPO = os.path.dirname(os.path.dirname(HERE))
REF_INC = os.path.join(os.environ.get("WEMA_REF_DIR",
                                      os.path.join(os.path.dirname(REPO), "reference")), "src")

with tempfile.TemporaryDirectory() as d:
    exe = os.path.join(d, "layout")
    subprocess.run(["gcc", "-std=c11", "-I", REF_INC, SRC, "-o", exe], check=True)
    out = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
with open(os.path.join(HERE, "abi_layout.json"), "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
print("wrote", len(out), "entries")
