"""The reference-side binding of INTEGRATION.md compiles against the
reference's own headers and links the reference's driver (dock.C + loaders)
with libgpudock.so into a drop-in linear_dock.  Needs the reference
checkout; skipped where it is absent (the GPU box)."""
import os
import re
import subprocess

import pytest

from gpudock_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("GD_REFERENCE", "/root/reference")
SRC = os.path.join(REF, "gpudocksm-rem-1.2", "src")


@pytest.mark.skipif(not os.path.isdir(SRC), reason="reference sources not available")
def test_run_shim_links_reference_driver(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    code = re.findall(r"```cpp\n(.*?)```", text, re.S)[0]
    shim = tmp_path / "run_b200.cc"
    shim.write_text(code)
    lib.load()
    libdir = os.path.join(ROOT, "gpudock_b200", "_lib")
    exe = tmp_path / "linear_dock_b200"
    cmd = ["g++", "-O1", "-w", f"-I{SRC}", f"-I{ROOT}/include", "-o", str(exe), str(shim),
           os.path.join(ROOT, "oracle", "ref", "u3b_kabsch.cc"),
           *[os.path.join(SRC, f) for f in ("dock.C", "load.C", "data.C", "util.C",
                                            "quicksort.C")],
           f"-L{libdir}", "-lgpudock", f"-Wl,-rpath,{libdir}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    syms = subprocess.run(["nm", "-C", str(exe)], capture_output=True, text=True).stdout
    assert "Run(Ligand const*" in syms and "gd_run" in syms
