"""The reference-side binding integration/run_b200.cc (Run() of
gpudocksm-rem-1.2/src/run.h on this library) compiles against the
reference's own headers and links the reference's driver (dock.C + loaders)
with libgpudock.so into a drop-in linear_dock.  Needs the reference
checkout; skipped where it is absent (the GPU box)."""
import os
import subprocess

import pytest

from gpudock_b200 import lib
from oracle.oracle import reference_root

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = reference_root() or ""
SRC = os.path.join(REF, "gpudocksm-rem-1.2", "src")


@pytest.mark.skipif(not os.path.isdir(SRC), reason="reference sources not available")
def test_run_shim_links_reference_driver(tmp_path):
    shim = os.path.join(ROOT, "integration", "run_b200.cc")
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
