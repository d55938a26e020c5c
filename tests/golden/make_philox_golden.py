"""Generates tests/golden/philox4x32_10.json from the Random123 philox.h that
the reference project vendors (docking/ising/src/Random123, the generator the
reference's Ising code uses), so that the oracle's Philox4x32-10 is pinned to
an independent implementation.

    python tests/golden/make_philox_golden.py [REFERENCE_ROOT]

Compiles a small C++ driver against that header (g++), evaluates seeded
random counters/keys plus the corner cases, and writes the vectors.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = r"""
#include <cstdio>
#include <cstdint>
#include "Random123/philox.h"
int main() {
  unsigned c0, c1, c2, c3, k0, k1;
  while (scanf("%u %u %u %u %u %u", &c0, &c1, &c2, &c3, &k0, &k1) == 6) {
    r123::Philox4x32_R<10> g;
    r123::Philox4x32_R<10>::ctr_type c = {{c0, c1, c2, c3}};
    r123::Philox4x32_R<10>::key_type k = {{k0, k1}};
    r123::Philox4x32_R<10>::ctr_type o = g(c, k);
    printf("%u %u %u %u\n", o.v[0], o.v[1], o.v[2], o.v[3]);
  }
  return 0;
}
"""


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("GD_REFERENCE")
    if not ref:
        sys.exit("usage: give the reference checkout as the argument or in GD_REFERENCE")
    inc = os.path.join(ref, "docking", "ising", "src")
    rng = np.random.default_rng(20240601)
    rows = [[0, 0, 0, 0, 0, 0], [0xFFFFFFFF] * 6,
            [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344, 0xa4093822, 0x299f31d0]]
    rows += rng.integers(0, 2 ** 32, size=(61, 6), dtype=np.uint64).tolist()
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "kat.cc")
        exe = os.path.join(d, "kat")
        with open(src, "w") as f:
            f.write(DRIVER)
        subprocess.run(["g++", "-O1", "-I" + inc, src, "-o", exe], check=True)
        inp = "\n".join(" ".join(str(int(v)) for v in r) for r in rows) + "\n"
        out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout
    outs = [[int(v) for v in line.split()] for line in out.strip().splitlines()]
    data = {"generator": "Random123 philox.h Philox4x32_R<10> (vendored by the reference)",
            "ctr": [r[:4] for r in rows], "key": [r[4:] for r in rows], "out": outs}
    with open(os.path.join(HERE, "philox4x32_10.json"), "w") as f:
        json.dump(data, f)
    print("wrote", len(outs), "vectors")


if __name__ == "__main__":
    main(sys.argv)
