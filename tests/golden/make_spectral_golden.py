"""Extract the nPol = 4 GLL/GLJ tables of the reference as a golden fixture.

Reads SOLVER/src/preloop/se_model/quad/spectrals.hpp of the reference checkout
(as text, nothing is compiled or executed) and writes spectral_npol4.json next
to this script. Run once where a reference checkout is present, naming its root:

    python tests/golden/make_spectral_golden.py <reference checkout>
"""
import json
import os
import re
import sys


def extract(path):
    src = open(path).read()
    block = src.split("#elif _NPOL == 4", 1)[1].split("#elif", 1)[0]
    out = {}
    for name in ("pGLL", "pGLJ", "wGLL", "wGLJ", "gGLL", "gGLJ"):
        m = re.search(r"%s\s*=\s*\{([^}]*)\}" % name, block)
        out[name] = [float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_spectral_golden.py <reference checkout root>")
    ref = sys.argv[1]
    tables = extract(os.path.join(ref, "SOLVER/src/preloop/se_model/quad/spectrals.hpp"))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "spectral_npol4.json")
    with open(dst, "w") as f:
        json.dump({"source": "SOLVER/src/preloop/se_model/quad/spectrals.hpp:73-102 (_NPOL == 4)",
                   "tables": tables}, f, indent=1)
    print("wrote", dst)
