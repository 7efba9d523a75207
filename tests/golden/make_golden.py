"""Generates the committed golden fixtures under tests/golden/ from the
reference's source text (run once in a container that has the reference;
the fixtures travel, the reference does not).

  peirce_m14.json  -- the m = 14 Peirce sphere-quadrature node/weight
                      literals of include/alluvion/dg/peirce_quadrature.hpp
                      (lines 180-304), used to pin the oracle's and the
                      engine's independently computed tables.

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def peirce_m14(ref_root):
    path = os.path.join(ref_root, "include", "alluvion", "dg", "peirce_quadrature.hpp")
    text = open(path).read()
    start = text.index("kPeirceM == 14")
    end = text.index("kPeirceM == 20")
    block = text[start:end]
    out = {}
    for name in ("cosphi", "sinphi", "b", "r", "c"):
        vals = {}
        for m in re.finditer(r"\b%s\[(\d+)\]\s*=\s*([-+0-9.eE]+);" % name, block):
            vals[int(m.group(1))] = float(m.group(2))
        out[name] = [vals[k] for k in range(len(vals))]
    return {"source": "include/alluvion/dg/peirce_quadrature.hpp (kPeirceM == 14 block)",
            "tables": out}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    with open(os.path.join(HERE, "peirce_m14.json"), "w") as f:
        json.dump(peirce_m14(ref), f, indent=1)
    print("wrote", os.path.join(HERE, "peirce_m14.json"))


if __name__ == "__main__":
    main()
