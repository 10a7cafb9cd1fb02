"""Generates the golden fixtures of the parity tests from the reference itself.

Run in a tree where the reference's sources exist (they are compiled into oracle/_ref/libreaxref.so by
oracle/Makefile):  python tests/golden/make_golden.py

Writes, for every small parity system (tests/helpers.py small_systems), the reference cpu64 engine's 13 energies,
the owner-folded gradient and the 7-row decision census into tests/golden/<name>.npz, and the reference's canonical
table dump of the synthetic force field into tests/golden/ffield_synthetic.dump.txt.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "metal-reax_b200"))
sys.path.insert(0, str(HERE.parent))

from helpers import fixed_charges, ffield_text, small_systems  # noqa: E402
from oracle.oracle import RefOracle  # noqa: E402


def main():
    ref = RefOracle(ffield_text(), shell=15.0)
    (HERE / "ffield_synthetic.dump.txt").write_text(ref.table_dump())
    for s in small_systems():
        q = fixed_charges(s)
        r = ref.single_point(s, q)
        np.savez_compressed(HERE / (s["name"] + ".npz"), x=s["x"], type=s["type"], tag=s["tag"], box=s["box"],
                            origin=s["origin"], periodic=s["periodic"], q=q, e=r["e"], grad=r["grad"], census=r["census"],
                            counts=r["counts"])
        print(s["name"], len(s["type"]), r["counts"])


if __name__ == "__main__":
    main()
