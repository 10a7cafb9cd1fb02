"""Generates the golden fixtures of the parity tests from the reference itself.

Run in a tree where the reference's sources exist (they are compiled into oracle/_ref/libreaxref.so by
oracle/Makefile):  python tests/golden/make_golden.py

Writes, for every small parity system (tests/helpers.py small_systems), the reference cpu64 engine's 13 energies,
the owner-folded gradient, the 7-row decision census and the fdotr virial (sum over owned + ghost atoms of x f) into
tests/golden/<name>.npz; the same for the water box under the force-field variants vdw1, vdw2 and lg
(tests/golden/water192_<variant>.npz), the ACKS2 variant with seeded kinetic potentials included; and the reference's canonical table dump of the synthetic force field into
tests/golden/ffield_synthetic.dump.txt.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "metal-reax_b200"))
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(REPO / "metal-reax_b200" / "data"))

from helpers import acks2_potentials, fixed_charges, ffield_text, small_systems  # noqa: E402
from oracle.oracle import RefOracle  # noqa: E402


def _save(path, s, q, r, **extra):
    np.savez_compressed(path, x=s["x"], type=s["type"], tag=s["tag"], box=s["box"], origin=s["origin"],
                        periodic=s["periodic"], q=q, e=r["e"], grad=r["grad"], census=r["census"], counts=r["counts"],
                        virial=r["virial"], **extra)
    print(path.name, len(s["type"]), r["counts"])


def main():
    import make_synthetic_ffield
    ref = RefOracle(ffield_text(), shell=15.0)
    (HERE / "ffield_synthetic.dump.txt").write_text(ref.table_dump())
    for s in small_systems():
        q = fixed_charges(s)
        _save(HERE / (s["name"] + ".npz"), s, q, ref.single_point(s, q))
    # the force-field variants that switch the non-bonded branches, on the water box
    s = small_systems()[0]
    q = fixed_charges(s)
    for v in ("vdw1", "vdw2", "lg"):
        rv = RefOracle(make_synthetic_ffield.render(v), shell=15.0, lgvdw=(v == "lg"))
        _save(HERE / ("%s_%s.npz" % (s["name"], v)), s, q, rv.single_point(s, q))
    # the pair side of the ACKS2 charge model, with seeded kinetic potentials
    s_kin = acks2_potentials(len(s["type"]))
    ra = RefOracle(make_synthetic_ffield.render("acks2"), shell=15.0)
    _save(HERE / ("%s_acks2.npz" % s["name"]), s, q, ra.single_point(s, q, s_kin=s_kin), s_kin=s_kin)


if __name__ == "__main__":
    main()
