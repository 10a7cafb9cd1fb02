#!/usr/bin/env python3
"""Writes ``ffield.synthetic.cho``: a SYNTHETIC three-element (C, H, O) ReaxFF parameter file.

The pinned ``ffield.reax.cho`` of the reference (sha256 c5240c07...9aee, listed in the reference's
tests/fixtures/ffield_manifest.tsv:9) is not available here, so every CHO workload of this project runs on
this file instead. Its values are chosen by hand to be of plausible ReaxFF magnitude; they are not the
published CHO parameters and results obtained with them are labelled "synthetic".

The layout is the one the reference's reader accepts (src/io/ffield_parser.cpp:91-451):
39 general parameters, four lines per element, two lines per bond block, off-diagonal lines,
valence-angle, torsion and hydrogen-bond lines. The file is built so that every energy term of the hot
path is active:
  * vdW type 3 (inner wall + shielding): every element has rcore2/acore2 > 0.01 and gamma_w > 0.5;
  * bond-order corrections with and without f1 (ovc) and f4/f5 (v13cor);
  * C2 correction (gp[5] > 0.001), triple-bond stabilisation (C mass 12.0000, O mass 15.9990);
  * lone pair, over/under coordination, angles with positive and negative p_val1, penalty, coalition;
  * explicit and 0-X-Y-0 torsions, O-H...O hydrogen bonds, and the light-element valency override for O.

Run:  python make_synthetic_ffield.py [output path [variant]]   (variants: see VARIANTS)
"""
import sys
from pathlib import Path

GENERAL = [
    50.0,    # 0  p_boc1
    9.5,     # 1  p_boc2
    26.0,    # 2  p_coa2
    1.75,    # 3  triple-bond stabilisation
    6.5,     # 4  triple-bond stabilisation
    55.0,    # 5  p_lp3 (C2 correction)
    1.05,    # 6  p_ovun6
    4.5,     # 7  triple-bond stabilisation
    12.0,    # 8  p_ovun7
    13.0,    # 9  p_ovun8
    -65.0,   # 10 triple-bond stabilisation energy
    0.0,     # 11 lower taper radius
    10.0,    # 12 upper taper radius
    2.5,     # 13 (unused)
    33.0,    # 14 p_val6
    6.0,     # 15 p_lp1
    1.05,    # 16 p_val9
    2.0,     # 17 p_val10
    6.0,     # 18 (unused)
    7.0,     # 19 p_pen2
    0.4,     # 20 p_pen3
    4.0,     # 21 p_pen4
    -2.5,    # 22 (unused)
    5.5,     # 23 p_tor2
    10.0,    # 24 p_tor3
    2.0,     # 25 p_tor4
    -1.25,   # 26 (unused)
    2.0,     # 27 p_cot2
    1.55,    # 28 p_vdW1
    0.1,     # 29 bond-order cutoff x 100
    2.0,     # 30 p_coa4
    0.7,     # 31 p_ovun4
    50.0,    # 32 p_ovun3
    1.8,     # 33 p_val8
    0.5,     # 34 (unused)
    20.0,    # 35 lg scaling (unused without lgvdw)
    5.0,     # 36 (unused)
    0.0,     # 37 gp37: 0 -> triple-bond stabilisation only for the C/O mass pair
    2.75,    # 38 p_coa3
]

# per element: four lines of values (after the symbol on the first line)
ATOMS = [
    ("C", [1.38, 4.0, 12.0000, 1.95, 0.085, 0.90, 1.24, 4.0],
          [9.8, 2.2, 4.0, 33.0, 0.0, 5.9, 7.0, 0.0],
          [1.20, 0.0, 13.0, 30.0, 2.0, 8.0, 0.0, 0.0],
          [-4.0, 2.0, 1.0, 4.0, 2.9, 1.85, 0.05, 10.0]),
    ("H", [0.86, 1.0, 1.0080, 1.40, 0.090, 0.82, -0.10, 1.0],
          [9.4, 5.0, 1.0, 0.0, 0.0, 3.7, 9.6, 1.0],
          [-0.10, 0.0, 1.0, 3.0, 1.0, 4.0, 0.0, 0.0],
          [-15.0, 2.0, 1.0, 1.0, 2.9, 1.30, 0.02, 8.0]),
    ("O", [1.24, 2.0, 15.9990, 2.35, 0.100, 1.08, 1.05, 6.0],
          [9.7, 13.0, 4.0, 37.0, 0.0, 8.5, 8.3, 2.0],
          [0.92, 0.45, 0.0, 1.0, 2.5, 1.0, 0.0, 0.0],
          [-3.6, 2.9, 1.0, 2.0, 2.9, 1.90, 0.04, 9.0]),
]

# (i, j) 1-based: line 1 De_s De_p De_pp p_be1 p_bo5 v13cor p_bo6 p_ovun1 ; line 2 p_be2 p_bo3 p_bo4 (skip) p_bo1 p_bo2 ovc (skip)
BONDS = [
    (1, 1, [156.0, 100.0, 78.0, -0.75, -0.40, 1.0, 27.0, 0.44], [0.43, -0.08, 6.8, 1.0, -0.08, 6.8, 1.0, 0.0]),
    (1, 2, [168.0, 0.0, 0.0, -0.50, 0.0, 1.0, 6.0, 0.72], [6.0, -0.10, 6.0, 0.0, -0.05, 6.8, 0.0, 0.0]),
    (1, 3, [160.0, 120.0, 140.0, -0.10, -0.50, 1.0, 30.0, 0.95], [0.50, -0.30, 7.0, 1.0, -0.10, 5.2, 1.0, 0.0]),
    (2, 2, [150.0, 0.0, 0.0, -0.50, 0.0, 1.0, 6.0, 0.73], [6.0, -0.10, 6.0, 0.0, -0.08, 6.1, 0.0, 0.0]),
    (2, 3, [180.0, 0.0, 0.0, -0.95, 0.0, 1.0, 6.0, 0.60], [1.00, -0.10, 6.0, 0.0, -0.09, 4.5, 0.0, 0.0]),
    (3, 3, [140.0, 150.0, 0.0, 0.25, -0.20, 1.0, 30.0, 0.60], [0.50, -0.12, 7.5, 1.0, -0.12, 5.5, 1.0, 0.0]),
]

# (i, j) D r_vdW alpha r_s r_p r_pp   (values <= 0 keep the mixed value)
OFFDIAG = [
    (1, 2, [0.11, 1.90, 10.0, 1.10, -1.0, -1.0]),
    (1, 3, [0.12, 1.80, 10.2, 1.30, 1.10, 1.20]),
    (2, 3, [0.03, 1.70, 10.5, 0.95, -1.0, -1.0]),
]

# (i, j, k) centre j:  theta_00 p_val1 p_val2 p_coa1 p_val7 p_pen1 p_val4
ANGLES = [
    (1, 1, 1, [68.0, 22.0, 1.6, 0.0, 1.8, 15.0, 1.8]),
    (1, 1, 1, [60.0, -4.0, 1.0, 0.0, 0.5, 0.0, 1.2]),
    (1, 1, 2, [72.0, 30.0, 2.0, 0.0, 1.0, 0.0, 1.1]),
    (2, 1, 2, [70.0, 25.0, 3.4, 0.0, 0.0, 0.0, 3.0]),
    (1, 1, 3, [75.0, 35.0, 1.2, -25.0, 2.0, 50.0, 1.1]),
    (2, 1, 3, [70.0, 33.0, 1.5, 0.0, 1.5, 0.0, 1.1]),
    (3, 1, 3, [77.0, 40.0, 0.8, -26.0, 2.5, 60.0, 1.1]),
    (1, 3, 1, [70.0, 20.0, 1.5, 0.0, 1.0, 0.0, 1.2]),
    (1, 3, 2, [76.0, 12.0, 1.8, 0.0, 2.0, 0.0, 1.2]),
    (2, 3, 2, [78.0, 15.0, 2.0, 0.0, 1.0, 0.0, 1.2]),
    (2, 3, 3, [80.0, 10.0, 2.5, 0.0, 1.0, 0.0, 1.2]),
    (3, 3, 3, [80.0, 30.0, 1.2, 0.0, 1.5, 40.0, 1.1]),
    (1, 2, 1, [0.0, 3.0, 1.0, 0.0, 1.0, 0.0, 1.0]),
    (3, 2, 3, [0.0, 4.0, 2.0, 0.0, 1.0, 0.0, 1.2]),
    (1, 2, 3, [0.0, -2.0, 1.5, 0.0, 1.0, 0.0, 1.1]),
]

# (i, j, k, l): V1 V2 V3 p_tor1 p_cot1 (+ two unused columns); 0 = wildcard end atom
TORSIONS = [
    (1, 1, 1, 1, [-0.25, 34.0, 0.03, -6.5, -2.4, 0.0, 0.0]),
    (1, 1, 1, 2, [-0.20, 38.0, 0.20, -4.8, -2.0, 0.0, 0.0]),
    (2, 1, 1, 2, [-0.18, 38.0, 0.34, -4.5, -2.0, 0.0, 0.0]),
    (0, 1, 1, 0, [0.0, 50.0, 0.30, -4.0, -2.0, 0.0, 0.0]),
    (0, 1, 3, 0, [0.50, 0.0, 0.60, -5.0, -1.5, 0.0, 0.0]),
    (0, 3, 3, 0, [0.60, 40.0, 0.45, -2.5, -1.2, 0.0, 0.0]),
    (0, 2, 3, 0, [0.0, 0.10, 0.02, -2.5, 0.0, 0.0, 0.0]),
    (2, 3, 1, 1, [-1.5, 60.0, 0.15, -9.0, -1.0, 0.0, 0.0]),
]

# (donor i, H j, acceptor k): r0_hb p_hb1 p_hb2 p_hb3
HBONDS = [
    (3, 2, 3, [2.10, -3.0, 1.5, 15.0]),
    (1, 2, 3, [2.25, -1.0, 1.2, 12.0]),
]


def fmt(v):
    return f"{v:10.4f}"


# lgvdw data per element (fifth atom line): lgcij, lgre; the off-diagonal lines then carry an lgcij column
LG = {"C": (400.0, 1.95), "H": (30.0, 1.40), "O": (150.0, 1.75)}
OFFDIAG_LG = {(1, 2): 110.0, (1, 3): -1.0, (2, 3): 60.0}

# variants of the file that switch the non-bonded branches (the van der Waals method follows from the atom lines,
# src/io/ffield_parser.cpp:207-230): "vdw3" inner wall + shielding (the default), "vdw1" shielding only (no inner
# wall: rcore2 = acore2 = 0), "vdw2" inner wall only (gamma_w <= 0.5), "lg" the default with lgvdw data (read with
# `lgvdw yes`; gp[35] = 0.5 so that lgre = sqrt(lgre_i lgre_j))
# "acks2": the default with ACKS2 bond-softness cut-offs on the atom lines (bcut_acks2, line 3 column 7) and the
# softness gp[34] = 2.0, for the pair side of the ACKS2 charge model
ACKS2_BCUT = {"C": 5.5, "H": 4.5, "O": 5.0}
VARIANTS = ("vdw3", "vdw1", "vdw2", "lg", "acks2")


def render(variant="vdw3"):
    if variant not in VARIANTS:
        raise ValueError("unknown variant %r" % variant)
    general = list(GENERAL)
    atoms = [(n, list(l1), list(l2), list(l3), list(l4)) for n, l1, l2, l3, l4 in ATOMS]
    if variant == "vdw1":
        for a in atoms:
            a[4][5] = a[4][7] = 0.0
    elif variant == "vdw2":
        for a in atoms:
            a[2][1] = 0.4
    elif variant == "lg":
        general[35] = 0.5
    elif variant == "acks2":
        general[34] = 2.0
        for a in atoms:
            a[3][6] = ACKS2_BCUT[a[0]]
    title = "Synthetic C/H/O ReaxFF parameter set (not the published CHO file; see make_synthetic_ffield.py)"
    out = [title if variant == "vdw3" else title + " variant " + variant]
    out.append(f"{len(general):3d}       ! Number of general parameters")
    for i, v in enumerate(general):
        out.append(f"{fmt(v)} !gp{i}")
    out.append(f"{len(ATOMS):3d}    ! Nr of atoms; cov.r; valency;a.m;Rvdw;Evdw;gammaEEM;cov.r2;#")
    out.append("            alfa;gammavdW;valency;Eunder;Eover;chiEEM;etaEEM;n.u.")
    out.append("            cov r3;Elp;Heat inc.;n.u.;n.u.;n.u.;n.u.")
    out.append("            ov/un;val1;n.u.;val3,vval4")
    for name, l1, l2, l3, l4 in atoms:
        out.append(f" {name:<2}" + "".join(fmt(v) for v in l1))
        out.append("   " + "".join(fmt(v) for v in l2))
        out.append("   " + "".join(fmt(v) for v in l3))
        out.append("   " + "".join(fmt(v) for v in l4))
        if variant == "lg":
            out.append("   " + "".join(fmt(v) for v in LG[name]))
    out.append(f"{len(BONDS):3d}      ! Nr of bonds; Edis1;LPpen;n.u.;pbe1;pbo5;13corr;pbo6")
    out.append("                         pbe2;pbo3;pbo4;n.u.;pbo1;pbo2;ovcorr")
    for i, j, l1, l2 in BONDS:
        out.append(f"{i:3d}{j:3d}" + "".join(fmt(v) for v in l1))
        out.append("      " + "".join(fmt(v) for v in l2))
    out.append(f"{len(OFFDIAG):3d}    ! Nr of off-diagonal terms; at1;at2;Dij;RvdW;alfa;ro(sigma);ro(pi);ro(pipi)")
    for i, j, vals in OFFDIAG:
        extra = [OFFDIAG_LG[(i, j)]] if variant == "lg" else []
        out.append(f"{i:3d}{j:3d}" + "".join(fmt(v) for v in list(vals) + extra))
    out.append(f"{len(ANGLES):3d}    ! Nr of angles;at1;at2;at3;Thetao,o;ka;kb;pv1;pv2")
    for i, j, k, vals in ANGLES:
        out.append(f"{i:3d}{j:3d}{k:3d}" + "".join(fmt(v) for v in vals))
    out.append(f"{len(TORSIONS):3d}    ! Nr of torsions;at1;at2;at3;at4;;V1;V2;V3;V2(BO);vconj;n.u;n")
    for i, j, k, l, vals in TORSIONS:
        out.append(f"{i:3d}{j:3d}{k:3d}{l:3d}" + "".join(fmt(v) for v in vals))
    out.append(f"{len(HBONDS):3d}    ! Nr of hydrogen bonds;at1;at2;at3;Rhb;Dehb;vhb1")
    for i, j, k, vals in HBONDS:
        out.append(f"{i:3d}{j:3d}{k:3d}" + "".join(fmt(v) for v in vals))
    return "\n".join(out) + "\n"


def main():
    path = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("ffield.synthetic.cho")
    variant = sys.argv[2] if len(sys.argv) > 2 else "vdw3"
    path.write_text(render(variant))
    print(path)


if __name__ == "__main__":
    main()
