"""TEST INFRASTRUCTURE ONLY: a Python restatement of the reference's ffield reader and of its canonical table dump.

* ``parse(text)`` follows src/io/ffield_parser.cpp:91-451 (strict mode, no lgvdw): general parameters, atom blocks
  (with the light-element valency override, :233-240, and the vdW-type rule, :207-231), bond blocks, the mixing rules
  (:284-306), off-diagonal overrides (:308-333), valence-angle sets mirrored into (l, k, j) (:335-368), torsions with
  the compact 0-X-Y-0 form and its order-dependent overwrite (:370-401), and the optional H-bond block (:403-426).
* ``canonical_dump(t)`` restates src/io/table_dump.cpp:20-84 (the "%.17g" text the reference uses to prove two parses
  identical), so a parse here can be compared byte for byte with the reference's own.
* ``oracle_arrays(t)`` lays the tables out for the C restatement (rx_oracle.h field offsets).
"""
import math

import numpy as np

SB_FIELDS = ["r_s", "valency", "mass", "r_vdw", "epsilon", "gamma", "r_pi", "valency_e", "nlp_opt", "alpha", "gamma_w",
             "valency_boc", "p_ovun5", "chi", "eta", "p_hbond", "r_pi_pi", "p_lp2", "b_o_131", "b_o_132", "b_o_133",
             "p_ovun2", "p_val3", "valency_val", "p_val5", "rcore2", "ecore2", "acore2", "heavy", "c2species", "bcut_acks2"]
TB_FIELDS = ["p_bo1", "p_bo2", "p_bo3", "p_bo4", "p_bo5", "p_bo6", "r_s", "r_p", "r_pp", "p_boc3", "p_boc4", "p_boc5",
             "p_be1", "p_be2", "De_s", "De_p", "De_pp", "p_ovun1", "D", "alpha", "r_vdW", "gamma_w", "rcore", "ecore",
             "acore", "lgcij", "lgre", "gamma", "v13cor", "ovc", "triple_stab"]
TH_FIELDS = ["theta_00", "p_val1", "p_val2", "p_val4", "p_val7", "p_pen1", "p_coa1"]
FB_FIELDS = ["V1", "V2", "V3", "p_tor1", "p_cot1"]
HB_FIELDS = ["r0_hb", "p_hb1", "p_hb2", "p_hb3"]
MAX_THB = 5


class FfieldError(ValueError):
    pass


class _Reader:
    def __init__(self, text):
        self.lines = text.split("\n")
        self.pos = 0

    def raw(self):
        if self.pos >= len(self.lines):
            return None
        line = self.lines[self.pos]
        self.pos += 1
        return line

    def values(self, required=True):
        while True:
            line = self.raw()
            if line is None:
                if required:
                    raise FfieldError("unexpected end of file")
                return None
            toks = line.split()
            if toks:
                return toks

    def skip(self):
        if self.raw() is None:
            raise FfieldError("unexpected end of file")


def _f(tok):
    v = float(tok)
    if not math.isfinite(v):
        raise FfieldError("non-finite value %r" % tok)
    return v


def parse(text, lgvdw=False):
    """The reader's tables; lgvdw=True reads `pair_style reaxff lgvdw yes` files (a fifth line per element with lgcij
    and lgre, an lgcij column on the off-diagonal lines: src/io/ffield_parser.cpp:196-205,314-330)."""
    rd = _Reader(text)
    first = rd.values()  # header comment line (src/io/ffield_parser.cpp:100-115)
    if (first and first[0].isdigit() and len(first) >= 2 and first[1].startswith("!")
            and "general parameters" in " ".join(first) + " "):
        raise FfieldError("first line of ReaxFF potential file must be a comment or empty")
    v = rd.values()
    ngp = int(v[0])
    if ngp < 38:
        raise FfieldError("need at least 38 general parameters")
    gp = [_f(rd.values()[0]) for _ in range(ngp)]
    nt = int(rd.values()[0])
    rd.skip(); rd.skip(); rd.skip()
    sbp = []
    vdw_type = 0
    for _ in range(nt):
        s = {}
        t = rd.values()
        if len(t) < 9:
            raise FfieldError("atom line 1 needs 9 columns")
        s["name"] = t[0][:3].upper()
        for k, key in enumerate(["r_s", "valency", "mass", "r_vdw", "epsilon", "gamma", "r_pi", "valency_e"]):
            s[key] = _f(t[1 + k])
        s["nlp_opt"] = 0.5 * (s["valency_e"] - s["valency"])
        t = rd.values()
        if len(t) < 8:
            raise FfieldError("atom line 2 needs 8 columns")
        s["alpha"], s["gamma_w"], s["valency_boc"], s["p_ovun5"] = (_f(x) for x in t[0:4])
        s["chi"] = _f(t[5])
        s["eta"] = 2.0 * _f(t[6])
        s["p_hbond"] = int(_f(t[7]))
        t = rd.values()
        if len(t) < 8:
            raise FfieldError("atom line 3 needs 8 columns")
        s["r_pi_pi"], s["p_lp2"] = _f(t[0]), _f(t[1])
        s["b_o_131"], s["b_o_132"], s["b_o_133"], s["bcut_acks2"] = (_f(x) for x in t[3:7])
        t = rd.values()
        if len(t) < 8:
            raise FfieldError("atom line 4 needs 8 columns")
        s["p_ovun2"], s["p_val3"] = _f(t[0]), _f(t[1])
        s["valency_val"], s["p_val5"], s["rcore2"], s["ecore2"], s["acore2"] = (_f(x) for x in t[3:8])
        if lgvdw:
            t = rd.values()
            try:
                float(t[0])
            except ValueError:
                raise FfieldError("ReaxFF potential file is not compatible with 'lgvdw yes'")
            if len(t) < 2:
                raise FfieldError("lgvdw line needs 2 columns")
            s["lgcij"], s["lgre"] = _f(t[0]), _f(t[1])
        else:
            s["lgcij"] = s["lgre"] = 0.0
        inner = s["rcore2"] > 0.01 and s["acore2"] > 0.01
        shield = s["gamma_w"] > 0.5
        want = 3 if (inner and shield) else 2 if inner else 1 if shield else 0
        if want == 0:
            raise FfieldError("no shielding or inner wall for element " + s["name"])
        if vdw_type == 0:
            vdw_type = want
        sbp.append(s)
    for s in sbp:
        s["heavy"] = 1.0 if s["mass"] > 21.0 else 0.0
        s["c2species"] = 1.0 if s["name"] == "C" else 0.0
        if s["mass"] < 21 and s["valency_val"] != s["valency_boc"]:
            s["valency_val"] = s["valency_boc"]
    tb = [[dict.fromkeys(TB_FIELDS, 0.0) for _ in range(nt)] for _ in range(nt)]
    listed = np.zeros((nt, nt), dtype=bool)
    nb = int(rd.values()[0])
    rd.skip()
    for _ in range(nb):
        t = rd.values()
        j, k = int(t[0]) - 1, int(t[1]) - 1
        t2 = rd.values()
        if j < nt and k < nt:
            vals1 = dict(zip(["De_s", "De_p", "De_pp", "p_be1", "p_bo5", "v13cor", "p_bo6", "p_ovun1"], (_f(x) for x in t[2:10])))
            vals2 = {"p_be2": _f(t2[0]), "p_bo3": _f(t2[1]), "p_bo4": _f(t2[2]), "p_bo1": _f(t2[4]), "p_bo2": _f(t2[5]),
                     "ovc": _f(t2[6]) if len(t2) > 6 else 0.0}
            for d in (vals1, vals2):
                for key, val in d.items():
                    tb[j][k][key] = val
                    tb[k][j][key] = val
            listed[j, k] = listed[k, j] = True
    for i in range(nt):
        for j in range(i, nt):
            si, sj = sbp[i], sbp[j]
            mix = {
                "r_s": 0.5 * (sj["r_s"] + si["r_s"]),
                "r_p": 0.5 * (sj["r_pi"] + si["r_pi"]),
                "r_pp": 0.5 * (sj["r_pi_pi"] + si["r_pi_pi"]),
                "p_boc3": math.sqrt(sj["b_o_132"] * si["b_o_132"]),
                "p_boc4": math.sqrt(sj["b_o_131"] * si["b_o_131"]),
                "p_boc5": math.sqrt(sj["b_o_133"] * si["b_o_133"]),
                "D": math.sqrt(sj["epsilon"] * si["epsilon"]),
                "alpha": math.sqrt(sj["alpha"] * si["alpha"]),
                "r_vdW": 2.0 * math.sqrt(sj["r_vdw"] * si["r_vdw"]),
                "gamma_w": math.sqrt(sj["gamma_w"] * si["gamma_w"]),
                "gamma": math.pow(sj["gamma"] * si["gamma"], -1.5),
                "rcore": math.sqrt(si["rcore2"] * sj["rcore2"]),
                "ecore": math.sqrt(si["ecore2"] * sj["ecore2"]),
                "acore": math.sqrt(si["acore2"] * sj["acore2"]),
                "lgcij": math.sqrt(si["lgcij"] * sj["lgcij"]),
                "lgre": 2.0 * gp[35] * math.sqrt(si["lgre"] * sj["lgre"]),
            }
            for key, val in mix.items():
                tb[i][j][key] = val
                tb[j][i][key] = val
    no = int(rd.values()[0])
    for _ in range(no):
        t = rd.values()
        if len(t) < 8 + (1 if lgvdw else 0):
            raise FfieldError("off-diagonal line needs %d columns" % (8 + (1 if lgvdw else 0)))
        j, k = int(t[0]) - 1, int(t[1]) - 1
        if j < nt and k < nt:
            for key, tok, scale in (("D", t[2], 1.0), ("r_vdW", t[3], 2.0), ("alpha", t[4], 1.0), ("r_s", t[5], 1.0),
                                    ("r_p", t[6], 1.0), ("r_pp", t[7], 1.0)):
                val = _f(tok)
                if val > 0.0:
                    tb[j][k][key] = scale * val
                    tb[k][j][key] = scale * val
            if lgvdw:
                val = _f(t[8])
                if val >= 0.0:
                    tb[j][k]["lgcij"] = val
                    tb[k][j]["lgcij"] = val
    thb = {}
    slots = {}
    n3 = int(rd.values()[0])
    for _ in range(n3):
        t = rd.values()
        j, k, l = int(t[0]) - 1, int(t[1]) - 1, int(t[2]) - 1
        if j < nt and k < nt and l < nt:
            vals = [_f(x) for x in t[3:10]]  # theta_00 p_val1 p_val2 p_coa1 p_val7 p_pen1 p_val4
            s = {"theta_00": vals[0], "p_val1": vals[1], "p_val2": vals[2], "p_coa1": vals[3], "p_val7": vals[4],
                 "p_pen1": vals[5], "p_val4": vals[6]}
            slots[(j, k, l)] = slots.get((j, k, l), 0) + 1
            slots[(l, k, j)] = slots.get((l, k, j), 0) + 1
            if slots[(j, k, l)] > MAX_THB or slots[(l, k, j)] > MAX_THB:
                raise FfieldError("too many valence-angle sets for one triple")
            thb.setdefault((j, k, l), []).append(s)
            if j != l:
                thb.setdefault((l, k, j), []).append(s)
    fbp = {}
    explicit = set()
    n4 = int(rd.values()[0])
    for _ in range(n4):
        t = rd.values()
        j, k, l, m = (int(x) - 1 for x in t[0:4])
        vals = dict(zip(FB_FIELDS, (_f(x) for x in t[4:9])))
        if j >= 0 and m >= 0:
            if j < nt and k < nt and l < nt and m < nt:
                explicit.add((j, k, l, m))
                explicit.add((m, l, k, j))
                fbp[(j, k, l, m)] = vals
                fbp[(m, l, k, j)] = vals
        elif k < nt and l < nt:
            for p in range(nt):
                for o in range(nt):
                    if (p, k, l, o) not in explicit:
                        fbp[(p, k, l, o)] = vals
                    if (o, l, k, p) not in explicit:
                        fbp[(o, l, k, p)] = vals
    hbp = {}
    t = rd.values(required=False)
    if t is not None:
        for _ in range(int(t[0])):
            t = rd.values()
            j, k, l = int(t[0]) - 1, int(t[1]) - 1, int(t[2]) - 1
            if j < nt and k < nt and l < nt:
                hbp[(j, k, l)] = dict(zip(HB_FIELDS, (_f(x) for x in t[3:7])))
    gp37 = float(int(gp[37])) == 2
    for i in range(nt):
        for j in range(nt):
            mi, mj = sbp[i]["mass"], sbp[j]["mass"]
            tb[i][j]["triple_stab"] = 1.0 if (gp37 or (mi == 12.0000 and mj == 15.9990) or (mj == 12.0000 and mi == 15.9990)) else 0.0
    return {"gp": gp, "nt": nt, "sbp": sbp, "tbp": tb, "thb": thb, "fbp": fbp, "hbp": hbp, "vdw_type": vdw_type,
            "bo_cut": 0.01 * gp[29], "nonb_low": gp[11], "nonb_cut": gp[12], "listed": listed}


def _g(v):
    return " %s" % repr_17g(v)


def repr_17g(v):
    return "%.17g" % v


def canonical_dump(t, portable=False):
    """src/io/table_dump.cpp:20-84"""
    o = ["FFIELD-TABLES 1"]
    o.append("GP %d %d" % (len(t["gp"]), t["vdw_type"]))
    for i, v in enumerate(t["gp"]):
        o.append("G %d%s" % (i, _g(v)))
    n = t["nt"]
    for i, s in enumerate(t["sbp"]):
        line = "S %d %s" % (i, s["name"])
        for key in ["r_s", "valency", "mass", "r_vdw", "epsilon", "gamma", "r_pi", "valency_e", "nlp_opt", "alpha", "gamma_w",
                    "valency_boc", "p_ovun5"]:
            line += _g(s[key])
        line += " %d" % s["p_hbond"]
        for key in ["chi", "eta", "r_pi_pi", "p_lp2", "b_o_131", "b_o_132", "b_o_133", "bcut_acks2", "p_ovun2", "p_val3",
                    "valency_val", "p_val5", "rcore2", "ecore2", "acore2", "lgcij", "lgre"]:
            line += _g(s[key])
        o.append(line)
    for i in range(n):
        for j in range(i, n):
            tp = t["tbp"][i][j]
            line = "T %d %d" % (i, j)
            for key in ["p_bo1", "p_bo2", "p_bo3", "p_bo4", "p_bo5", "p_bo6", "r_s", "r_p", "r_pp", "p_boc3", "p_boc4", "p_boc5",
                        "p_be1", "p_be2", "De_s", "De_p", "De_pp", "p_ovun1", "D", "alpha", "r_vdW", "gamma_w", "rcore", "ecore",
                        "acore", "lgcij", "lgre"]:
                line += _g(tp[key])
            if not portable:
                line += _g(tp["gamma"])
            line += _g(tp["v13cor"]) + _g(tp["ovc"])
            o.append(line)
    for j in range(n):
        for k in range(n):
            for l in range(n):
                sets = t["thb"].get((j, k, l))
                if not sets:
                    continue
                line = "H3 %d %d %d %d" % (j, k, l, len(sets))
                for s in sets:
                    for key in ["theta_00", "p_val1", "p_val2", "p_val4", "p_val7", "p_pen1", "p_coa1"]:
                        line += _g(s[key])
                o.append(line)
    for j in range(n):
        for k in range(n):
            for l in range(n):
                for m in range(n):
                    f = t["fbp"].get((j, k, l, m))
                    if f is None:
                        continue
                    o.append("H4 %d %d %d %d" % (j, k, l, m) + "".join(_g(f[key]) for key in FB_FIELDS))
    for j in range(n):
        for k in range(n):
            for l in range(n):
                h = t["hbp"].get((j, k, l))
                if h is None or (h["r0_hb"] == -1.0 and h["p_hb1"] == 0 and h["p_hb2"] == 0 and h["p_hb3"] == 0):
                    continue
                o.append("HB %d %d %d" % (j, k, l) + "".join(_g(h[key]) for key in HB_FIELDS))
    return "\n".join(o) + "\n"


def oracle_arrays(t):
    """Flat arrays in the layout of oracle/rx_oracle.h."""
    nt = t["nt"]
    sbp = np.array([[s[k] for k in SB_FIELDS] for s in t["sbp"]], dtype=np.float64)
    tbp = np.array([[[t["tbp"][i][j][k] for k in TB_FIELDS] for j in range(nt)] for i in range(nt)], dtype=np.float64)
    thb_n = np.zeros((nt, nt, nt), dtype=np.int32)
    thb = np.zeros((nt, nt, nt, MAX_THB, len(TH_FIELDS)))
    for (j, k, l), sets in t["thb"].items():
        thb_n[j, k, l] = len(sets)
        for s_i, s in enumerate(sets):
            thb[j, k, l, s_i] = [s[key] for key in TH_FIELDS]
    fbp_on = np.zeros((nt,) * 4, dtype=np.int32)
    fbp = np.zeros((nt,) * 4 + (len(FB_FIELDS),))
    for key, f in t["fbp"].items():
        fbp_on[key] = 1
        fbp[key] = [f[k] for k in FB_FIELDS]
    hbp_on = np.zeros((nt,) * 3, dtype=np.int32)
    hbp = np.zeros((nt,) * 3 + (len(HB_FIELDS),))
    for key, h in t["hbp"].items():
        hbp_on[key] = 1
        hbp[key] = [h[k] for k in HB_FIELDS]
    gp = np.zeros(max(39, len(t["gp"])))   # a 38-parameter file has no p_coa3 (gp[38]): it reads 0, as on the device
    gp[:len(t["gp"])] = t["gp"]
    return {"gp": gp, "sbp": np.ascontiguousarray(sbp), "tbp": np.ascontiguousarray(tbp),
            "thb_n": thb_n, "thb": np.ascontiguousarray(thb), "fbp_on": fbp_on, "fbp": np.ascontiguousarray(fbp),
            "hbp_on": hbp_on, "hbp": np.ascontiguousarray(hbp)}
