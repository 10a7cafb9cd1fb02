// ReaxFF parameter-file reader (see ffield.hpp for the reference behaviour it follows).
#include "ffield.hpp"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <optional>
#include <set>
#include <array>

namespace rx {
namespace {

struct Line {
  std::vector<std::string> tok;
  int lineno = 0;
};

class Reader {
 public:
  explicit Reader(std::string_view t) : text_(t) {}
  std::optional<std::string_view> raw() {
    if (pos_ >= text_.size()) return std::nullopt;
    const size_t nl = text_.find('\n', pos_);
    const size_t end = nl == std::string_view::npos ? text_.size() : nl;
    std::string_view l = text_.substr(pos_, end - pos_);
    pos_ = nl == std::string_view::npos ? text_.size() : nl + 1;
    ++lineno_;
    return l;
  }
  std::optional<Line> line() {
    while (auto l = raw()) {
      Line out;
      out.lineno = lineno_;
      size_t i = 0;
      while (i < l->size()) {
        while (i < l->size() && isspace(static_cast<unsigned char>((*l)[i]))) ++i;
        if (i >= l->size()) break;
        const size_t s = i;
        while (i < l->size() && !isspace(static_cast<unsigned char>((*l)[i]))) ++i;
        out.tok.emplace_back(l->substr(s, i - s));
      }
      if (!out.tok.empty()) return out;
    }
    return std::nullopt;
  }
  Line values() {
    auto l = line();
    if (!l) throw FfieldError("unexpected end of force-field file at line " + std::to_string(lineno_));
    return *l;
  }
  void skip() {
    if (!raw()) throw FfieldError("unexpected end of force-field file at line " + std::to_string(lineno_));
  }

 private:
  std::string_view text_;
  size_t pos_ = 0;
  int lineno_ = 0;
};

double num(const Line& l, size_t k) {
  if (k >= l.tok.size()) throw FfieldError("line " + std::to_string(l.lineno) + ": missing value");
  const std::string& s = l.tok[k];
  char* end = nullptr;
  errno = 0;
  const double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || static_cast<size_t>(end - s.c_str()) != s.size())
    throw FfieldError("line " + std::to_string(l.lineno) + ": '" + s + "' is not a number");
  if (!std::isfinite(v)) throw FfieldError("line " + std::to_string(l.lineno) + ": '" + s + "' is not finite");
  return v;
}
int inum(const Line& l, size_t k) {
  if (k >= l.tok.size()) throw FfieldError("line " + std::to_string(l.lineno) + ": missing value");
  const std::string& s = l.tok[k];
  char* end = nullptr;
  const long v = std::strtol(s.c_str(), &end, 10);
  if (end == s.c_str() || static_cast<size_t>(end - s.c_str()) != s.size())
    throw FfieldError("line " + std::to_string(l.lineno) + ": '" + s + "' is not an integer");
  return static_cast<int>(v);
}
void need(const Line& l, size_t n) {
  if (l.tok.size() < n)
    throw FfieldError("line " + std::to_string(l.lineno) + ": expected " + std::to_string(n) + " columns, found " +
                      std::to_string(l.tok.size()));
}

}  // namespace

ForceField parse_force_field(std::string_view text, bool lg) {
  ForceField ff;
  Reader rd(text);
  // header (src/io/ffield_parser.cpp:100-115): the first non-blank line is a comment, and is rejected when it looks
  // like the "N ! Number of general parameters" line (a file whose comment line is missing)
  {
    auto first = rd.line();
    if (!first) throw FfieldError("empty force-field file");
    const auto& w = first->tok;
    bool digits = !w.empty() && !w[0].empty();
    for (char c : w[0]) digits = digits && c >= '0' && c <= '9';
    std::string joined;
    for (const auto& x : w) joined += x + " ";
    if (digits && w.size() >= 2 && !w[1].empty() && w[1][0] == '!' && joined.find("general parameters") != std::string::npos)
      throw FfieldError("line " + std::to_string(first->lineno) + ": first line of ReaxFF potential file must be a comment or empty");
  }
  // general parameters (src/io/ffield_parser.cpp:118-129: at least 38). A file with 38 has no p_coa3 (gp[38]); the
  // device copy of the list is zero-padded, so the coalition term then reads 0 there.
  {
    Line v = rd.values();
    const int n = inum(v, 0);
    if (n < 1) throw FfieldError("line " + std::to_string(v.lineno) + ": invalid number of global parameters");
    if (n < 38) throw FfieldError("the force field has only " + std::to_string(n) + " general parameters (>= 38 required)");
    ff.gp.resize(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) ff.gp[static_cast<size_t>(i)] = num(rd.values(), 0);
  }
  const int nt = inum(rd.values(), 0);
  if (nt < 1) throw FfieldError("invalid number of atom types");
  rd.skip(); rd.skip(); rd.skip();
  ff.nt = nt;
  ff.sb.assign(static_cast<size_t>(nt) * SB_NFIELDS, 0.0);
  ff.tb.assign(static_cast<size_t>(nt) * nt * TB_NFIELDS, 0.0);
  auto S = [&](int t, int f) -> double& { return ff.sb[static_cast<size_t>(t) * SB_NFIELDS + f]; };
  auto T = [&](int a, int b, int f) -> double& { return ff.tb[(static_cast<size_t>(a) * nt + b) * TB_NFIELDS + f]; };
  auto T2 = [&](int a, int b, int f, double v) { T(a, b, f) = v; T(b, a, f) = v; };
  for (int i = 0; i < nt; ++i) {
    Line v = rd.values();
    if (v.tok.size() < 8 && !lg) throw FfieldError("this force field file requires using 'lgvdw yes'");
    need(v, 9);
    std::string nm;
    for (char c : v.tok[0]) {
      if (nm.size() == 3) break;
      nm.push_back(static_cast<char>(toupper(static_cast<unsigned char>(c))));
    }
    ff.names.push_back(nm);
    const int l1[8] = {SB_R_S, SB_VALENCY, SB_MASS, SB_R_VDW, SB_EPSILON, SB_GAMMA, SB_R_PI, SB_VALENCY_E};
    for (int k = 0; k < 8; ++k) S(i, l1[k]) = num(v, static_cast<size_t>(1 + k));
    S(i, SB_NLP_OPT) = 0.5 * (S(i, SB_VALENCY_E) - S(i, SB_VALENCY));
    v = rd.values();
    need(v, 8);
    S(i, SB_ALPHA) = num(v, 0); S(i, SB_GAMMA_W) = num(v, 1); S(i, SB_VALENCY_BOC) = num(v, 2); S(i, SB_P_OVUN5) = num(v, 3);
    S(i, SB_CHI) = num(v, 5); S(i, SB_ETA) = 2.0 * num(v, 6); S(i, SB_P_HBOND) = static_cast<double>(static_cast<int>(num(v, 7)));
    v = rd.values();
    need(v, 8);
    S(i, SB_R_PI_PI) = num(v, 0); S(i, SB_P_LP2) = num(v, 1); S(i, SB_B_O_131) = num(v, 3); S(i, SB_B_O_132) = num(v, 4);
    S(i, SB_B_O_133) = num(v, 5); S(i, SB_BCUT_ACKS2) = num(v, 6);
    v = rd.values();
    need(v, 8);
    S(i, SB_P_OVUN2) = num(v, 0); S(i, SB_P_VAL3) = num(v, 1); S(i, SB_VALENCY_VAL) = num(v, 3); S(i, SB_P_VAL5) = num(v, 4);
    S(i, SB_RCORE2) = num(v, 5); S(i, SB_ECORE2) = num(v, 6); S(i, SB_ACORE2) = num(v, 7);
    if (lg) {
      v = rd.values();
      need(v, 2);
      S(i, SB_LGCIJ) = num(v, 0); S(i, SB_LGRE) = num(v, 1);
    }
    const bool inner = S(i, SB_RCORE2) > 0.01 && S(i, SB_ACORE2) > 0.01;
    const bool shield = S(i, SB_GAMMA_W) > 0.5;
    if (!inner && !shield) throw FfieldError("inconsistent van der Waals parameters: no shielding or inner wall for element " + nm);
    const int want = inner ? (shield ? 3 : 2) : 1;
    if (ff.vdw_type == 0) ff.vdw_type = want;
    else if (ff.vdw_type != want) ff.warnings.push_back("element " + nm + " indicates another van der Waals method; keeping the earlier one");
  }
  for (int i = 0; i < nt; ++i) {
    const double mass = S(i, SB_MASS);
    S(i, SB_HEAVY) = mass > 21.0 ? 1.0 : 0.0;
    S(i, SB_C2SPECIES) = ff.names[static_cast<size_t>(i)] == "C" ? 1.0 : 0.0;
    if (mass < 21 && S(i, SB_VALENCY_VAL) != S(i, SB_VALENCY_BOC)) {
      ff.warnings.push_back("Changed valency_val to valency_boc for " + ff.names[static_cast<size_t>(i)]);
      S(i, SB_VALENCY_VAL) = S(i, SB_VALENCY_BOC);
    }
  }
  // bond blocks
  {
    const int nb = inum(rd.values(), 0);
    rd.skip();
    for (int b = 0; b < nb; ++b) {
      Line v = rd.values();
      need(v, 10);
      const int j = inum(v, 0) - 1, k = inum(v, 1) - 1;
      if (j < 0 || k < 0) throw FfieldError("inconsistent force field file");
      Line w = rd.values();
      need(w, 7);
      if (j < nt && k < nt) {
        const int f1[8] = {TB_DE_S, TB_DE_P, TB_DE_PP, TB_P_BE1, TB_P_BO5, TB_V13COR, TB_P_BO6, TB_P_OVUN1};
        for (int q = 0; q < 8; ++q) T2(j, k, f1[q], num(v, static_cast<size_t>(2 + q)));
        T2(j, k, TB_P_BE2, num(w, 0)); T2(j, k, TB_P_BO3, num(w, 1)); T2(j, k, TB_P_BO4, num(w, 2));
        T2(j, k, TB_P_BO1, num(w, 4)); T2(j, k, TB_P_BO2, num(w, 5));
        T2(j, k, TB_OVC, w.tok.size() > 6 ? num(w, 6) : 0.0);
        T2(j, k, TB_LISTED, 1.0);
      }
    }
  }
  // mixing rules
  for (int i = 0; i < nt; ++i)
    for (int j = i; j < nt; ++j) {
      T2(i, j, TB_R_S, 0.5 * (S(j, SB_R_S) + S(i, SB_R_S)));
      T2(i, j, TB_R_P, 0.5 * (S(j, SB_R_PI) + S(i, SB_R_PI)));
      T2(i, j, TB_R_PP, 0.5 * (S(j, SB_R_PI_PI) + S(i, SB_R_PI_PI)));
      T2(i, j, TB_P_BOC3, std::sqrt(S(j, SB_B_O_132) * S(i, SB_B_O_132)));
      T2(i, j, TB_P_BOC4, std::sqrt(S(j, SB_B_O_131) * S(i, SB_B_O_131)));
      T2(i, j, TB_P_BOC5, std::sqrt(S(j, SB_B_O_133) * S(i, SB_B_O_133)));
      T2(i, j, TB_D, std::sqrt(S(j, SB_EPSILON) * S(i, SB_EPSILON)));
      T2(i, j, TB_ALPHA, std::sqrt(S(j, SB_ALPHA) * S(i, SB_ALPHA)));
      T2(i, j, TB_R_VDW, 2.0 * std::sqrt(S(j, SB_R_VDW) * S(i, SB_R_VDW)));
      T2(i, j, TB_GAMMA_W, std::sqrt(S(j, SB_GAMMA_W) * S(i, SB_GAMMA_W)));
      T2(i, j, TB_GAMMA, std::pow(S(j, SB_GAMMA) * S(i, SB_GAMMA), -1.5));
      T2(i, j, TB_RCORE, std::sqrt(S(i, SB_RCORE2) * S(j, SB_RCORE2)));
      T2(i, j, TB_ECORE, std::sqrt(S(i, SB_ECORE2) * S(j, SB_ECORE2)));
      T2(i, j, TB_ACORE, std::sqrt(S(i, SB_ACORE2) * S(j, SB_ACORE2)));
      T2(i, j, TB_LGCIJ, std::sqrt(S(i, SB_LGCIJ) * S(j, SB_LGCIJ)));
      T2(i, j, TB_LGRE, 2.0 * ff.gp[35] * std::sqrt(S(i, SB_LGRE) * S(j, SB_LGRE)));
    }
  // off-diagonal overrides
  {
    const int no = inum(rd.values(), 0);
    for (int o = 0; o < no; ++o) {
      Line v = rd.values();
      need(v, static_cast<size_t>(8 + (lg ? 1 : 0)));
      const int j = inum(v, 0) - 1, k = inum(v, 1) - 1;
      if (j < 0 || k < 0) throw FfieldError("inconsistent force field file");
      if (j < nt && k < nt) {
        const int fld[6] = {TB_D, TB_R_VDW, TB_ALPHA, TB_R_S, TB_R_P, TB_R_PP};
        const double scale[6] = {1.0, 2.0, 1.0, 1.0, 1.0, 1.0};
        for (int q = 0; q < 6; ++q) {
          const double val = num(v, static_cast<size_t>(2 + q));
          if (val > 0.0) T2(j, k, fld[q], scale[q] * val);
        }
        if (lg) {
          const double val = num(v, 8);
          if (val >= 0.0) T2(j, k, TB_LGCIJ, val);
        }
      }
    }
  }
  const size_t n3 = static_cast<size_t>(nt) * nt * nt;
  ff.thb_n.assign(n3, 0);
  ff.thb.assign(n3 * kMaxThbSets * TH_NFIELDS, 0.0);
  ff.hb_on.assign(n3, 0);
  ff.hb.assign(n3 * HB_NFIELDS, 0.0);
  ff.fb_on.assign(n3 * static_cast<size_t>(nt), 0);
  ff.fb.assign(n3 * static_cast<size_t>(nt) * FB_NFIELDS, 0.0);
  auto k3 = [&](int a, int b, int c) { return (static_cast<size_t>(a) * nt + b) * nt + c; };
  // valence-angle sets
  {
    const int na = inum(rd.values(), 0);
    std::vector<int> slots(n3, 0);
    for (int q = 0; q < na; ++q) {
      Line v = rd.values();
      need(v, 10);
      const int j = inum(v, 0) - 1, k = inum(v, 1) - 1, l = inum(v, 2) - 1;
      if (j < 0 || k < 0 || l < 0) throw FfieldError("inconsistent force field file");
      if (j < nt && k < nt && l < nt) {
        double set[TH_NFIELDS];
        set[TH_THETA_00] = num(v, 3); set[TH_P_VAL1] = num(v, 4); set[TH_P_VAL2] = num(v, 5); set[TH_P_COA1] = num(v, 6);
        set[TH_P_VAL7] = num(v, 7); set[TH_P_PEN1] = num(v, 8); set[TH_P_VAL4] = num(v, 9);
        slots[k3(j, k, l)] += 1;
        slots[k3(l, k, j)] += 1;
        if (slots[k3(j, k, l)] > kMaxThbSets || slots[k3(l, k, j)] > kMaxThbSets)
          throw FfieldError("too many valence-angle parameter sets for one triple (at most 2 for j==l, 5 otherwise)");
        auto push = [&](size_t key) {
          const int idx = ff.thb_n[key]++;
          for (int f = 0; f < TH_NFIELDS; ++f) ff.thb[(key * kMaxThbSets + static_cast<size_t>(idx)) * TH_NFIELDS + f] = set[f];
        };
        push(k3(j, k, l));
        if (j != l) push(k3(l, k, j));
      }
    }
  }
  // torsions
  {
    const int n4 = inum(rd.values(), 0);
    std::set<std::array<int, 4>> expl;
    auto put = [&](int a, int b, int c, int d, const double* v) {
      const size_t key = k3(a, b, c) * static_cast<size_t>(nt) + static_cast<size_t>(d);
      ff.fb_on[key] = 1;
      for (int f = 0; f < FB_NFIELDS; ++f) ff.fb[key * FB_NFIELDS + f] = v[f];
    };
    for (int q = 0; q < n4; ++q) {
      Line v = rd.values();
      need(v, 9);
      const int j = inum(v, 0) - 1, k = inum(v, 1) - 1, l = inum(v, 2) - 1, m = inum(v, 3) - 1;
      if (j < -1 || k < 0 || l < 0 || m < -1) throw FfieldError("inconsistent force field file");
      double p[FB_NFIELDS];
      for (int f = 0; f < FB_NFIELDS; ++f) p[f] = num(v, static_cast<size_t>(4 + f));
      if (j >= 0 && m >= 0) {
        if (j < nt && k < nt && l < nt && m < nt) {
          expl.insert({j, k, l, m});
          expl.insert({m, l, k, j});
          put(j, k, l, m, p);
          put(m, l, k, j, p);
        }
      } else if (k < nt && l < nt) {
        for (int a = 0; a < nt; ++a)
          for (int o = 0; o < nt; ++o) {
            if (!expl.count({a, k, l, o})) put(a, k, l, o, p);
            if (!expl.count({o, l, k, a})) put(o, l, k, a, p);
          }
      }
    }
  }
  // hydrogen bonds (the whole block may be absent)
  if (auto first = rd.line()) {
    const int nh = inum(*first, 0);
    for (int q = 0; q < nh; ++q) {
      Line v = rd.values();
      need(v, 7);
      const int j = inum(v, 0) - 1, k = inum(v, 1) - 1, l = inum(v, 2) - 1;
      if (j < 0 || k < 0 || l < 0) throw FfieldError("inconsistent force field file");
      if (j < nt && k < nt && l < nt) {
        const size_t key = k3(j, k, l);
        ff.hb_on[key] = 1;
        for (int f = 0; f < HB_NFIELDS; ++f) ff.hb[key * HB_NFIELDS + f] = num(v, static_cast<size_t>(3 + f));
      }
    }
  } else {
    ff.warnings.push_back("the force field has no hydrogen-bond parameters");
  }
  ff.bo_cut = 0.01 * ff.gp[29];
  ff.nonb_low = ff.gp[11];
  ff.nonb_cut = ff.gp[12];
  const double g37 = ff.gp[37];
  const bool gp37 = (g37 > -2147483649.0 && g37 < 2147483648.0) && static_cast<double>(static_cast<int>(g37)) == 2;
  for (int i = 0; i < nt; ++i)
    for (int j = 0; j < nt; ++j) {
      const double mi = S(i, SB_MASS), mj = S(j, SB_MASS);
      T(i, j, TB_TRIPLE_STAB) = (gp37 || (mi == 12.0000 && mj == 15.9990) || (mj == 12.0000 && mi == 15.9990)) ? 1.0 : 0.0;
    }
  return ff;
}

namespace {
void put(std::string& o, double v) {
  char b[40];
  std::snprintf(b, sizeof b, " %.17g", v);
  o += b;
}
}  // namespace

std::string ForceField::canonical_dump(bool portable) const {
  std::string o = "FFIELD-TABLES 1\n";
  o += "GP " + std::to_string(gp.size()) + " " + std::to_string(vdw_type) + "\n";
  for (size_t i = 0; i < gp.size(); ++i) {
    o += "G " + std::to_string(i);
    put(o, gp[i]);
    o += "\n";
  }
  for (int i = 0; i < nt; ++i) {
    o += "S " + std::to_string(i) + " " + names[static_cast<size_t>(i)];
    for (int f : {SB_R_S, SB_VALENCY, SB_MASS, SB_R_VDW, SB_EPSILON, SB_GAMMA, SB_R_PI, SB_VALENCY_E, SB_NLP_OPT, SB_ALPHA, SB_GAMMA_W,
                  SB_VALENCY_BOC, SB_P_OVUN5})
      put(o, s(i, f));
    o += " " + std::to_string(static_cast<int>(s(i, SB_P_HBOND)));
    for (int f : {SB_CHI, SB_ETA, SB_R_PI_PI, SB_P_LP2, SB_B_O_131, SB_B_O_132, SB_B_O_133, SB_BCUT_ACKS2, SB_P_OVUN2, SB_P_VAL3,
                  SB_VALENCY_VAL, SB_P_VAL5, SB_RCORE2, SB_ECORE2, SB_ACORE2, SB_LGCIJ, SB_LGRE})
      put(o, s(i, f));
    o += "\n";
  }
  for (int i = 0; i < nt; ++i)
    for (int j = i; j < nt; ++j) {
      o += "T " + std::to_string(i) + " " + std::to_string(j);
      for (int f : {TB_P_BO1, TB_P_BO2, TB_P_BO3, TB_P_BO4, TB_P_BO5, TB_P_BO6, TB_R_S, TB_R_P, TB_R_PP, TB_P_BOC3, TB_P_BOC4, TB_P_BOC5,
                    TB_P_BE1, TB_P_BE2, TB_DE_S, TB_DE_P, TB_DE_PP, TB_P_OVUN1, TB_D, TB_ALPHA, TB_R_VDW, TB_GAMMA_W, TB_RCORE, TB_ECORE,
                    TB_ACORE, TB_LGCIJ, TB_LGRE})
        put(o, p(i, j, f));
      if (!portable) put(o, p(i, j, TB_GAMMA));
      put(o, p(i, j, TB_V13COR));
      put(o, p(i, j, TB_OVC));
      o += "\n";
    }
  const size_t n = static_cast<size_t>(nt);
  for (size_t j = 0; j < n; ++j)
    for (size_t k = 0; k < n; ++k)
      for (size_t l = 0; l < n; ++l) {
        const size_t key = (j * n + k) * n + l;
        if (thb_n[key] == 0) continue;
        o += "H3 " + std::to_string(j) + " " + std::to_string(k) + " " + std::to_string(l) + " " + std::to_string(thb_n[key]);
        for (int q = 0; q < thb_n[key]; ++q)
          for (int f = 0; f < TH_NFIELDS; ++f) put(o, thb[(key * kMaxThbSets + static_cast<size_t>(q)) * TH_NFIELDS + f]);
        o += "\n";
      }
  for (size_t j = 0; j < n; ++j)
    for (size_t k = 0; k < n; ++k)
      for (size_t l = 0; l < n; ++l)
        for (size_t m = 0; m < n; ++m) {
          const size_t key = ((j * n + k) * n + l) * n + m;
          if (!fb_on[key]) continue;
          o += "H4 " + std::to_string(j) + " " + std::to_string(k) + " " + std::to_string(l) + " " + std::to_string(m);
          for (int f = 0; f < FB_NFIELDS; ++f) put(o, fb[key * FB_NFIELDS + f]);
          o += "\n";
        }
  for (size_t j = 0; j < n; ++j)
    for (size_t k = 0; k < n; ++k)
      for (size_t l = 0; l < n; ++l) {
        const size_t key = (j * n + k) * n + l;
        if (!hb_on[key]) continue;
        const double* h = &hb[key * HB_NFIELDS];
        if (h[0] == -1.0 && h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0) continue;
        o += "HB " + std::to_string(j) + " " + std::to_string(k) + " " + std::to_string(l);
        for (int f = 0; f < HB_NFIELDS; ++f) put(o, h[f]);
        o += "\n";
      }
  return o;
}

}  // namespace rx
