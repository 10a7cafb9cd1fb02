// ReaxFF parameter-file reader of the CUDA engine and the flat parameter tables it uploads to the device.
//
// Behaviour follows the reference's strict reader (src/io/ffield_parser.cpp:91-451, include/reaxmetal/forcefield.hpp):
// fixed column positions, eta stored as twice the file value, the light-element valency override (:233-240), the
// system-wide vdW type rule (:207-231), the pair mixing rules (:284-306), off-diagonal overrides (:308-333), valence
// angle sets mirrored into (l, k, j) with the five-slot bound (:335-368), torsions with the 0-X-Y-0 wildcard form and
// its order-dependent overwrite (:370-401), an optional H-bond block (:403-426) and the derived control values
// (bo_cut = 0.01 gp[29], taper radii gp[11]/gp[12], :436-449).
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace rx {

struct FfieldError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// per-type fields (doubles)
enum SbField {
  SB_R_S, SB_VALENCY, SB_MASS, SB_R_VDW, SB_EPSILON, SB_GAMMA, SB_R_PI, SB_VALENCY_E, SB_NLP_OPT, SB_ALPHA, SB_GAMMA_W,
  SB_VALENCY_BOC, SB_P_OVUN5, SB_CHI, SB_ETA, SB_P_HBOND, SB_R_PI_PI, SB_P_LP2, SB_B_O_131, SB_B_O_132, SB_B_O_133,
  SB_BCUT_ACKS2, SB_P_OVUN2, SB_P_VAL3, SB_VALENCY_VAL, SB_P_VAL5, SB_RCORE2, SB_ECORE2, SB_ACORE2, SB_LGCIJ, SB_LGRE,
  SB_HEAVY, SB_C2SPECIES, SB_NFIELDS
};
// per-pair fields (symmetric nt x nt)
enum TbField {
  TB_P_BO1, TB_P_BO2, TB_P_BO3, TB_P_BO4, TB_P_BO5, TB_P_BO6, TB_R_S, TB_R_P, TB_R_PP, TB_P_BOC3, TB_P_BOC4, TB_P_BOC5,
  TB_P_BE1, TB_P_BE2, TB_DE_S, TB_DE_P, TB_DE_PP, TB_P_OVUN1, TB_D, TB_ALPHA, TB_R_VDW, TB_GAMMA_W, TB_RCORE, TB_ECORE,
  TB_ACORE, TB_LGCIJ, TB_LGRE, TB_GAMMA, TB_V13COR, TB_OVC, TB_TRIPLE_STAB, TB_LISTED, TB_NFIELDS
};
enum ThField { TH_THETA_00, TH_P_VAL1, TH_P_VAL2, TH_P_VAL4, TH_P_VAL7, TH_P_PEN1, TH_P_COA1, TH_NFIELDS };
enum FbField { FB_V1, FB_V2, FB_V3, FB_P_TOR1, FB_P_COT1, FB_NFIELDS };
enum HbField { HB_R0, HB_P_HB1, HB_P_HB2, HB_P_HB3, HB_NFIELDS };
constexpr int kMaxThbSets = 5;

struct ForceField {
  int nt = 0;
  std::vector<double> gp;
  int vdw_type = 0;
  double bo_cut = 0, nonb_low = 0, nonb_cut = 0;
  std::vector<std::string> names;
  std::vector<double> sb;    // nt * SB_NFIELDS
  std::vector<double> tb;    // nt * nt * TB_NFIELDS
  std::vector<int> thb_n;    // nt^3
  std::vector<double> thb;   // nt^3 * kMaxThbSets * TH_NFIELDS
  std::vector<int> fb_on;    // nt^4
  std::vector<double> fb;    // nt^4 * FB_NFIELDS
  std::vector<int> hb_on;    // nt^3
  std::vector<double> hb;    // nt^3 * HB_NFIELDS
  std::vector<std::string> warnings;

  double s(int t, int f) const { return sb[static_cast<size_t>(t) * SB_NFIELDS + f]; }
  double p(int a, int b, int f) const { return tb[(static_cast<size_t>(a) * nt + b) * TB_NFIELDS + f]; }
  // Canonical table dump in the reference's "%.17g" format (src/io/table_dump.cpp:20-84), for byte-wise comparison.
  std::string canonical_dump(bool portable) const;
};

ForceField parse_force_field(std::string_view text, bool lgvdw = false);

}  // namespace rx
