// Bond orders and every bond-order term of the hot path, FP64 on the device.
//
// Order of the launches (one MD force evaluation):
//   k_bonds            bond list + uncorrected bond orders BO' and their derivatives (src/cpu/bonded.cpp:107-162)
//   k_bond_sym         index of the reverse slot of every bond
//   k_bo_correct       corrected bond orders + the 11 C*dbo coefficients (terms.hpp:66-132)
//   k_atom_quantities  Delta, Delta_e, nlp, ... of every atom (terms.hpp:141-164)
//   k_bonded_atom      per centre atom: bond energy, lone pair, C2, over/under, valence/penalty/coalition, H-bonds
//   k_torsion          torsion + 4-body conjugation per central bond
//   k_fold             torsion contributions to second neighbors + CdDelta totals
//   k_dbond            Add_dBond_to_Forces, own part (src/cpu/bonded.cpp:717-766)
//   k_force_final      gather of every contribution written for this atom by its bond partners
// Each kernel writes only the atom's own data and the bond slots it owns, so the whole chain is atomic-free.
#include "device.cuh"
#include "kernels.hpp"

namespace rx {

namespace {
constexpr double kConstPi = 3.14159265;   // reaxff_defs.h constPI (src/cpu/bonded.cpp:52)
constexpr double kHbThreshold = 1e-2;     // HB_THRESHOLD
constexpr double kMinSine = 1e-10;        // MIN_SINE

__device__ inline const double* SBp(const DevFF& ff, int t) { return ff.sb + static_cast<size_t>(t) * SB_N; }
__device__ inline const double* TBp(const DevFF& ff, int a, int b) { return ff.tb + (static_cast<size_t>(a) * ff.nt + b) * TB_N; }

__device__ inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// reaxff_valence_angles.cpp:36-70 (restated in src/cpu/bonded.cpp:58-75)
__device__ inline void calc_theta(const double* dji, double d_ji, const double* djk, double d_jk, double& theta, double& cos_theta) {
  double c = dot3(dji, djk) / (d_ji * d_jk);
  if (c > 1.0) c = 1.0;
  if (c < -1.0) c = -1.0;
  cos_theta = c;
  theta = acos(c);
}
__device__ inline void calc_dcos(const double* dji, double d_ji, const double* djk, double d_jk, double* di, double* dj, double* dk) {
  const double sq_ji = d_ji * d_ji, sq_jk = d_jk * d_jk;
  const double inv = 1.0 / (d_ji * d_jk);
  const double inv3 = inv * inv * inv;
  const double Cdot = dot3(dji, djk) * inv3;
  for (int t = 0; t < 3; ++t) {
    di[t] = djk[t] * inv - Cdot * sq_jk * dji[t];
    dj[t] = -(djk[t] + dji[t]) * inv + Cdot * (sq_jk * dji[t] + sq_ji * djk[t]);
    dk[t] = dji[t] * inv - Cdot * sq_ji * djk[t];
  }
}

// tag-order choice of the end that evaluates a bond term (src/cpu/bonded.cpp:226-232, :487-493): true = skip here.
// For an image of the atom itself the reference compares coordinates (x_j < x_i on z, then y, then x); x_j - x_i is
// the bond vector, so the same test reads its components.
__device__ inline bool skip_by_tag(const Dev& d, int i, int j, const double4& dv) {
  const long long ti = d.tag[i], tj = d.tag[j];
  if (ti > tj) return true;
  if (ti == tj) {
    if (dv.z < 0.0) return true;
    if (dv.z == 0.0 && dv.y < 0.0) return true;
    if (dv.z == 0.0 && dv.y == 0.0 && dv.x < 0.0) return true;
  }
  return false;
}

__device__ inline void add3(double4& a, double s, const double* v) { a.x += s * v[0]; a.y += s * v[1]; a.z += s * v[2]; }
}  // namespace

// ------------------------------------------------------------------------------------------------ bond list
// One warp per atom over its neighbor row: entries within bond_cut whose uncorrected bond order passes bo_cut
// (terms::bo_prime, terms.hpp:50-56; gate src/cpu/bonded.cpp:130) become bond slots, in row order.
__global__ void k_bonds(Dev d, DevFF ff, DevCtl ctl) {
  if (lists_failed(d)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  const int i = warp;
  const SysInfo s = d.sys[d.sys_of[i]];
  const int ti = d.type[i];
  const double* si = SBp(ff, ti);
  const int cnt = min(d.near_cnt[i], d.ncap_near);
  const unsigned lt = (1u << lane) - 1u;
  const double bo_cut = ff.bo_cut;
  int nb = 0;
  double tbo = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int base = 0; base < cnt; base += 32) {
    const int e = base + lane;
    bool isb = false;
    unsigned code = 0;
    double dv[3] = {0, 0, 0}, dd = 0, BOt = 0, BO_s = 0, BO_pi = 0, BO_pi2 = 0, C12 = 0, C34 = 0, C56 = 0;
    const double* tb = nullptr;
    if (e < cnt) {
      code = d.near[static_cast<size_t>(i) * d.ncap_near + e];
      const int j = static_cast<int>(code & d.amask);
      const int sidx = static_cast<int>(code >> d.abits);
      pair_dvec(d, s, i, j, sidx, dv);
      const double r2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
      dd = sqrt(r2);
      const int tj = d.type[j];
      if (dd <= ctl.bond_cut && r2 <= ff.rbo2[ti * ff.nt + tj]) {
        const double* sj = SBp(ff, tj);
        tb = TBp(ff, ti, tj);
        if (si[SB_R_S] > 0.0 && sj[SB_R_S] > 0.0) { C12 = tb[TB_P_BO1] * pow(dd / tb[TB_R_S], tb[TB_P_BO2]); BO_s = (1.0 + bo_cut) * exp(C12); }
        if (si[SB_R_PI] > 0.0 && sj[SB_R_PI] > 0.0) { C34 = tb[TB_P_BO3] * pow(dd / tb[TB_R_P], tb[TB_P_BO4]); BO_pi = exp(C34); }
        if (si[SB_R_PI_PI] > 0.0 && sj[SB_R_PI_PI] > 0.0) { C56 = tb[TB_P_BO5] * pow(dd / tb[TB_R_PP], tb[TB_P_BO6]); BO_pi2 = exp(C56); }
        BOt = BO_s + BO_pi + BO_pi2;
        isb = BOt >= bo_cut;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, isb);
    if (isb) {
      const int pos = nb + __popc(m & lt);
      const double rr2 = 1.0 / (dd * dd);
      const double Cln_s = tb[TB_P_BO2] * C12 * rr2, Cln_pi = tb[TB_P_BO4] * C34 * rr2, Cln_pi2 = tb[TB_P_BO6] * C56 * rr2;
      const double cb = -(BO_s * Cln_s + BO_pi * Cln_pi + BO_pi2 * Cln_pi2);
      const double dB[3] = {cb * dv[0], cb * dv[1], cb * dv[2]};
      if (pos < d.bcap) {
        const size_t b = static_cast<size_t>(i) * d.bcap + pos;
        d.bcode[b] = code;
        d.bdv[b] = make_double4(dv[0], dv[1], dv[2], dd);
        d.bBO[b] = make_double4(BOt - bo_cut, BO_s - bo_cut, BO_pi, BO_pi2);
        d.bdBOp[b] = make_double4(dB[0], dB[1], dB[2], 0.0);
        d.bdlnpi[b] = make_double4(-BO_pi * Cln_pi * dv[0], -BO_pi * Cln_pi * dv[1], -BO_pi * Cln_pi * dv[2], 0.0);
        d.bdlnpi2[b] = make_double4(-BO_pi2 * Cln_pi2 * dv[0], -BO_pi2 * Cln_pi2 * dv[1], -BO_pi2 * Cln_pi2 * dv[2], 0.0);
      }
      tbo += BOt - bo_cut;
      g0 += dB[0]; g1 += dB[1]; g2 += dB[2];
    }
    nb += __popc(m);
  }
  tbo = warp_sum(tbo); g0 = warp_sum(g0); g1 = warp_sum(g1); g2 = warp_sum(g2);
  if (lane == 0) {
    d.bcnt[i] = nb;
    if (nb > d.bcap) {
      atomicOr(d.status, ST_BOND_OVERFLOW);
      atomicMax(d.status + 2, nb);
    }
    d.Deltap[i] = tbo - si[SB_VALENCY];
    d.Deltap_boc[i] = tbo - si[SB_VALENCY_VAL];
    d.dDp_self[i] = make_double4(g0, g1, g2, 0.0);
  }
}

__global__ void k_bond_sym(Dev d) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *d.tor_n = 0;   // the central bonds of this evaluation's torsions (k_bo_correct)
  if (lists_failed(d)) return;
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long long>(d.na) * d.bcap) return;
  const int a = static_cast<int>(t / d.bcap), k = static_cast<int>(t % d.bcap);
  if (k >= min(d.bcnt[a], d.bcap)) return;
  const unsigned code = d.bcode[t];
  const int j = static_cast<int>(code & d.amask);
  const unsigned sidx = code >> d.abits;
  const unsigned want = static_cast<unsigned>(a) | ((static_cast<unsigned>(d.S * d.S * d.S - 1) - sidx) << d.abits);
  const int nj = min(d.bcnt[j], d.bcap);
  int found = -1;
  for (int q = 0; q < nj; ++q)
    if (d.bcode[static_cast<size_t>(j) * d.bcap + q] == want) { found = j * d.bcap + q; break; }
  if (found < 0) {
    atomicOr(d.status, ST_SYM_MISSING);
    found = static_cast<int>(t);
  }
  d.bsym[t] = found;
}

// terms::bo_correct (include/reaxmetal/terms.hpp:66-132) for every slot, the slot's atom as "i". The corrected bond
// orders are symmetric in (i, j) bit for bit, so both slots of a bond hold the same values.
__global__ void k_bo_correct(Dev d, DevFF ff, DevCtl ctl) {
  if (lists_failed(d)) return;
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long long>(d.na) * d.bcap) return;
  const int a = static_cast<int>(t / d.bcap), k = static_cast<int>(t % d.bcap);
  if (k >= min(d.bcnt[a], d.bcap)) return;
  const int j = static_cast<int>(d.bcode[t] & d.amask);
  const int ti = d.type[a], tj = d.type[j];
  const double* tb = TBp(ff, ti, tj);
  const double p_boc1 = ff.gp[0], p_boc2 = ff.gp[1];
  const double val_i = SBp(ff, ti)[SB_VALENCY], val_j = SBp(ff, tj)[SB_VALENCY];
  const double Deltap_i = d.Deltap[a], Deltap_j = d.Deltap[j], Dboc_i = d.Deltap_boc[a], Dboc_j = d.Deltap_boc[j];
  const double4 bo = d.bBO[t];
  const double BO = bo.x, BO_s = bo.y, BO_pi = bo.z, BO_pi2 = bo.w;
  double oBO, oBO_s, oBO_pi, oBO_pi2;
  double C1dbo, C2dbo = 0, C3dbo = 0, C1dbopi, C2dbopi = 0, C3dbopi = 0, C4dbopi = 0, C1dbopi2, C2dbopi2 = 0, C3dbopi2 = 0, C4dbopi2 = 0;
  const double ovc = tb[TB_OVC], v13cor = tb[TB_V13COR];
  if (ovc < 0.001 && v13cor < 0.001) {
    oBO = BO; oBO_s = BO_s; oBO_pi = BO_pi; oBO_pi2 = BO_pi2;
    C1dbo = 1.0; C1dbopi = 1.0; C1dbopi2 = 1.0;
  } else {
    double f1, Cf1_ij, Cf1_ji, f4, f5, f4f5, Cf45_ij, Cf45_ji;
    if (ovc >= 0.001) {
      const double exp_p1i = safe_exp(-p_boc1 * Deltap_i), exp_p2i = safe_exp(-p_boc2 * Deltap_i);
      const double exp_p1j = safe_exp(-p_boc1 * Deltap_j), exp_p2j = safe_exp(-p_boc2 * Deltap_j);
      const double f2 = exp_p1i + exp_p1j;
      const double f3 = -1.0 / p_boc2 * log(0.5 * (exp_p2i + exp_p2j));
      f1 = 0.5 * ((val_i + f2) / (val_i + f2 + f3) + (val_j + f2) / (val_j + f2 + f3));
      const double temp = f2 + f3;
      const double u1_ij = val_i + temp, u1_ji = val_j + temp;
      const double Cf1A_ij = 0.5 * f3 * (1.0 / (u1_ij * u1_ij) + 1.0 / (u1_ji * u1_ji));
      const double Cf1B_ij = -0.5 * ((u1_ij - f3) / (u1_ij * u1_ij) + (u1_ji - f3) / (u1_ji * u1_ji));
      Cf1_ij = 0.50 * (-p_boc1 * exp_p1i / u1_ij - ((val_i + f2) / (u1_ij * u1_ij)) * (-p_boc1 * exp_p1i + exp_p2i / (exp_p2i + exp_p2j)) +
                       -p_boc1 * exp_p1i / u1_ji - ((val_j + f2) / (u1_ji * u1_ji)) * (-p_boc1 * exp_p1i + exp_p2i / (exp_p2i + exp_p2j)));
      Cf1_ji = -Cf1A_ij * p_boc1 * exp_p1j + Cf1B_ij * exp_p2j / (exp_p2i + exp_p2j);
    } else {
      f1 = 1.0; Cf1_ij = Cf1_ji = 0.0;
    }
    const double p_boc3 = tb[TB_P_BOC3], p_boc4 = tb[TB_P_BOC4], p_boc5 = tb[TB_P_BOC5];
    if (v13cor >= 0.001) {
      const double exp_f4 = safe_exp(-(p_boc4 * (BO * BO) - Dboc_i) * p_boc3 + p_boc5);
      const double exp_f5 = safe_exp(-(p_boc4 * (BO * BO) - Dboc_j) * p_boc3 + p_boc5);
      f4 = 1.0 / (1.0 + exp_f4);
      f5 = 1.0 / (1.0 + exp_f5);
      f4f5 = f4 * f5;
      Cf45_ij = -f4 * exp_f4;
      Cf45_ji = -f5 * exp_f5;
    } else {
      f4 = f5 = f4f5 = 1.0; Cf45_ij = Cf45_ji = 0.0;
    }
    const double A0 = f1 * f4f5;
    const double A1 = -2 * p_boc3 * p_boc4 * BO * (Cf45_ij + Cf45_ji);
    const double A2_ij = Cf1_ij / f1 + p_boc3 * Cf45_ij;
    const double A2_ji = Cf1_ji / f1 + p_boc3 * Cf45_ji;
    const double A3_ij = A2_ij + Cf1_ij / f1;
    const double A3_ji = A2_ji + Cf1_ji / f1;
    oBO = BO * A0;
    oBO_pi = BO_pi * A0 * f1;
    oBO_pi2 = BO_pi2 * A0 * f1;
    oBO_s = oBO - (oBO_pi + oBO_pi2);
    C1dbo = A0 + oBO * A1;
    C2dbo = oBO * A2_ij;
    C3dbo = oBO * A2_ji;
    C1dbopi = f1 * f1 * f4 * f5;
    C2dbopi = oBO_pi * A1;
    C3dbopi = oBO_pi * A3_ij;
    C4dbopi = oBO_pi * A3_ji;
    C1dbopi2 = f1 * f1 * f4 * f5;
    C2dbopi2 = oBO_pi2 * A1;
    C3dbopi2 = oBO_pi2 * A3_ij;
    C4dbopi2 = oBO_pi2 * A3_ji;
  }
  if (oBO < 1e-10) oBO = 0;
  if (oBO_s < 1e-10) oBO_s = 0;
  if (oBO_pi < 1e-10) oBO_pi = 0;
  if (oBO_pi2 < 1e-10) oBO_pi2 = 0;
  d.bBO[t] = make_double4(oBO, oBO_s, oBO_pi, oBO_pi2);
  {   // a central bond of the torsions (src/cpu/bonded.cpp:487-506): evaluated by the tag-order end, BO above thb_cut.
      // The slots are listed in any order (each writes only its own rows), so k_torsion runs dense warps.
    const bool central = oBO > ctl.thb_cut && !skip_by_tag(d, a, j, d.bdv[t]);
    d.tflag[t] = central ? 1 : 0;
    if (central) d.tor_list[atomicAdd(d.tor_n, 1)] = static_cast<int>(t);
  }
  d.bC0[t] = make_double4(C1dbo, C2dbo, C3dbo, C1dbopi);
  d.bC1[t] = make_double4(C2dbopi, C3dbopi, C4dbopi, C1dbopi2);
  d.bC2[t] = make_double4(C2dbopi2, C3dbopi2, C4dbopi2, 0.0);
}

__global__ void k_atom_quantities(Dev d, DevFF ff) {
  if (lists_failed(d)) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  const int t = d.type[a];
  const double* s = SBp(ff, t);
  const int nb = min(d.bcnt[a], d.bcap);
  double tbo = 0.0;
  for (int k = 0; k < nb; ++k) tbo += d.bBO[static_cast<size_t>(a) * d.bcap + k].x;
  const double p_lp1 = ff.gp[15];
  AtomQ q;
  q.total_bo = tbo;
  q.Delta = tbo - s[SB_VALENCY];
  q.Delta_e = tbo - s[SB_VALENCY_E];
  q.Delta_boc = tbo - s[SB_VALENCY_BOC];
  q.Delta_val = tbo - s[SB_VALENCY_VAL];
  const double half_trunc = static_cast<double>(static_cast<int>(q.Delta_e / 2.0));
  q.vlpex = q.Delta_e - 2.0 * half_trunc;
  const double explp1 = exp(-p_lp1 * ((2.0 + q.vlpex) * (2.0 + q.vlpex)));
  q.nlp = explp1 - half_trunc;
  q.Delta_lp = s[SB_NLP_OPT] - q.nlp;
  const double Clp = 2.0 * p_lp1 * explp1 * (2.0 + q.vlpex);
  q.dDelta_lp = Clp;
  if (s[SB_HEAVY] != 0.0) q.Delta_lp_temp = s[SB_NLP_OPT] - 0.5 * (s[SB_VALENCY_E] - s[SB_VALENCY]);
  else q.Delta_lp_temp = s[SB_NLP_OPT] - q.nlp;
  d.aq[a] = q;
  d.census[0 * d.na + a] = nb;
  d.census[6 * d.na + a] = static_cast<int>(q.Delta_e / 2.0);
}

// ------------------------------------------------------------------------------------------------ per-centre terms
// One thread per atom j: bond energy + triple-bond stabilisation (src/cpu/bonded.cpp:219-253), lone pair + C2
// (:255-281), over/under coordination (:282-318), valence angle + penalty + coalition centred at j (:321-474). Coefficients of j's own bonds go to j's slots; contributions to a bond partner
// (its CdDelta, its gradient) go to the slot naming it, for the partner to gather.
__global__ void k_bonded_atom(Dev d, DevFF ff, DevCtl ctl) {
  if (lists_failed(d)) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.na) return;
  const int tj = d.type[j];
  const double* sj = SBp(ff, tj);
  const int nb = min(d.bcnt[j], d.bcap);
  const size_t base = static_cast<size_t>(j) * d.bcap;
  const AtomQ aqj = d.aq[j];
  const double* gp = ff.gp;
  for (int k = 0; k < nb; ++k) {
    d.bacc[base + k] = make_double4(0, 0, 0, 0);
    d.bfn[base + k] = make_double4(0, 0, 0, 0);
  }
  double fj[3] = {0, 0, 0}, cdd = 0.0;
  double e_bond = 0, e_lp = 0, e_ov = 0, e_un = 0, e_ang = 0, e_pen = 0, e_coa = 0;
  double vir[kVir] = {0, 0, 0, 0, 0, 0};
  double pe_own = 0.0;   // per-atom tally of this atom (bond-energy and C2 halves of its partners go to them)

  // ---- bond energy (owned end chosen by tag order)
  {
    const double gp3 = gp[3], gp4 = gp[4], gp7 = gp[7], gp10 = gp[10];
    for (int k = 0; k < nb; ++k) {
      const size_t b = base + k;
      const int p = static_cast<int>(d.bcode[b] & d.amask);
      if (skip_by_tag(d, j, p, d.bdv[b])) continue;
      const double* tb = TBp(ff, tj, d.type[p]);
      const double4 bo = d.bBO[b];
      const double pow_BOs_be2 = bo.y == 0.0 ? 0.0 : pow(bo.y, tb[TB_P_BE2]);
      const double exp_be12 = exp(tb[TB_P_BE1] * (1.0 - pow_BOs_be2));
      const double CEbo = -tb[TB_DE_S] * exp_be12 * (1.0 - tb[TB_P_BE1] * tb[TB_P_BE2] * pow_BOs_be2);
      double eb = -tb[TB_DE_S] * bo.y * exp_be12 - tb[TB_DE_P] * bo.z - tb[TB_DE_PP] * bo.w;
      e_bond += eb;
      double4 acc = d.bacc[b];
      acc.x += CEbo;
      acc.y -= (CEbo + tb[TB_DE_P]);
      acc.z -= (CEbo + tb[TB_DE_PP]);
      if (bo.x >= 1.00 && tb[TB_TRIPLE_STAB] != 0.0) {
        const double BO = bo.x;
        const AtomQ aqp = d.aq[p];
        const double exphu = exp(-gp7 * ((BO - 2.50) * (BO - 2.50)));
        const double exphua1 = exp(-gp3 * (aqj.total_bo - BO));
        const double exphub1 = exp(-gp3 * (aqp.total_bo - BO));
        const double exphuov = exp(gp4 * (aqj.Delta + aqp.Delta));
        const double hulpov = 1.0 / (1.0 + 25.0 * exphuov);
        e_bond += gp10 * exphu * hulpov * (exphua1 + exphub1);
        eb += gp10 * exphu * hulpov * (exphua1 + exphub1);
        acc.x += gp10 * exphu * hulpov * (exphua1 + exphub1) * (gp3 - 2.0 * gp7 * (BO - 2.50));
        cdd += -gp10 * exphu * hulpov * (gp3 * exphua1 + 25.0 * gp4 * exphuov * hulpov * (exphua1 + exphub1));
        acc.w += -gp10 * exphu * hulpov * (gp3 * exphub1 + 25.0 * gp4 * exphuov * hulpov * (exphua1 + exphub1));
      }
      d.bacc[b] = acc;
      if (d.pe_on) {   // etally_half (src/cpu/bonded.cpp:239,246)
        pe_own += 0.5 * eb;
        pe_add(d, p, 0.5 * eb);
      }
    }
  }
  // ---- lone pair + C2 correction
  {
    if (nb > 0 || ctl.enobonds) {
      const double p_lp2 = sj[SB_P_LP2], Delta_lp = aqj.Delta_lp;
      const double expvd2 = safe_exp(-75 * Delta_lp);
      const double inv = 1.0 / (1.0 + expvd2);
      e_lp += p_lp2 * Delta_lp * inv;
      pe_own += p_lp2 * Delta_lp * inv;
      const double dElp = p_lp2 * inv + 75 * p_lp2 * Delta_lp * expvd2 * (inv * inv);
      cdd += dElp * aqj.dDelta_lp;
    }
    const double p_lp3 = gp[5];
    if (p_lp3 > 0.001 && sj[SB_C2SPECIES] != 0.0) {
      for (int k = 0; k < nb; ++k) {
        const size_t b = base + k;
        const int p = static_cast<int>(d.bcode[b] & d.amask);
        if (SBp(ff, d.type[p])[SB_C2SPECIES] == 0.0) continue;
        const double Di = aqj.Delta;
        const double vov3 = d.bBO[b].x - Di - 0.040 * pow(Di, 4.);
        if (vov3 > 3.) {
          const double dd = vov3 - 3.0;
          e_lp += p_lp3 * (dd * dd);
          if (d.pe_on) {   // etally_half(i, nbr, c2.e) (src/cpu/bonded.cpp:275)
            pe_own += 0.5 * p_lp3 * (dd * dd);
            pe_add(d, p, 0.5 * p_lp3 * (dd * dd));
          }
          d.bacc[b].x += 2. * p_lp3 * (vov3 - 3.);
          cdd += 2. * p_lp3 * (vov3 - 3.) * (-1. - 0.16 * pow(Di, 3.));
        }
      }
    }
  }
  // ---- over / under coordination
  {
    const double p_ovun3 = gp[32], p_ovun4 = gp[31], p_ovun6 = gp[6], p_ovun7 = gp[8], p_ovun8 = gp[9];
    const double dfvl = sj[SB_HEAVY] != 0.0 ? 0.0 : 1.0;
    double sum1 = 0, sum2 = 0;
    for (int k = 0; k < nb; ++k) {
      const size_t b = base + k;
      const int p = static_cast<int>(d.bcode[b] & d.amask);
      const double* tb = TBp(ff, tj, d.type[p]);
      const double4 bo = d.bBO[b];
      const AtomQ aqp = d.aq[p];
      sum1 += tb[TB_P_OVUN1] * tb[TB_DE_S] * bo.x;
      sum2 += (aqp.Delta - dfvl * aqp.Delta_lp_temp) * (bo.z + bo.w);
    }
    const bool under_active = nb > 0 || ctl.enobonds;
    const double Delta = aqj.Delta, Delta_lp_temp = aqj.Delta_lp_temp, dDelta_lp = aqj.dDelta_lp;
    const double valency = sj[SB_VALENCY], p_ovun2 = sj[SB_P_OVUN2], p_ovun5 = sj[SB_P_OVUN5];
    const double exp_ovun1 = p_ovun3 * safe_exp(p_ovun4 * sum2);
    const double inv_exp_ovun1 = 1.0 / (1 + exp_ovun1);
    const double Delta_lpcorr = Delta - (dfvl * Delta_lp_temp) * inv_exp_ovun1;
    const double exp_ovun2 = safe_exp(p_ovun2 * Delta_lpcorr);
    const double inv_exp_ovun2 = 1.0 / (1.0 + exp_ovun2);
    const double DlpVi = 1.0 / (Delta_lpcorr + valency + 1e-8);
    const double CEover1 = Delta_lpcorr * DlpVi * inv_exp_ovun2;
    e_ov += sum1 * CEover1;
    const double CEover2 = sum1 * DlpVi * inv_exp_ovun2 * (1.0 - Delta_lpcorr * (DlpVi + p_ovun2 * exp_ovun2 * inv_exp_ovun2));
    const double CEover3 = CEover2 * (1.0 - dfvl * dDelta_lp * inv_exp_ovun1);
    const double CEover4 = CEover2 * (dfvl * Delta_lp_temp) * p_ovun4 * exp_ovun1 * (inv_exp_ovun1 * inv_exp_ovun1);
    const double exp_ovun2n = safe_exp(-p_ovun2 * Delta_lpcorr);
    const double exp_ovun6 = safe_exp(p_ovun6 * Delta_lpcorr);
    const double exp_ovun8 = p_ovun7 * safe_exp(p_ovun8 * sum2);
    const double inv_exp_ovun2n = 1.0 / (1.0 + exp_ovun2n);
    const double inv_exp_ovun8 = 1.0 / (1.0 + exp_ovun8);
    const double eun = under_active ? -p_ovun5 * (1.0 - exp_ovun6) * inv_exp_ovun2n * inv_exp_ovun8 : 0.0;
    const double CEunder1 = inv_exp_ovun2n * (p_ovun5 * p_ovun6 * exp_ovun6 * inv_exp_ovun8 + p_ovun2 * eun * exp_ovun2n);
    const double CEunder2 = -eun * p_ovun8 * exp_ovun8 * inv_exp_ovun8;
    const double CEunder3 = CEunder1 * (1.0 - dfvl * dDelta_lp * inv_exp_ovun1);
    const double CEunder4 = CEunder1 * (dfvl * Delta_lp_temp) * p_ovun4 * exp_ovun1 * (inv_exp_ovun1 * inv_exp_ovun1) + CEunder2;
    if (under_active) e_un += eun;
    cdd += CEover3;
    if (under_active) cdd += CEunder3;
    for (int k = 0; k < nb; ++k) {
      const size_t b = base + k;
      const int p = static_cast<int>(d.bcode[b] & d.amask);
      const double* tb = TBp(ff, tj, d.type[p]);
      const double4 bo = d.bBO[b];
      const AtomQ aqp = d.aq[p];
      double4 acc = d.bacc[b];
      acc.x += CEover1 * tb[TB_P_OVUN1] * tb[TB_DE_S];
      const double pis = bo.z + bo.w;
      const double dj = aqp.Delta - dfvl * aqp.Delta_lp_temp;
      acc.w += CEover4 * (1.0 - dfvl * aqp.dDelta_lp) * pis;
      acc.y += CEover4 * dj;
      acc.z += CEover4 * dj;
      acc.w += CEunder4 * (1.0 - dfvl * aqp.dDelta_lp) * pis;
      acc.y += CEunder4 * dj;
      acc.z += CEunder4 * dj;
      d.bacc[b] = acc;
    }
  }
  // ---- valence angle / penalty / coalition (centre j)
  {
    const double p_val6 = gp[14], p_val8 = gp[33], p_val9 = gp[16], p_val10 = gp[17];
    const double p_val3 = sj[SB_P_VAL3], p_val5 = sj[SB_P_VAL5];
    const double thb_cut = ctl.thb_cut, thb_cutsq = ctl.thb_cutsq;
    double SBOp = 0, prod_SBO = 1;
    for (int k = 0; k < nb; ++k) {
      const double4 bo = d.bBO[base + k];
      SBOp += (bo.z + bo.w);
      double temp = bo.x * bo.x;
      temp *= temp;
      temp *= temp;
      prod_SBO *= exp(-temp);
    }
    double vlpadj, dSBO2;
    if (aqj.vlpex >= 0) { vlpadj = 0; dSBO2 = prod_SBO - 1; }
    else { vlpadj = aqj.nlp; dSBO2 = (prod_SBO - 1) * (1 - p_val8 * aqj.dDelta_lp); }
    const double Dboc = aqj.Delta_boc;
    const double SBO = SBOp + (1 - prod_SBO) * (-Dboc - p_val8 * vlpadj);
    const double dSBO1 = -8 * prod_SBO * (Dboc + p_val8 * vlpadj);
    double SBO2, CSBO2;
    if (SBO <= 0) { SBO2 = 0; CSBO2 = 0; }
    else if (SBO > 0 && SBO <= 1) { SBO2 = pow(SBO, p_val9); CSBO2 = p_val9 * pow(SBO, p_val9 - 1); }
    else if (SBO > 1 && SBO < 2) { SBO2 = 2 - pow(2 - SBO, p_val9); CSBO2 = p_val9 * pow(2 - SBO, p_val9 - 1); }
    else { SBO2 = 2; CSBO2 = 0; }
    const double expval6 = exp(p_val6 * Dboc);
    d.census[5 * d.na + j] = SBO <= 0 ? 0 : (SBO <= 1 ? 1 : (SBO < 2 ? 2 : 3));
    double S5 = 0.0, S6 = 0.0;   // sums of CEval5 and CEval6 over every evaluated set (applied to all bonds of j)
    int nsets = 0;
    for (int pi = 0; pi < nb; ++pi) {
      const size_t bi = base + pi;
      const double4 boi = d.bBO[bi];
      const double BOA_ij = boi.x - thb_cut;
      if (!(BOA_ij > 0.0)) continue;
      const int ia = static_cast<int>(d.bcode[bi] & d.amask);
      const int type_i = d.type[ia];
      const double4 dvi = d.bdv[bi];
      const double vi[3] = {dvi.x, dvi.y, dvi.z};
      for (int pk = pi + 1; pk < nb; ++pk) {
        const size_t bk = base + pk;
        const double4 bok = d.bBO[bk];
        const double BOA_jk = bok.x - thb_cut;
        if (!((BOA_jk > 0.0) && (boi.x > thb_cut) && (bok.x > thb_cut) && (boi.x * bok.x > thb_cutsq))) continue;
        const int ka = static_cast<int>(d.bcode[bk] & d.amask);
        const int type_k = d.type[ka];
        const double4 dvk = d.bdv[bk];
        const double vk[3] = {dvk.x, dvk.y, dvk.z};
        double theta, cos_theta, dci[3], dcj[3], dck[3];
        calc_theta(vi, dvi.w, vk, dvk.w, theta, cos_theta);
        calc_dcos(vi, dvi.w, vk, dvk.w, dci, dcj, dck);
        double sin_theta = sin(theta);
        if (sin_theta < 1.0e-5) sin_theta = 1.0e-5;
        ++nsets;
        const size_t key = (static_cast<size_t>(type_i) * ff.nt + tj) * ff.nt + type_k;
        const int nset = ff.thb_n[key];
        for (int q = 0; q < nset; ++q) {
          const double* th = ff.thb + (key * kMaxThbSets + q) * TH_NFIELDS;
          if (!(fabs(th[TH_P_VAL1]) > 0.001)) continue;
          const double p_val1 = th[TH_P_VAL1], p_val2 = th[TH_P_VAL2], p_val4 = th[TH_P_VAL4], p_val7 = th[TH_P_VAL7];
          const double theta_00 = th[TH_THETA_00];
          const double exp3ij = exp(-p_val3 * pow(BOA_ij, p_val4));
          const double f7_ij = 1.0 - exp3ij;
          const double Cf7ij = p_val3 * p_val4 * pow(BOA_ij, p_val4 - 1.0) * exp3ij;
          const double exp3jk = exp(-p_val3 * pow(BOA_jk, p_val4));
          const double f7_jk = 1.0 - exp3jk;
          const double Cf7jk = p_val3 * p_val4 * pow(BOA_jk, p_val4 - 1.0) * exp3jk;
          const double expval7 = exp(-p_val7 * Dboc);
          const double trm8 = 1.0 + expval6 + expval7;
          const double f8_Dj = p_val5 - ((p_val5 - 1.0) * (2.0 + expval6) / trm8);
          const double Cf8j = ((1.0 - p_val5) / (trm8 * trm8)) * (p_val6 * expval6 * trm8 - (2.0 + expval6) * (p_val6 * expval6 - p_val7 * expval7));
          double theta_0 = 180.0 - theta_00 * (1.0 - exp(-p_val10 * (2.0 - SBO2)));
          theta_0 = theta_0 * kConstPi / 180.0;
          const double expval2theta = exp(-p_val2 * ((theta_0 - theta) * (theta_0 - theta)));
          const double expval12theta = p_val1 >= 0 ? p_val1 * (1.0 - expval2theta) : p_val1 * -expval2theta;
          const double CEval1 = Cf7ij * f7_jk * f8_Dj * expval12theta;
          const double CEval2 = Cf7jk * f7_ij * f8_Dj * expval12theta;
          const double CEval3 = Cf8j * f7_ij * f7_jk * expval12theta;
          const double CEval4 = -2.0 * p_val1 * p_val2 * f7_ij * f7_jk * f8_Dj * expval2theta * (theta_0 - theta);
          const double Ctheta_0 = p_val10 * (theta_00 * kConstPi / 180.0) * exp(-p_val10 * (2.0 - SBO2));
          const double CEval5 = -CEval4 * Ctheta_0 * CSBO2;
          const double CEval6 = CEval5 * dSBO1;
          const double CEval7 = CEval5 * dSBO2;
          const double CEval8 = -CEval4 / sin_theta;
          e_ang += f7_ij * f7_jk * f8_Dj * expval12theta;
          const double p_pen1 = th[TH_P_PEN1], p_pen2 = gp[19], p_pen3 = gp[20], p_pen4 = gp[21];
          const double exp_pen2ij = exp(-p_pen2 * ((BOA_ij - 2.0) * (BOA_ij - 2.0)));
          const double exp_pen2jk = exp(-p_pen2 * ((BOA_jk - 2.0) * (BOA_jk - 2.0)));
          const double exp_pen3 = exp(-p_pen3 * aqj.Delta);
          const double exp_pen4 = exp(p_pen4 * aqj.Delta);
          const double trm_pen34 = 1.0 + exp_pen3 + exp_pen4;
          const double f9_Dj = (2.0 + exp_pen3) / trm_pen34;
          const double Cf9j = (-p_pen3 * exp_pen3 * trm_pen34 - (2.0 + exp_pen3) * (-p_pen3 * exp_pen3 + p_pen4 * exp_pen4)) / (trm_pen34 * trm_pen34);
          const double e_pen_t = p_pen1 * f9_Dj * exp_pen2ij * exp_pen2jk;
          e_pen += e_pen_t;
          const double CEpen1 = e_pen_t * Cf9j / f9_Dj;
          const double tmp = -2.0 * p_pen2 * e_pen_t;
          const double CEpen2 = tmp * (BOA_ij - 2.0), CEpen3 = tmp * (BOA_jk - 2.0);
          const double p_coa1 = th[TH_P_COA1], p_coa2 = gp[2], p_coa3 = gp[38], p_coa4 = gp[30];
          const double exp_coa2 = exp(p_coa2 * aqj.Delta_val);
          const double dti = d.aq[ia].total_bo - BOA_ij, dtk = d.aq[ka].total_bo - BOA_jk;
          const double e_coa_t = p_coa1 / (1. + exp_coa2) * exp(-p_coa3 * (dti * dti)) * exp(-p_coa3 * (dtk * dtk)) *
                                 exp(-p_coa4 * ((BOA_ij - 1.5) * (BOA_ij - 1.5))) * exp(-p_coa4 * ((BOA_jk - 1.5) * (BOA_jk - 1.5)));
          e_coa += e_coa_t;
          const double CEcoa1 = -2 * p_coa4 * (BOA_ij - 1.5) * e_coa_t;
          const double CEcoa2 = -2 * p_coa4 * (BOA_jk - 1.5) * e_coa_t;
          const double CEcoa3 = -p_coa2 * exp_coa2 * e_coa_t / (1 + exp_coa2);
          const double CEcoa4 = -2 * p_coa3 * dti * e_coa_t;
          const double CEcoa5 = -2 * p_coa3 * dtk * e_coa_t;
          d.bacc[bi].x += (CEval1 + CEpen2 + (CEcoa1 - CEcoa4));
          d.bacc[bk].x += (CEval2 + CEpen3 + (CEcoa2 - CEcoa5));
          cdd += ((CEval3 + CEval7) + CEpen1 + CEcoa3);
          d.bacc[bi].w += CEcoa4;
          d.bacc[bk].w += CEcoa5;
          S5 += CEval5;
          S6 += CEval6;
          add3(d.bfn[bi], CEval8, dci);
          fj[0] += CEval8 * dcj[0]; fj[1] += CEval8 * dcj[1]; fj[2] += CEval8 * dcj[2];
          add3(d.bfn[bk], CEval8, dck);
          vir_add(vir, vi, dci, CEval8);
          vir_add(vir, vk, dck, CEval8);
        }
      }
    }
    if (S5 != 0.0 || S6 != 0.0) {
      for (int k = 0; k < nb; ++k) {
        const size_t b = base + k;
        const double bo = d.bBO[b].x;
        const double cube = bo * bo * bo;
        double4 acc = d.bacc[b];
        acc.x += S6 * (cube * cube * bo);
        acc.y += S5;
        acc.z += S5;
        d.bacc[b] = acc;
      }
    }
    d.census[1 * d.na + j] = nsets;
  }
  d.fown[j] = make_double4(fj[0], fj[1], fj[2], cdd);
  for (int c = 0; c < kVir; ++c) d.vir[static_cast<size_t>(j) * kVir + c] = vir[c];   // first writer of the step
  double* ea = d.eatom + static_cast<size_t>(j) * kTerms;
  ea[E_BOND] = e_bond; ea[E_OV] = e_ov; ea[E_UN] = e_un; ea[E_LP] = e_lp;
  pe_add(d, j, pe_own + e_ov + e_un + e_ang + e_pen + e_coa);   // over/under and the angle sets stay with j
  ea[E_ANG] = e_ang; ea[E_PEN] = e_pen; ea[E_COA] = e_coa;
}

// Hydrogen bonds (src/cpu/bonded.cpp:654-715) of one triple: the donor bond of hydrogen j (its data loaded once per
// bond: partner ia, its type and tag, BO, the bond vector), acceptor k at the canonical vector vk (x_k - x_j) and
// distance r_jk. Every gate of the reference is taken in FP64 (types, tags, BO >= HB_THRESHOLD, parameters present,
// r_jk <= hbond_cut by the caller); the term itself is FP32. sin^4(theta/2) is formed as ((1 - cos theta) / 2)^2, the
// same quantity as the reference's sin(acos(c) / 2)^4.
struct HbDonor { int type_i; long long tag_i; float BO, vi[3], d_ji; };
struct HbOut { float e, CEhb1, CEhb2, CEhb3, dti[3], dtj[3], dtk[3]; };
__device__ inline bool hbond_triple(const DevFF& ff, const HbDonor& dn, int tj, int type_k, long long tag_k, const float* vk,
                                    float r_jk, HbOut& o) {
  if (dn.tag_i == tag_k) return false;
  const size_t key = (static_cast<size_t>(dn.type_i) * ff.nt + tj) * ff.nt + type_k;
  if (!ff.hb_on[key]) return false;
  const double* hb = ff.hb + key * HB_NFIELDS;
  if (hb[HB_R0] <= 0.0) return false;
  const float r0 = static_cast<float>(hb[HB_R0]), p1 = static_cast<float>(hb[HB_P_HB1]);
  const float p2 = static_cast<float>(hb[HB_P_HB2]), p3 = static_cast<float>(hb[HB_P_HB3]);
  const float* vi = dn.vi;
  const float d_ji = dn.d_ji;
  // reaxff_valence_angles.cpp:36-70 (calculate_theta / calculate_dcos_theta) in FP32
  const float inv = 1.0f / (d_ji * r_jk);
  const float dotv = vi[0] * vk[0] + vi[1] * vk[1] + vi[2] * vk[2];
  float c = dotv * inv;
  c = fminf(1.0f, fmaxf(-1.0f, c));
  const float Cdot = dotv * inv * inv * inv;
  const float sq_ji = d_ji * d_ji, sq_jk = r_jk * r_jk;
  for (int t = 0; t < 3; ++t) {
    o.dti[t] = vk[t] * inv - Cdot * sq_jk * vi[t];
    o.dtj[t] = -(vk[t] + vi[t]) * inv + Cdot * (sq_jk * vi[t] + sq_ji * vk[t]);
    o.dtk[t] = vi[t] * inv - Cdot * sq_ji * vk[t];
  }
  const float half = 0.5f * (1.0f - c);
  const float sin_xhz4 = half * half;
  const float cos_xhz1 = 1.0f - c;
  const float exp_hb2 = __expf(-p2 * dn.BO);
  const float exp_hb3 = __expf(-p3 * (r0 / r_jk + r_jk / r0 - 2.0f));
  o.e = p1 * (1.0f - exp_hb2) * exp_hb3 * sin_xhz4;
  o.CEhb1 = p1 * p2 * exp_hb2 * exp_hb3 * sin_xhz4;
  o.CEhb2 = -p1 / 2.0f * (1.0f - exp_hb2) * exp_hb3 * cos_xhz1;
  o.CEhb3 = -p3 * (-r0 / (r_jk * r_jk) + 1.0f / r0) * o.e;
  return true;
}

// One warp per hydrogen j (p_hbond = 1): for every donor bond of j, the lanes walk j's acceptor row (p_hbond = 2 atoms,
// r <= hbond_cut taken again exactly here); each triple is evaluated once. Energy, the gradient of j and the coefficient /
// gradient of the donor bond are reduced over the warp in fixed order (the donor's share goes to j's slot for the
// donor to gather); the acceptor's gradient is added to its fixed-point accumulator (zeroed by k_nbr_check).
__global__ void __launch_bounds__(256) k_hbond(Dev d, DevFF ff, DevCtl ctl) {
  if (lists_failed(d)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  const int j = warp;
  const int tj = d.type[j];
  {   // this kernel's accumulators of atom j start at zero
    const int nbj = min(d.bcnt[j], d.bcap);
    for (int k = lane; k < nbj; k += 32) {
      d.bcdbo_h[static_cast<size_t>(j) * d.bcap + k] = 0.0;
      d.bfn_h[static_cast<size_t>(j) * d.bcap + k] = make_double4(0, 0, 0, 0);
    }
    if (lane < kVir) d.vir_h[static_cast<size_t>(j) * kVir + lane] = 0.0;
    if (lane == 0) d.fown_h[j] = make_double4(0, 0, 0, 0);
    __syncwarp();
  }
  if (!(ctl.hbond_cut > 0) || static_cast<int>(SBp(ff, tj)[SB_P_HBOND]) != 1) {
    if (lane == 0) {
      d.eatom[static_cast<size_t>(j) * kTerms + E_HB] = 0.0;
      d.census[3 * d.na + j] = 0;
    }
    return;
  }
  const SysInfo s = d.sys[d.sys_of[j]];
  const int cnt = min(d.acc_cnt[j], d.ncap_acc);
  const int nb = min(d.bcnt[j], d.bcap);
  const double hc2 = ctl.hbond_cut * ctl.hbond_cut;
  const size_t base = static_cast<size_t>(j) * d.bcap;
  double e = 0.0, fj0 = 0.0, fj1 = 0.0, fj2 = 0.0;
  double vir[kVir] = {0, 0, 0, 0, 0, 0};
  int ntrip = 0;
  for (int pi = 0; pi < nb; ++pi) {
    const size_t bi = base + pi;
    HbDonor dn;
    {  // donor gates that do not depend on the acceptor (warp-uniform), and the donor's data
      const int ia = static_cast<int>(d.bcode[bi] & d.amask);
      dn.type_i = d.type[ia];
      const double BOd = d.bBO[bi].x;
      if (static_cast<int>(SBp(ff, dn.type_i)[SB_P_HBOND]) != 2 || !(BOd >= kHbThreshold)) continue;
      dn.tag_i = d.tag[ia];
      dn.BO = static_cast<float>(BOd);
      const double4 dvi = d.bdv[bi];
      dn.vi[0] = static_cast<float>(dvi.x); dn.vi[1] = static_cast<float>(dvi.y); dn.vi[2] = static_cast<float>(dvi.z);
      dn.d_ji = static_cast<float>(dvi.w);
    }
    double c1 = 0.0, fi0 = 0.0, fi1 = 0.0, fi2 = 0.0;
    const double4 dvi = d.bdv[bi];
    const double pi3[3] = {dvi.x, dvi.y, dvi.z};
    for (int e0 = 0; e0 < cnt; e0 += 32) {
      const int ee = e0 + lane;
      if (ee >= cnt) continue;
      const unsigned code = d.acc[static_cast<size_t>(j) * d.ncap_acc + ee];   // p_hbond = 2 atoms only
      const int ka = static_cast<int>(code & d.amask);
      const int type_k = d.type[ka];
      double dvjk[3];
      pair_dvec(d, s, j, ka, static_cast<int>(code >> d.abits), dvjk);
      const double r2 = dot3(dvjk, dvjk);
      if (!(r2 <= hc2)) continue;
      const double r_jkd = sqrt(r2);
      if (!(r_jkd <= ctl.hbond_cut)) continue;
      const float vk[3] = {static_cast<float>(dvjk[0]), static_cast<float>(dvjk[1]), static_cast<float>(dvjk[2])};
      const float r_jk = static_cast<float>(r_jkd);
      HbOut o;
      if (!hbond_triple(ff, dn, tj, type_k, d.tag[ka], vk, r_jk, o)) continue;
      ++ntrip;
      e += o.e;
      if (d.pe_on) {   // a third to each of donor, hydrogen, acceptor (src/cpu/bonded.cpp:704)
        pe_add(d, static_cast<int>(d.bcode[bi] & d.amask), o.e / 3.0);
        pe_add(d, ka, o.e / 3.0);
      }
      c1 += o.CEhb1;
      fi0 += o.CEhb2 * o.dti[0]; fi1 += o.CEhb2 * o.dti[1]; fi2 += o.CEhb2 * o.dti[2];
      const float c3 = -o.CEhb3 / r_jk;
      fj0 += o.CEhb2 * o.dtj[0] + c3 * vk[0];
      fj1 += o.CEhb2 * o.dtj[1] + c3 * vk[1];
      fj2 += o.CEhb2 * o.dtj[2] + c3 * vk[2];
      const float gk[3] = {o.CEhb2 * o.dtk[0] - c3 * vk[0], o.CEhb2 * o.dtk[1] - c3 * vk[1], o.CEhb2 * o.dtk[2] - c3 * vk[2]};
      const float gi[3] = {o.CEhb2 * o.dti[0], o.CEhb2 * o.dti[1], o.CEhb2 * o.dti[2]};
      for (int c = 0; c < 3; ++c) fix_add(d.fix_h + 3 * static_cast<size_t>(ka) + c, static_cast<double>(gk[c]));
      // virial of the triple about the hydrogen: donor at the bond vector, acceptor at vk
      vir_add(vir, pi3, gi);
      vir_add(vir, vk, gk);
    }
    c1 = warp_sum(c1); fi0 = warp_sum(fi0); fi1 = warp_sum(fi1); fi2 = warp_sum(fi2);
    if (lane == 0) {
      d.bcdbo_h[bi] = c1;
      d.bfn_h[bi] = make_double4(fi0, fi1, fi2, 0.0);
    }
    __syncwarp();
  }
  e = warp_sum(e); fj0 = warp_sum(fj0); fj1 = warp_sum(fj1); fj2 = warp_sum(fj2);
  for (int c = 0; c < kVir; ++c) vir[c] = warp_sum(vir[c]);
  for (int o = 16; o > 0; o >>= 1) ntrip += __shfl_xor_sync(0xffffffffu, ntrip, o);
  if (lane == 0) {
    d.fown_h[j] = make_double4(fj0, fj1, fj2, 0.0);
    for (int c = 0; c < kVir; ++c) d.vir_h[static_cast<size_t>(j) * kVir + c] = vir[c];
    d.eatom[static_cast<size_t>(j) * kTerms + E_HB] = e;
    d.census[3 * d.na + j] = ntrip;
    pe_add(d, j, e / 3.0);
  }
}

// ------------------------------------------------------------------------------------------------ torsion
// One thread per central bond j -> k (slot t of atom j, listed by k_bo_correct: the end that evaluates it in tag order,
// src/cpu/bonded.cpp:480-506, with BO_jk > thb_cut): all bonds i of j (i != k) and l of k (l != j) with the gates of
// :510 and :530 (i != l as images, a torsion entry for (ti, tj, tk, tl), BO_kl > thb_cut, BO_ij BO_jk BO_kl > thb_cut).
// Every write goes to slot t's own rows: its coefficients and the gradient of k (bacc_t/bfn_t[t]), the contributions
// to the bond k-l and the atom l (Tl[t * bcap + position of l in k's slots]) and to the bond j-i and the atom i
// (Ti[t * bcap + position of i in j's slots]), and j's own gradient, CdDelta, energies, count and virial (Tsum[t],
// Tvir[t]); k_fold gathers the rows of the listed slots (tflag) only.
__global__ void k_torsion(Dev d, DevFF ff, DevCtl ctl) {
  if (lists_failed(d)) return;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= static_cast<long long>(*d.tor_n)) return;
  const long long slot = d.tor_list[tid];
  const int j = static_cast<int>(slot / d.bcap), pk = static_cast<int>(slot % d.bcap);
  const int nbj = min(d.bcnt[j], d.bcap);
  const int type_j = d.type[j];
  const size_t base = static_cast<size_t>(j) * d.bcap;
  const size_t bjk = base + pk;
  const double thb_cut = ctl.thb_cut;
  const double* gp = ff.gp;
  const double p_tor2 = gp[23], p_tor3 = gp[24], p_tor4 = gp[25], p_cot2 = gp[27];
  {   // this slot's rows start at zero
    const int ka0 = static_cast<int>(d.bcode[bjk] & d.amask);
    const int nbk0 = min(d.bcnt[ka0], d.bcap);
    for (int q = 0; q < nbk0; ++q) d.Tl[bjk * d.bcap + q] = make_double4(0, 0, 0, 0);
    for (int q = 0; q < nbj; ++q) d.Ti[bjk * d.bcap + q] = make_double4(0, 0, 0, 0);
  }
  double fj[3] = {0, 0, 0}, cdd = 0.0, e_tor = 0.0, e_con = 0.0, pe_tor_own = 0.0;
  double vir[kVir] = {0, 0, 0, 0, 0, 0};
  double4 acc_jk = make_double4(0, 0, 0, 0), fk_own = make_double4(0, 0, 0, 0);
  int ntor = 0;
  const double Delta_j = d.aq[j].Delta_boc;
  do {
    const double4 dvk4 = d.bdv[bjk];
    const unsigned code_k = d.bcode[bjk];
    const int ka = static_cast<int>(code_k & d.amask);
    if (skip_by_tag(d, j, ka, dvk4)) break;
    const double4 bo_jk = d.bBO[bjk];
    if (!(bo_jk.x > thb_cut)) break;
    const int sym_jk = d.bsym[bjk];
    const int nbk = min(d.bcnt[ka], d.bcap);
    const size_t base_k = static_cast<size_t>(ka) * d.bcap;
    const int type_k = d.type[ka];
    int skx, sky, skz;
    decode_shift(static_cast<int>(code_k >> d.abits), d.S, d.smax, skx, sky, skz);
    const double BOA_jk = bo_jk.x - thb_cut;
    const double Delta_k = d.aq[ka].Delta_boc;
    const double r_jk = dvk4.w;
    const double exp_tor2_jk = exp(-p_tor2 * BOA_jk);
    const double exp_cot2_jk = exp(-p_cot2 * ((BOA_jk - 1.5) * (BOA_jk - 1.5)));
    const double exp_tor3_DjDk = exp(-p_tor3 * (Delta_j + Delta_k));
    const double exp_tor4_DjDk = exp(p_tor4 * (Delta_j + Delta_k));
    const double exp_tor34_inv = 1.0 / (1.0 + exp_tor3_DjDk + exp_tor4_DjDk);
    const double f11_DjDk = (2.0 + exp_tor3_DjDk) * exp_tor34_inv;
    const double djk[3] = {dvk4.x, dvk4.y, dvk4.z};
    const double4 dkj4 = d.bdv[sym_jk];
    const double dkj[3] = {dkj4.x, dkj4.y, dkj4.z};
    for (int pi = 0; pi < nbj; ++pi) {
      if (pi == pk) continue;
      const size_t bij = base + pi;
      const double4 bo_ij = d.bBO[bij];
      if (!(bo_ij.x > thb_cut)) continue;
      const unsigned code_i = d.bcode[bij];
      const int ia = static_cast<int>(code_i & d.amask);
      int six, siy, siz;
      decode_shift(static_cast<int>(code_i >> d.abits), d.S, d.smax, six, siy, siz);
      const int type_i = d.type[ia];
      const double4 dvi4 = d.bdv[bij];
      const double dij[3] = {dvi4.x, dvi4.y, dvi4.z};
      const double r_ij = dvi4.w;
      const double BOA_ij = bo_ij.x - thb_cut;
      // p_ijk: angle i-j-k seen from the list of bond j->k (dcos_di w.r.t. k, dcos_dk w.r.t. i)
      double th_ijk, cos_t, pijk_di[3], pijk_dj[3], pijk_dk[3];
      calc_theta(djk, r_jk, dij, r_ij, th_ijk, cos_t);
      calc_dcos(djk, r_jk, dij, r_ij, pijk_di, pijk_dj, pijk_dk);
      const double sin_ijk = sin(th_ijk), cos_ijk = cos(th_ijk);
      double tan_ijk_i;
      if (sin_ijk >= 0 && sin_ijk <= kMinSine) tan_ijk_i = cos_ijk / kMinSine;
      else if (sin_ijk <= 0 && sin_ijk >= -kMinSine) tan_ijk_i = cos_ijk / -kMinSine;
      else tan_ijk_i = cos_ijk / sin_ijk;
      const double exp_tor2_ij = exp(-p_tor2 * BOA_ij);
      const double exp_cot2_ij = exp(-p_cot2 * ((BOA_ij - 1.5) * (BOA_ij - 1.5)));
      for (int pl = 0; pl < nbk; ++pl) {
        const size_t bkl = base_k + pl;
        if (static_cast<int>(bkl) == sym_jk) continue;
        const double4 bo_kl = d.bBO[bkl];
        if (!(bo_kl.x > thb_cut)) continue;
        const unsigned code_l = d.bcode[bkl];
        const int la = static_cast<int>(code_l & d.amask);
        int slx, sly, slz;
        decode_shift(static_cast<int>(code_l >> d.abits), d.S, d.smax, slx, sly, slz);
        if (la == ia && six == skx + slx && siy == sky + sly && siz == skz + slz) continue;   // i != l
        const int type_l = d.type[la];
        const size_t key4 = ((static_cast<size_t>(type_i) * ff.nt + type_j) * ff.nt + type_k) * ff.nt + type_l;
        if (!ff.fb_on[key4]) continue;
        if (!(bo_ij.x * bo_jk.x * bo_kl.x > thb_cut)) continue;
        const double* fb = ff.fb + key4 * FB_NFIELDS;
        ++ntor;
        const double4 dvl4 = d.bdv[bkl];
        const double dkl[3] = {dvl4.x, dvl4.y, dvl4.z};
        const double r_kl = dvl4.w;
        const double BOA_kl = bo_kl.x - thb_cut;
        // p_jkl: angle j-k-l from the list of bond k->j (dcos_di w.r.t. j, dcos_dj w.r.t. k, dcos_dk w.r.t. l)
        double th_jkl, cos_t2, pjkl_di[3], pjkl_dj[3], pjkl_dk[3];
        calc_theta(dkj, r_jk, dkl, r_kl, th_jkl, cos_t2);
        calc_dcos(dkj, r_jk, dkl, r_kl, pjkl_di, pjkl_dj, pjkl_dk);
        const double sin_jkl = sin(th_jkl), cos_jkl = cos(th_jkl);
        double tan_jkl_i;
        if (sin_jkl >= 0 && sin_jkl <= kMinSine) tan_jkl_i = cos_jkl / kMinSine;
        else if (sin_jkl <= 0 && sin_jkl >= -kMinSine) tan_jkl_i = cos_jkl / -kMinSine;
        else tan_jkl_i = cos_jkl / sin_jkl;
        // x_i - x_l from the three bond vectors
        const double dvec_li[3] = {dij[0] - djk[0] - dkl[0], dij[1] - djk[1] - dkl[1], dij[2] - djk[2] - dkl[2]};
        const double r_li = sqrt(dot3(dvec_li, dvec_li));
        double dco_i[3], dco_j[3], dco_k[3], dco_l[3], omega;
        {
          double s_ijk = sin(th_ijk), c_ijk = cos(th_ijk), s_jkl = sin(th_jkl), c_jkl = cos(th_jkl);
          if (s_ijk >= 0 && s_ijk <= kMinSine) s_ijk = kMinSine; else if (s_ijk <= 0 && s_ijk >= -kMinSine) s_ijk = -kMinSine;
          if (s_jkl >= 0 && s_jkl <= kMinSine) s_jkl = kMinSine; else if (s_jkl <= 0 && s_jkl >= -kMinSine) s_jkl = -kMinSine;
          const double unnorm_cos_omega = -dot3(dij, djk) * dot3(djk, dkl) + (r_jk * r_jk) * dot3(dij, dkl);
          const double cjkkl[3] = {djk[1] * dkl[2] - djk[2] * dkl[1], djk[2] * dkl[0] - djk[0] * dkl[2], djk[0] * dkl[1] - djk[1] * dkl[0]};
          const double unnorm_sin_omega = -r_jk * dot3(dij, cjkkl);
          omega = atan2(unnorm_sin_omega, unnorm_cos_omega);
          const double htra = r_ij + c_ijk * (r_kl * c_jkl - r_jk);
          const double htrb = r_jk - r_ij * c_ijk - r_kl * c_jkl;
          const double htrc = r_kl + c_jkl * (r_ij * c_ijk - r_jk);
          const double hthd = r_ij * s_ijk * (r_jk - r_kl * c_jkl);
          const double hthe = r_kl * s_jkl * (r_jk - r_ij * c_ijk);
          const double hnra = r_kl * s_ijk * s_jkl;
          const double hnrc = r_ij * s_ijk * s_jkl;
          const double hnhd = r_ij * r_kl * c_ijk * s_jkl;
          const double hnhe = r_ij * r_kl * s_ijk * c_jkl;
          const double tel = (r_ij * r_ij) + (r_jk * r_jk) + (r_kl * r_kl) - (r_li * r_li) -
                             2.0 * (r_ij * r_jk * c_ijk - r_ij * r_kl * c_ijk * c_jkl + r_jk * r_kl * c_jkl);
          const double poem = 2.0 * r_ij * r_kl * s_ijk * s_jkl;
          double arg = tel / poem;
          if (arg > 1.0) arg = 1.0;
          if (arg < -1.0) arg = -1.0;
          for (int c = 0; c < 3; ++c) {
            dco_i[c] = (htra - arg * hnra) / r_ij * dij[c] + -1. * dvec_li[c];
            dco_i[c] += -(hthd - arg * hnhd) / s_ijk * pijk_dk[c];
            dco_i[c] = 2.0 / poem * dco_i[c];
            dco_j[c] = -(htra - arg * hnra) / r_ij * dij[c] + -htrb / r_jk * djk[c];
            dco_j[c] += -(hthd - arg * hnhd) / s_ijk * pijk_dj[c];
            dco_j[c] += -(hthe - arg * hnhe) / s_jkl * pjkl_di[c];
            dco_j[c] = 2.0 / poem * dco_j[c];
            dco_k[c] = -(htrc - arg * hnrc) / r_kl * dkl[c] + htrb / r_jk * djk[c];
            dco_k[c] += -(hthd - arg * hnhd) / s_ijk * pijk_di[c];
            dco_k[c] += -(hthe - arg * hnhe) / s_jkl * pjkl_dj[c];
            dco_k[c] = 2.0 / poem * dco_k[c];
            dco_l[c] = (htrc - arg * hnrc) / r_kl * dkl[c] + 1. * dvec_li[c];
            dco_l[c] += -(hthe - arg * hnhe) / s_jkl * pjkl_dk[c];
            dco_l[c] = 2.0 / poem * dco_l[c];
          }
        }
        const double cos_omega = cos(omega), cos2omega = cos(2. * omega), cos3omega = cos(3. * omega);
        const double V1 = fb[FB_V1], V2 = fb[FB_V2], V3 = fb[FB_V3], p_tor1 = fb[FB_P_TOR1], p_cot1 = fb[FB_P_COT1];
        const double exp_tor1 = exp(p_tor1 * ((2.0 - bo_jk.z - f11_DjDk) * (2.0 - bo_jk.z - f11_DjDk)));
        const double exp_tor2_kl = exp(-p_tor2 * BOA_kl);
        const double exp_cot2_kl = exp(-p_cot2 * ((BOA_kl - 1.5) * (BOA_kl - 1.5)));
        const double fn10 = (1.0 - exp_tor2_ij) * (1.0 - exp_tor2_jk) * (1.0 - exp_tor2_kl);
        const double CV = 0.5 * (V1 * (1.0 + cos_omega) + V2 * exp_tor1 * (1.0 - cos2omega) + V3 * (1.0 + cos3omega));
        e_tor += fn10 * sin_ijk * sin_jkl * CV;
        const double dfn11 = (-p_tor3 * exp_tor3_DjDk + (p_tor3 * exp_tor3_DjDk - p_tor4 * exp_tor4_DjDk) * (2.0 + exp_tor3_DjDk) * exp_tor34_inv) * exp_tor34_inv;
        const double CEtors1 = sin_ijk * sin_jkl * CV;
        const double CEtors2 = -fn10 * 2.0 * p_tor1 * V2 * exp_tor1 * (2.0 - bo_jk.z - f11_DjDk) * (1.0 - (cos_omega * cos_omega)) * sin_ijk * sin_jkl;
        const double CEtors3 = CEtors2 * dfn11;
        const double CEtors4 = CEtors1 * p_tor2 * exp_tor2_ij * (1.0 - exp_tor2_jk) * (1.0 - exp_tor2_kl);
        const double CEtors5 = CEtors1 * p_tor2 * (1.0 - exp_tor2_ij) * exp_tor2_jk * (1.0 - exp_tor2_kl);
        const double CEtors6 = CEtors1 * p_tor2 * (1.0 - exp_tor2_ij) * (1.0 - exp_tor2_jk) * exp_tor2_kl;
        const double cmn = -fn10 * CV;
        const double CEtors7 = cmn * sin_jkl * tan_ijk_i;
        const double CEtors8 = cmn * sin_ijk * tan_jkl_i;
        const double CEtors9 = fn10 * sin_ijk * sin_jkl * (0.5 * V1 - 2.0 * V2 * exp_tor1 * cos_omega + 1.5 * V3 * (cos2omega + 2.0 * (cos_omega * cos_omega)));
        const double fn12 = exp_cot2_ij * exp_cot2_jk * exp_cot2_kl;
        e_con += p_cot1 * fn12 * (1.0 + ((cos_omega * cos_omega) - 1.0) * sin_ijk * sin_jkl);
        if (d.pe_on) {   // etally_half(j, k, e_tor + e_con) (src/cpu/bonded.cpp:637)
          const double et = fn10 * sin_ijk * sin_jkl * CV + p_cot1 * fn12 * (1.0 + ((cos_omega * cos_omega) - 1.0) * sin_ijk * sin_jkl);
          pe_tor_own += 0.5 * et;
          pe_add(d, ka, 0.5 * et);
        }
        const double Cconj = -2.0 * fn12 * p_cot1 * p_cot2 * (1.0 + ((cos_omega * cos_omega) - 1.0) * sin_ijk * sin_jkl);
        const double CEconj1 = Cconj * (BOA_ij - 1.5e0), CEconj2 = Cconj * (BOA_jk - 1.5e0), CEconj3 = Cconj * (BOA_kl - 1.5e0);
        const double CEconj4 = -p_cot1 * fn12 * ((cos_omega * cos_omega) - 1.0) * sin_jkl * tan_ijk_i;
        const double CEconj5 = -p_cot1 * fn12 * ((cos_omega * cos_omega) - 1.0) * sin_ijk * tan_jkl_i;
        const double CEconj6 = 2.0 * p_cot1 * fn12 * cos_omega * sin_ijk * sin_jkl;
        // coefficients
        acc_jk.y += CEtors2;
        cdd += CEtors3;
        acc_jk.w += CEtors3;
        double4& ti = d.Ti[bjk * d.bcap + pi];
        ti.w += (CEtors4 + CEconj1);
        acc_jk.x += (CEtors5 + CEconj2);
        double4& tl = d.Tl[bjk * d.bcap + pl];
        tl.w += (CEtors6 + CEconj3);
        // gradient
        const double c78 = CEtors7 + CEconj4, c85 = CEtors8 + CEconj5, c96 = CEtors9 + CEconj6;
        double gi[3], gk[3], gl[3];
        for (int c = 0; c < 3; ++c) {
          gi[c] = c78 * pijk_dk[c] + c96 * dco_i[c];
          gk[c] = c78 * pijk_di[c] + c85 * pjkl_dj[c] + c96 * dco_k[c];
          gl[c] = c85 * pjkl_dk[c] + c96 * dco_l[c];
          (&ti.x)[c] += gi[c];
          fj[c] += c78 * pijk_dj[c] + c85 * pjkl_di[c] + c96 * dco_j[c];
          (&fk_own.x)[c] += gk[c];
          (&tl.x)[c] += gl[c];
        }
        {   // virial about j: i at dij, k at djk, l at djk + dkl
          const double pl[3] = {djk[0] + dkl[0], djk[1] + dkl[1], djk[2] + dkl[2]};
          vir_add(vir, dij, gi);
          vir_add(vir, djk, gk);
          vir_add(vir, pl, gl);
        }
      }
    }
  } while (false);
  pe_add(d, j, pe_tor_own);
  d.bacc_t[bjk] = acc_jk;
  d.bfn_t[bjk] = fk_own;
  d.Tsum[2 * bjk] = make_double4(fj[0], fj[1], fj[2], cdd);
  d.Tsum[2 * bjk + 1] = make_double4(e_tor, e_con, static_cast<double>(ntor), 0.0);
  for (int c = 0; c < kVir; ++c) d.Tvir[bjk * kVir + c] = vir[c];
}

// ------------------------------------------------------------------------------------------------ gathers
// k folds the torsion contributions written for its bonds (Tl of every central bond j -> k) into its own slots, and
// sums its total CdDelta: own part + the parts its partners wrote into their slots naming k.
__global__ void k_fold(Dev d) {
  if (lists_failed(d)) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  const int nb = min(d.bcnt[a], d.bcap);
  const size_t base = static_cast<size_t>(a) * d.bcap;
  {   // a's torsions as the central atom j: per-slot partials of its central bonds, in slot order
    double4 own = make_double4(0, 0, 0, 0), en = make_double4(0, 0, 0, 0);
    double vr[kVir] = {0, 0, 0, 0, 0, 0};
    for (int c = 0; c < nb; ++c) {
      if (!d.tflag[base + c]) continue;
      const double4 t0 = d.Tsum[2 * (base + c)], t1 = d.Tsum[2 * (base + c) + 1];
      own.x += t0.x; own.y += t0.y; own.z += t0.z; own.w += t0.w;
      en.x += t1.x; en.y += t1.y; en.z += t1.z;
      for (int k = 0; k < kVir; ++k) vr[k] += d.Tvir[(base + c) * kVir + k];
    }
    d.fown_t[a] = own;
    for (int k = 0; k < kVir; ++k) d.vir_t[static_cast<size_t>(a) * kVir + k] = vr[k];
    d.eatom[static_cast<size_t>(a) * kTerms + E_TOR] = en.x;
    d.eatom[static_cast<size_t>(a) * kTerms + E_CON] = en.y;
    d.census[2 * d.na + a] = static_cast<int>(en.z);
  }
  for (int p = 0; p < nb; ++p) {
    double4 acc = make_double4(0, 0, 0, 0);
    for (int b = 0; b < nb; ++b) {
      const int c = d.bsym[base + b];
      if (!d.tflag[c]) continue;
      const double4 t = d.Tl[static_cast<size_t>(c) * d.bcap + p];
      acc.x += t.x; acc.y += t.y; acc.z += t.z; acc.w += t.w;
    }
    for (int c = 0; c < nb; ++c) {   // torsions in which the bond a-p is the first bond i-j of a central bond of a
      if (!d.tflag[base + c]) continue;
      const double4 t = d.Ti[(base + c) * d.bcap + p];
      acc.x += t.x; acc.y += t.y; acc.z += t.z; acc.w += t.w;
    }
    const bool own = d.tflag[base + p] != 0;
    double4 at = own ? d.bacc_t[base + p] : make_double4(0, 0, 0, 0);
    at.x += acc.w;
    d.bacc_t[base + p] = at;
    double4 fn = own ? d.bfn_t[base + p] : make_double4(0, 0, 0, 0);
    fn.x += acc.x; fn.y += acc.y; fn.z += acc.z;
    d.bfn_t[base + p] = fn;
  }
  double cd = d.fown[a].w + d.fown_t[a].w;
  for (int b = 0; b < nb; ++b) {
    const int c = d.bsym[base + b];
    cd += d.bacc[c].w + (d.tflag[c] ? d.bacc_t[c].w : 0.0);   // .w of a listed slot: k_torsion's, unchanged here
  }
  d.cdtot[a] = cd;
}

// Add_dBond_to_Forces (src/cpu/bonded.cpp:717-766) rewritten per atom: for each bond of atom a the coefficient of
// dBOp(a->p), of dln_BOp_pi/pi2(a->p) and of dDeltap_self[a]; W[a] = sum of the dDeltap_self coefficients, which the
// bond partners apply to their own dBOp in k_force_final.
__global__ void k_dbond(Dev d) {
  if (lists_failed(d)) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  const int nb = min(d.bcnt[a], d.bcap);
  const size_t base = static_cast<size_t>(a) * d.bcap;
  double f[3] = {0, 0, 0}, W = 0.0;
  double vir[kVir] = {0, 0, 0, 0, 0, 0}, vw[kVir] = {0, 0, 0, 0, 0, 0};
  const double cda = d.cdtot[a];
  for (int k = 0; k < nb; ++k) {
    const size_t b = base + k;
    const int p = static_cast<int>(d.bcode[b] & d.amask);
    const int bs = d.bsym[b];
    const double4 A0 = d.bacc[b], B0 = d.bacc[bs], At = d.bacc_t[b], Bt = d.bacc_t[bs];
    const double4 A = make_double4(A0.x + d.bcdbo_h[b] + At.x, A0.y + At.y, A0.z + At.z, 0.0);
    const double4 B = make_double4(B0.x + d.bcdbo_h[bs] + Bt.x, B0.y + Bt.y, B0.z + Bt.z, 0.0);
    const double c_bo = A.x + B.x, c_pi = A.y + B.y, c_pi2 = A.z + B.z, c_dd = cda + d.cdtot[p];
    const double4 C0 = d.bC0[b], C1 = d.bC1[b], C2 = d.bC2[b];
    // C0 = (C1dbo, C2dbo, C3dbo, C1dbopi), C1 = (C2dbopi, C3dbopi, C4dbopi, C1dbopi2), C2 = (C2dbopi2, C3dbopi2, C4dbopi2)
    const double X1 = C0.x * c_bo + C0.x * c_dd + C1.x * c_pi + C2.x * c_pi2;
    const double Xs = C0.y * c_bo + C0.y * c_dd + C1.y * c_pi + C2.y * c_pi2;
    const double Ypi = C0.w * c_pi, Ypi2 = C1.w * c_pi2;
    const double4 g = d.bdBOp[b], l1 = d.bdlnpi[b], l2 = d.bdlnpi2[b];
    const double u[3] = {X1 * g.x + Ypi * l1.x + Ypi2 * l2.x, X1 * g.y + Ypi * l1.y + Ypi2 * l2.y, X1 * g.z + Ypi * l1.z + Ypi2 * l2.z};
    f[0] += u[0];
    f[1] += u[1];
    f[2] += u[2];
    W += Xs;
    // virial: u acts on a and -u on p (the reverse slot computes the same pair), so each slot carries half of it;
    // the dDeltap_self part W dBOp(a->p) pairs with -W dBOp(a->p) that p gathers in k_force_final: whole here
    const double4 dv = d.bdv[b];
    const double P[3] = {-dv.x, -dv.y, -dv.z};
    const double gg[3] = {g.x, g.y, g.z};
    vir_add(vir, P, u, 0.5);
    vir_add(vw, P, gg);
  }
  const double4 ds = d.dDp_self[a];
  f[0] += W * ds.x; f[1] += W * ds.y; f[2] += W * ds.z;
  d.W[a] = W;
  d.fdb[a] = make_double4(f[0], f[1], f[2], 0.0);
  for (int c = 0; c < kVir; ++c) d.vir[static_cast<size_t>(a) * kVir + c] += vir[c] + W * vw[c];
}

__global__ void k_force_final(Dev d) {
  if (lists_failed(d)) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  const int nb = min(d.bcnt[a], d.bcap);
  const size_t base = static_cast<size_t>(a) * d.bcap;
  const double4 f1 = d.fown[a], fh = d.fown_h[a], ft = d.fown_t[a], f2 = d.fdb[a], f3 = d.fnb[a];
  double g[3] = {f1.x + fh.x + ft.x + f2.x + f3.x, f1.y + fh.y + ft.y + f2.y + f3.y, f1.z + fh.z + ft.z + f2.z + f3.z};
  for (int c = 0; c < 3; ++c) g[c] += fix_value(d.fix_h[3 * static_cast<size_t>(a) + c]);   // H-bond acceptor gradient
  for (int k = 0; k < nb; ++k) {
    const size_t b = base + k;
    const int p = static_cast<int>(d.bcode[b] & d.amask);
    const int bs = d.bsym[b];
    const double4 fa = d.bfn[bs], fhb = d.bfn_h[bs], ftr = d.bfn_t[bs];
    const double4 fn = make_double4(fa.x + fhb.x + ftr.x, fa.y + fhb.y + ftr.y, fa.z + fhb.z + ftr.z, 0.0);
    const double Wp = d.W[p];
    const double4 dB = d.bdBOp[b];
    g[0] += fn.x + Wp * dB.x;
    g[1] += fn.y + Wp * dB.y;
    g[2] += fn.z + Wp * dB.z;
  }
  d.grad[a] = make_double4(g[0], g[1], g[2], 0.0);
}

}  // namespace rx
