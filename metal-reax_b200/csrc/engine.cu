// Host side of the engine: device buffers, capacity growth, the launch sequence of one force evaluation, the charge
// solve, the NVT loop, and the C ABI declared in include/rxcuda.h.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rxcuda.h"
#include "device.cuh"
#include "ffield.hpp"
#include "kernels.hpp"
#include "md.hpp"

namespace rx {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define RXCU(call)                                                                                             \
  do {                                                                                                         \
    cudaError_t e_ = (call);                                                                                   \
    if (e_ != cudaSuccess) throw ::rx::Error(RX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

// A device allocation that only grows.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { if (p) cudaFree(p); }
  void ensure(size_t want) {
    if (want <= n && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    const size_t m = want > 0 ? want : 1;
    RXCU(cudaMalloc(&p, m * sizeof(T)));
    n = m;
  }
};

static void taper_coeffs(double swa, double swb, double* c) {   // include/reaxmetal/terms_host.hpp:16-29
  const double d1 = swb - swa, d7 = std::pow(d1, 7.0);
  const double swa2 = swa * swa, swa3 = swa * swa * swa, swb2 = swb * swb, swb3 = swb * swb * swb;
  c[7] = 20.0 / d7;
  c[6] = -70.0 * (swa + swb) / d7;
  c[5] = 84.0 * (swa2 + 3.0 * swa * swb + swb2) / d7;
  c[4] = -35.0 * (swa3 + 9.0 * swa2 * swb + 9.0 * swa * swb2 + swb3) / d7;
  c[3] = 140.0 * (swa3 * swb + 3.0 * swa2 * swb2 + swa * swb3) / d7;
  c[2] = -210.0 * (swa3 * swb2 + swa2 * swb3) / d7;
  c[1] = 140.0 * swa3 * swb3 / d7;
  c[0] = (-35.0 * swa3 * swb2 * swb2 + 21.0 * swa2 * swb3 * swb2 - 7.0 * swa * swb3 * swb3 + swb3 * swb3 * swb) / d7;
}

struct Phase {
  const char* name;
  cudaEvent_t a, b;
  double ms;
};

struct Context {
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  // concurrent branches of an evaluation: the bonded chain (side), H-bonds (side_h) and torsions (side_t) next to
  // the charge solve and the non-bonded pairs on `stream`
  cudaStream_t side = nullptr, side_h = nullptr, side_t = nullptr;
  cudaStream_t side_c = nullptr;   // capture of the rebuild kernels into their graph conditional
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fork2 = nullptr, ev_join_h = nullptr, ev_join_t = nullptr;
  cudaEvent_t ev_tail = nullptr, ev_tail_done = nullptr;   // rx_compute: the gradient's copy beside the energy sums
  // one captured MD step (replayed for every step of rx_md_run); dropped whenever a buffer or a parameter it holds
  // changes
  cudaGraphExec_t md_graph = nullptr;
  // one captured evaluation without / with the charge solve (rx_compute, the batch evaluations)
  cudaGraphExec_t eval_graph[2] = {nullptr, nullptr};
  long long eval_launches[2] = {0, 0};
  bool graphs_ok = true;                // false after a capture failed: steps are then launched one by one
  void drop_graph() {
    if (md_graph) cudaGraphExecDestroy(md_graph);
    md_graph = nullptr;
    for (auto& g : eval_graph) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
  }
  std::string err;

  bool have_ff = false;
  ForceField ff;
  DBuf<double> ff_buf;
  DevFF dff{};
  DevCtl ctl{5.0, 7.5, 0.001, 0.00001, 1};
  QeqParams qp{};
  double qeq_tol = 1e-6;
  int qeq_imax = 200;
  int qeq_strict = 0;

  // systems
  int nsys = 0, na = 0;
  std::vector<SysInfo> hsys;
  std::vector<int> hsys_of;
  std::vector<long long> htag;
  std::vector<int> htype;
  std::vector<SysInfo> huser;   // systems as the caller gave them
  DBuf<SysInfo> sys;
  DBuf<int> sys_of, type, cell_key, cell_key_sorted, cell_atoms, atom_iota, cell_start, sys_flag;
  DBuf<float4> xs;
  DBuf<long long> tag;
  DBuf<double4> x;
  DBuf<double> q;
  DBuf<unsigned char> cub_tmp;
  int ncell_total = 0;
  int smax = 1, S = 3, abits = 27;
  bool have_pos = false;

  // lists
  int ncap = 0, bcap = 0, ncap_near = 0, ncap_acc = 0, vcap = 0;
  double skin = 1.0;   // Verlet skin [A]: rows hold every image within nonb_cut + skin, rebuilt per system on demand
  DBuf<unsigned> nbr, bcode, near, acc, vrow;
  DBuf<int> nbr_cnt, bsym, bcnt, near_cnt, acc_cnt, vcnt;
  DBuf<double4> shifts, xref;
  DBuf<float> hhi, hlo;
  DBuf<double4> bdv, bBO, bdBOp, bdlnpi, bdlnpi2, bC0, bC1, bC2, bacc, bfn, Tl, Ti, Tsum, bfn_h, bacc_t, bfn_t;
  DBuf<double> Tvir;
  DBuf<unsigned char> tflag;
  DBuf<int> tor_list, tor_n;
  DBuf<double> bcdbo_h;
  // atoms
  DBuf<double> Deltap, Deltap_boc, cdtot, W, eatom;
  DBuf<double4> dDp_self, fown, fdb, fnb, grad, fown_h, fown_t;
  DBuf<unsigned long long> fix_h, pe_fix;
  int pe_on = 0;
  DBuf<AtomQ> aq;
  DBuf<int> census, status;
  DBuf<long long> counters;
  DBuf<double> energies, virial, vir, vir_nb, vir_h, vir_t;
  DBuf<double> epart;   // per (system, 256-atom chunk) partial sums of the energy terms and virial components
  int echunks = 1;
  // QEq
  DBuf<double2> cg_x, cg_b, cg_r, cg_d, cg_p, cg_q;
  DBuf<float2> cg_df;
  DBuf<double> cg_eta, cg_part, s_hist, t_hist, cg_rel;
  DBuf<int> cg_iters, cg_nlive, cg_nref, cg_brk;
  DBuf<SysCg> cg_sys;
  DBuf<double2> cg_rb0, cg_rb1;
  std::vector<int> last_iters;
  std::vector<double> last_rel;
  // MD
  bool md_ready = false;
  DBuf<double4> v;
  DBuf<double> mass, ke, temp, scale, xi, vxi, kpart, ramp;
  DBuf<int> kfirst, ksys;
  MdDev md{};
  long long md_step = 0;
  // pinned host staging for per-step positions in and gradients out, and for the small results of an evaluation
  // (status words, CG counts, energies), so that one synchronisation brings all of them back
  double4* pinned = nullptr;
  size_t pinned_n = 0;
  char* pin_small = nullptr;
  size_t pin_small_n = 0;
  double* pin_e = nullptr;
  size_t pin_e_n = 0;
  double* energy_stage(size_t n) {
    if (pin_e_n < n) {
      if (pin_e) cudaFreeHost(pin_e);
      pin_e = nullptr;
      pin_e_n = 0;
      RXCU(cudaMallocHost(&pin_e, n * sizeof(double)));
      pin_e_n = n;
    }
    return pin_e;
  }
  char* small_stage(size_t bytes) {
    if (pin_small_n < bytes) {
      if (pin_small) cudaFreeHost(pin_small);
      pin_small = nullptr;
      pin_small_n = 0;
      RXCU(cudaMallocHost(&pin_small, bytes));
      pin_small_n = bytes;
    }
    return pin_small;
  }
  double4* stage(size_t n) {
    if (pinned_n < n) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      pinned_n = 0;
      RXCU(cudaMallocHost(&pinned, n * sizeof(double4)));
      pinned_n = n;
    }
    return pinned;
  }
  // kernels of this engine launched so far (library kernels such as the radix sort are not counted)
  long long launches = 0;
  int key_bits = 32;
  // timing
  bool timing = false;
  std::vector<Phase> phases;

  // dev < 0: a host-only context (force-field reading and inspection; every device entry point reports RX_ERR_STATE)
  bool host_only = false;
  explicit Context(int dev) : device(dev) {
    if (dev < 0) {
      host_only = true;
      device = 0;
      return;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) throw Error(RX_ERR_CUDA, "no CUDA device");
    if (dev < 0 || dev >= n) throw Error(RX_ERR_INVALID, "device ordinal out of range");
    RXCU(cudaSetDevice(dev));
    RXCU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    RXCU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (cudaStream_t* st : {&side, &side_h, &side_t, &side_c}) RXCU(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
    for (cudaEvent_t* ev : {&ev_fork, &ev_join, &ev_fork2, &ev_join_h, &ev_join_t, &ev_tail, &ev_tail_done})
      RXCU(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    status.ensure(kStatusWords);
    counters.ensure(8);
    set_qeq(0.0, 10.0, 1e-6, 200, 0);
  }
  ~Context() {
    if (host_only) return;
    if (pinned) cudaFreeHost(pinned);
    if (pin_small) cudaFreeHost(pin_small);
    if (pin_e) cudaFreeHost(pin_e);
    drop_graph();
    for (auto& p : phases) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (cudaEvent_t ev : {ev_fork, ev_join, ev_fork2, ev_join_h, ev_join_t, ev_tail, ev_tail_done})
      if (ev) cudaEventDestroy(ev);
    for (cudaStream_t st : {side, side_h, side_t, side_c})
      if (st) cudaStreamDestroy(st);
    if (stream) cudaStreamDestroy(stream);
  }

  // ------------------------------------------------------------------ configuration
  void set_forcefield(const char* text, int lg) {
    if (!text) throw Error(RX_ERR_INVALID, "null force-field text");
    try {
      ff = parse_force_field(text, lg != 0);
    } catch (const FfieldError& e) {
      throw Error(RX_ERR_FFIELD, e.what());
    }
    const size_t nsb = ff.sb.size(), ntb = ff.tb.size(), nthb = ff.thb.size(), nfb = ff.fb.size(), nhb = ff.hb.size();
    const size_t nthn = ff.thb_n.size(), nfo = ff.fb_on.size(), nho = ff.hb_on.size();
    // ints are stored in the same buffer as doubles (one double slot per int)
    std::vector<double> shld(static_cast<size_t>(ff.nt) * ff.nt);
    for (int a = 0; a < ff.nt; ++a)
      for (int b = 0; b < ff.nt; ++b) shld[static_cast<size_t>(a) * ff.nt + b] = std::pow(ff.s(a, SB_GAMMA) * ff.s(b, SB_GAMMA), -1.5);
    // single-precision pair table of the non-bonded kernel: alpha, D, r_vdW, (1/gamma_w)^p_vdW1, ecore, acore, rcore,
    // gamma (Coulomb shielding), lgcij, lgre^6, 1/r_vdW, 1/rcore (12 floats per type pair)
    std::vector<float> nbf(static_cast<size_t>(ff.nt) * ff.nt * 12, 0.0f);
    for (int a = 0; a < ff.nt; ++a)
      for (int b = 0; b < ff.nt; ++b) {
        float* o = nbf.data() + (static_cast<size_t>(a) * ff.nt + b) * 12;
        o[0] = static_cast<float>(ff.p(a, b, TB_ALPHA));
        o[1] = static_cast<float>(ff.p(a, b, TB_D));
        o[2] = static_cast<float>(ff.p(a, b, TB_R_VDW));
        o[3] = static_cast<float>(std::pow(1.0 / ff.p(a, b, TB_GAMMA_W), ff.gp[28]));
        o[4] = static_cast<float>(ff.p(a, b, TB_ECORE));
        o[5] = static_cast<float>(ff.p(a, b, TB_ACORE));
        o[6] = static_cast<float>(ff.p(a, b, TB_RCORE));
        o[7] = static_cast<float>(ff.p(a, b, TB_GAMMA));
        o[8] = static_cast<float>(ff.p(a, b, TB_LGCIJ));
        o[9] = static_cast<float>(std::pow(ff.p(a, b, TB_LGRE), 6.0));
        o[10] = static_cast<float>(1.0 / ff.p(a, b, TB_R_VDW));
        o[11] = static_cast<float>(1.0 / ff.p(a, b, TB_RCORE));
      }
    const size_t nbf_d = nbf.size() / 2;
    // Bond-order reach per type pair: beyond r_bo every uncorrected component BO'_s, BO'_pi, BO'_pipi is below bo_cut/3
    // (each decreases with r when its exponent pair is p_bo(odd) < 0 < p_bo(even)), so BO' < bo_cut there and the pair
    // is no bond (the gate of src/cpu/bonded.cpp:130). k_bonds skips their exponentials; the bond list is unchanged.
    // Pairs whose parameters do not decrease keep the whole bond_cut (r_bo = infinity).
    std::vector<double> rbo2(static_cast<size_t>(ff.nt) * ff.nt, HUGE_VAL);
    for (int a = 0; a < ff.nt; ++a)
      for (int b = 0; b < ff.nt; ++b) {
        const double c = ff.bo_cut / 3.0;
        double reach = 0.0;
        bool ok = c > 0.0;
        auto comp = [&](bool present, double r0, double p_odd, double p_even, double scale) {
          if (!present || !ok) return;
          if (!(r0 > 0.0) || !(p_odd < 0.0) || !(p_even > 0.0)) { ok = false; return; }
          const double arg = std::log(c / scale) / p_odd;   // (r / r0)^p_even at the crossing
          if (!(arg > 0.0)) { ok = false; return; }
          reach = std::max(reach, r0 * std::pow(arg, 1.0 / p_even));
        };
        comp(ff.s(a, SB_R_S) > 0.0 && ff.s(b, SB_R_S) > 0.0, ff.p(a, b, TB_R_S), ff.p(a, b, TB_P_BO1), ff.p(a, b, TB_P_BO2), 1.0 + ff.bo_cut);
        comp(ff.s(a, SB_R_PI) > 0.0 && ff.s(b, SB_R_PI) > 0.0, ff.p(a, b, TB_R_P), ff.p(a, b, TB_P_BO3), ff.p(a, b, TB_P_BO4), 1.0);
        comp(ff.s(a, SB_R_PI_PI) > 0.0 && ff.s(b, SB_R_PI_PI) > 0.0, ff.p(a, b, TB_R_PP), ff.p(a, b, TB_P_BO5), ff.p(a, b, TB_P_BO6), 1.0);
        if (ok && std::isfinite(reach)) {
          const double r = reach * (1.0 + 1e-6) + 1e-6;
          rbo2[static_cast<size_t>(a) * ff.nt + b] = r * r;
        }
      }
    const size_t total = 64 + nsb + ntb + nthb + nfb + nhb + nthn + nfo + nho + shld.size() + rbo2.size() + nbf_d;
    std::vector<double> h(total, 0.0);
    size_t off = 0;
    auto put = [&](const double* src, size_t n) { std::memcpy(h.data() + off, src, n * sizeof(double)); size_t o = off; off += n; return o; };
    std::vector<double> gp(64, 0.0);
    std::copy(ff.gp.begin(), ff.gp.begin() + std::min<size_t>(ff.gp.size(), 64), gp.begin());
    const size_t o_gp = put(gp.data(), 64), o_sb = put(ff.sb.data(), nsb), o_tb = put(ff.tb.data(), ntb), o_thb = put(ff.thb.data(), nthb);
    const size_t o_fb = put(ff.fb.data(), nfb), o_hb = put(ff.hb.data(), nhb), o_shld = put(shld.data(), shld.size());
    const size_t o_rbo2 = put(rbo2.data(), rbo2.size());
    const size_t o_nbf = off;
    std::memcpy(h.data() + off, nbf.data(), nbf.size() * sizeof(float));
    off += nbf_d;
    auto put_int = [&](const std::vector<int>& v) {
      const size_t o = off;
      std::memcpy(reinterpret_cast<int*>(h.data() + off), v.data(), v.size() * sizeof(int));
      off += (v.size() * sizeof(int) + sizeof(double) - 1) / sizeof(double);
      return o;
    };
    const size_t o_thn = put_int(ff.thb_n), o_fo = put_int(ff.fb_on), o_ho = put_int(ff.hb_on);
    if (host_only) {
      have_ff = true;
      return;
    }
    ff_buf.ensure(total);
    RXCU(cudaMemcpy(ff_buf.p, h.data(), total * sizeof(double), cudaMemcpyHostToDevice));
    dff.nt = ff.nt;
    dff.vdw_type = ff.vdw_type;
    dff.lg = lg != 0;
    dff.bo_cut = ff.bo_cut;
    dff.nonb_low = ff.nonb_low;
    dff.nonb_cut = ff.nonb_cut;
    dff.gp = ff_buf.p + o_gp;
    dff.sb = ff_buf.p + o_sb;
    dff.tb = ff_buf.p + o_tb;
    dff.thb = ff_buf.p + o_thb;
    dff.fb = ff_buf.p + o_fb;
    dff.hb = ff_buf.p + o_hb;
    dff.shld = ff_buf.p + o_shld;
    dff.rbo2 = ff_buf.p + o_rbo2;
    dff.nbf = reinterpret_cast<const float*>(ff_buf.p + o_nbf);
    dff.thb_n = reinterpret_cast<const int*>(ff_buf.p + o_thn);
    dff.fb_on = reinterpret_cast<const int*>(ff_buf.p + o_fo);
    dff.hb_on = reinterpret_cast<const int*>(ff_buf.p + o_ho);
    taper_coeffs(ff.nonb_low, ff.nonb_cut, dff.tap);
    have_ff = true;
    if (nsys > 0) layout_systems();
  }

  void set_control(double bond_cut, double hbond_cut, double thb_cut, double thb_cutsq, int enobonds) {
    if (!(bond_cut > 0) || !(hbond_cut >= 0) || !std::isfinite(bond_cut) || !std::isfinite(hbond_cut))
      throw Error(RX_ERR_INVALID, "cut-offs must be finite, bond_cut > 0, hbond_cut >= 0");
    ctl = DevCtl{bond_cut, hbond_cut, thb_cut, thb_cutsq, enobonds};
    drop_graph();
    if (have_ff && nsys > 0) layout_systems();   // the short Verlet rows hold the cut-offs: rebuild them
  }

  void set_neighbor(double sk) {
    if (!(sk >= 0.0) || !std::isfinite(sk) || sk > 10.0) throw Error(RX_ERR_INVALID, "neighbor skin must be in [0, 10] A");
    skin = sk;
    vcap = 0;
    if (have_ff && nsys > 0) layout_systems();
  }

  void set_qeq(double swa, double swb, double tol, int imax, int strict) {
    if (!(swb > swa) || !(tol > 0) || imax < 1) throw Error(RX_ERR_INVALID, "fix qeq: need swb > swa, tol > 0, imax >= 1");
    qp.swa = swa;
    qp.swb = swb;
    taper_coeffs(swa, swb, qp.tap);
    qeq_tol = tol;
    qeq_imax = imax;
    qeq_strict = strict;
    drop_graph();
  }

  void require_ff() const { if (!have_ff) throw Error(RX_ERR_STATE, "no force field set"); }
  void require_sys() const {
    if (host_only) throw Error(RX_ERR_STATE, "host-only context (created with device < 0)");
    if (nsys == 0) throw Error(RX_ERR_STATE, "no systems set");
  }

  void set_systems(int n_sys, const int* natoms, const double* origin, const double* box, const int* periodic, const int* types,
                   const int64_t* tags) {
    require_ff();
    if (host_only) throw Error(RX_ERR_STATE, "host-only context (created with device < 0)");
    if (n_sys <= 0 || !natoms || !origin || !box || !types || !tags) throw Error(RX_ERR_INVALID, "set_systems: null or empty input");
    long long total = 0;
    for (int s = 0; s < n_sys; ++s) {
      if (natoms[s] <= 0) throw Error(RX_ERR_INVALID, "every system needs at least one atom");
      total += natoms[s];
    }
    if (total > (1LL << 30)) throw Error(RX_ERR_INVALID, "too many atoms");
    for (long long a = 0; a < total; ++a)
      if (types[a] < 0 || types[a] >= ff.nt) throw Error(RX_ERR_INVALID, "atom " + std::to_string(a) + " has a type outside the force field");
    // the charge-equilibration histories of the previous systems, to carry over by (system index, tag): a caller that
    // re-neighbours or reorders its atoms (fix qeq/reaxff's s_hist/t_hist travel with the atoms) keeps its warm start
    std::vector<double> old_sh, old_th;
    std::vector<long long> old_tag = htag;
    std::vector<int> old_sys = hsys_of;
    const std::vector<SysInfo> old_info = hsys;
    const int old_nsys = nsys;
    if (na > 0 && s_hist.p && static_cast<size_t>(na) == old_tag.size()) {
      old_sh.resize(4 * static_cast<size_t>(na));
      old_th.resize(4 * static_cast<size_t>(na));
      RXCU(cudaMemcpy(old_sh.data(), s_hist.p, sizeof(double) * old_sh.size(), cudaMemcpyDeviceToHost));
      RXCU(cudaMemcpy(old_th.data(), t_hist.p, sizeof(double) * old_th.size(), cudaMemcpyDeviceToHost));
    }
    nsys = n_sys;
    na = static_cast<int>(total);
    hsys.assign(static_cast<size_t>(nsys), SysInfo{});
    huser.clear();
    hsys_of.resize(static_cast<size_t>(na));
    int begin = 0;
    for (int s = 0; s < nsys; ++s) {
      SysInfo& si = hsys[static_cast<size_t>(s)];
      for (int c = 0; c < 3; ++c) si.origin[c] = origin[3 * s + c];
      for (int c = 0; c < 9; ++c) si.L[c] = box[9 * s + c];
      for (int c = 0; c < 3; ++c) si.per[c] = periodic ? (periodic[3 * s + c] != 0) : 1;
      si.begin = begin;
      si.natoms = natoms[s];
      for (int a = 0; a < natoms[s]; ++a) hsys_of[static_cast<size_t>(begin + a)] = s;
      begin += natoms[s];
    }
    sys_of.ensure(static_cast<size_t>(na));
    type.ensure(static_cast<size_t>(na));
    tag.ensure(static_cast<size_t>(na));
    RXCU(cudaMemcpy(sys_of.p, hsys_of.data(), sizeof(int) * na, cudaMemcpyHostToDevice));
    RXCU(cudaMemcpy(type.p, types, sizeof(int) * na, cudaMemcpyHostToDevice));
    static_assert(sizeof(long long) == sizeof(int64_t), "tag width");
    RXCU(cudaMemcpy(tag.p, tags, sizeof(long long) * na, cudaMemcpyHostToDevice));
    x.ensure(static_cast<size_t>(na));
    q.ensure(static_cast<size_t>(na));
    RXCU(cudaMemset(q.p, 0, sizeof(double) * na));
    s_hist.ensure(4 * static_cast<size_t>(na));
    t_hist.ensure(4 * static_cast<size_t>(na));
    htag.assign(tags, tags + na);
    htype.assign(types, types + na);
    {
      std::vector<double> sh(4 * static_cast<size_t>(na), 0.0), th(4 * static_cast<size_t>(na), 0.0);
      if (!old_sh.empty()) {
        std::vector<std::unordered_map<long long, int>> by_sys(static_cast<size_t>(old_nsys));
        for (size_t k = 0; k < old_tag.size(); ++k) by_sys[static_cast<size_t>(old_sys[k])].emplace(old_tag[k], static_cast<int>(k));
        // a system is the same one handed over again (and keeps its atoms' histories) when its index, atom count and
        // lattice are unchanged; otherwise it starts cold
        std::vector<char> same(static_cast<size_t>(nsys), 0);
        for (int sy = 0; sy < std::min(nsys, old_nsys); ++sy) {
          const SysInfo& o = old_info[static_cast<size_t>(sy)];
          bool eq = o.natoms == natoms[sy];
          for (int c = 0; c < 9; ++c) eq = eq && o.L[c] == box[9 * sy + c];
          same[static_cast<size_t>(sy)] = eq ? 1 : 0;
        }
        for (int a = 0; a < na; ++a) {
          const int sy = hsys_of[static_cast<size_t>(a)];
          if (sy >= old_nsys || !same[static_cast<size_t>(sy)]) continue;
          const auto it = by_sys[static_cast<size_t>(sy)].find(htag[static_cast<size_t>(a)]);
          if (it == by_sys[static_cast<size_t>(sy)].end()) continue;
          for (int c = 0; c < 4; ++c) {
            sh[4 * static_cast<size_t>(a) + c] = old_sh[4 * static_cast<size_t>(it->second) + c];
            th[4 * static_cast<size_t>(a) + c] = old_th[4 * static_cast<size_t>(it->second) + c];
          }
        }
      }
      RXCU(cudaMemcpy(s_hist.p, sh.data(), sizeof(double) * sh.size(), cudaMemcpyHostToDevice));
      RXCU(cudaMemcpy(t_hist.p, th.data(), sizeof(double) * th.size(), cudaMemcpyHostToDevice));
    }
    huser = hsys;   // the caller's lattices and origins (non-periodic directions are re-fitted from the positions)
    have_pos = false;
    have_virial = false;
    forces_valid = false;
    acks2_on = false;
    md_ready = false;
    ncap = 0;
    bcap = 0;
    vcap = 0;
    layout_systems();
  }

  // cell grids, search ranges, shift encoding, neighbor capacity estimate
  void layout_systems() {
    drop_graph();
    const double rc0 = ff.nonb_cut;
    if (!(rc0 > 0)) throw Error(RX_ERR_INVALID, "force field has no positive non-bonded cut-off");
    const double rc = rc0 + skin;   // the Verlet radius sets the cell search range and the shift encoding
    if (ctl.bond_cut > rc0 || ctl.hbond_cut > rc0) throw Error(RX_ERR_INVALID, "bond_cut and hbond_cut must not exceed the non-bonded cut-off");
    if (qp.swb > rc0) throw Error(RX_ERR_INVALID, "fix qeq: the taper radius exceeds the force field's nonb_cut (qeq_device.cpp:14)");
    int cell_begin = 0, sm = 1;
    double max_density = 0;
    for (auto& si : hsys) {
      const double* L = si.L;
      const double* a = L; const double* b = L + 3; const double* c = L + 6;
      auto cross = [](const double* u, const double* w, double* o) { o[0] = u[1] * w[2] - u[2] * w[1]; o[1] = u[2] * w[0] - u[0] * w[2]; o[2] = u[0] * w[1] - u[1] * w[0]; };
      double bc[3], ca[3], ab[3];
      cross(b, c, bc); cross(c, a, ca); cross(a, b, ab);
      const double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
      if (!(det > 0) || !std::isfinite(det)) throw Error(RX_ERR_INVALID, "box must be right-handed and non-degenerate");
      for (int k = 0; k < 3; ++k) { si.R[k] = bc[k] / det; si.R[3 + k] = ca[k] / det; si.R[6 + k] = ab[k] / det; }
      const double h[3] = {det / std::sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]), det / std::sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]),
                           det / std::sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2])};
      long long ncell = 1;
      for (int k = 0; k < 3; ++k) si.h[k] = h[k];
      si.ext = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) + std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) +
               std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      {
        auto dotp = [](const double* u, const double* w) { return u[0] * w[0] + u[1] * w[1] + u[2] * w[2]; };
        si.ortho = (dotp(a, b) == 0.0 && dotp(a, c) == 0.0 && dotp(b, c) == 0.0) ? 1 : 0;
      }
      for (int k = 0; k < 3; ++k) {
        int n = static_cast<int>(std::floor(h[k] * 2.0 / rc));
        n = std::max(1, std::min(n, 512));
        si.nc[k] = n;
        const double w = h[k] / n;
        si.range[k] = static_cast<int>(std::ceil(rc / w - 1e-12));
        const int s_lo = (si.range[k] + n - 1) / n;
        const int s_hi = (n - 1 + si.range[k]) / n;
        sm = std::max(sm, std::max(s_lo, s_hi));
        ncell *= n;
      }
      si.cell_begin = cell_begin;
      si.shift_base = 0;
      cell_begin += static_cast<int>(ncell);
      max_density = std::max(max_density, si.natoms / det);
    }
    smax = sm;
    S = 2 * smax + 1;
    // Thresholds of the single-precision candidate test of the Verlet build (rows need only be supersets). With
    // u = 2^-24, each component of the separation (x_j - o) + (L s - (x_i - o)), both terms rounded to single precision
    // and then added, is off by at most delta = u (|x_j - o| + |L s - (x_i - o)| + |dv|) <= u ((2 + smax) ext + R_v)
    // (wrapped coordinates are within ext of the origin, |L s| <= smax ext). For a true distance r <= R the computed
    // r^2 is then at most R^2 (1 + 3u) + 2 sqrt(3) R delta + 3 delta^2: the thresholds exceed that and round up.
    for (auto& si : hsys) {
      const double u = 5.9604644775390625e-8, Rv = rc;
      const double delta = u * 1.001 * ((2.0 + smax) * si.ext + Rv);
      auto thr = [&](double R) {
        const double t = R * R * (1.0 + 6.0 * u) + 3.5 * R * delta + 3.0 * delta * delta;
        float f = static_cast<float>(t);
        if (static_cast<double>(f) < t) f = std::nextafter(f, std::numeric_limits<float>::infinity());
        return f;
      };
      si.vthr[0] = thr(Rv);
      si.vthr[1] = thr((ctl.bond_cut + skin) * (1.0 + 1e-9));
      si.vthr[2] = thr((ctl.hbond_cut + skin) * (1.0 + 1e-9));
      for (int k = 0; k < 3; ++k) { si.inv_nc[k] = 1.0 / si.nc[k]; si.inv_h[k] = 1.0 / si.h[k]; }
      si.inv_ncf0 = 1.0f / static_cast<float>(si.nc[0]);
    }
    const long long nshift = static_cast<long long>(S) * S * S;
    int sbits = 0;
    while ((1LL << sbits) < nshift) ++sbits;
    abits = 32 - sbits;
    if (static_cast<long long>(na) >= (1LL << abits))
      throw Error(RX_ERR_INVALID, "too many atoms for the periodic-image encoding of these boxes");
    ncell_total = cell_begin;
    {  // lattice shift table: for every system and shift index, L.s summed in the reference's order
      const int S3 = S * S * S;
      std::vector<double4> tab(static_cast<size_t>(nsys) * S3);
      for (int si = 0; si < nsys; ++si) {
        SysInfo& sy = hsys[static_cast<size_t>(si)];
        sy.shift_base = si * S3;
        for (int idx = 0; idx < S3; ++idx) {
          const int sv[3] = {idx / (S * S) - smax, (idx / S) % S - smax, idx % S - smax};
          double r[3] = {0.0, 0.0, 0.0};
          for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) r[c] += static_cast<double>(sv[k]) * sy.L[3 * k + c];
          tab[static_cast<size_t>(si) * S3 + idx] = make_double4(r[0], r[1], r[2], 0.0);
        }
      }
      shifts.ensure(tab.size());
      RXCU(cudaMemcpy(shifts.p, tab.data(), sizeof(double4) * tab.size(), cudaMemcpyHostToDevice));
    }
    sys.ensure(static_cast<size_t>(nsys));
    RXCU(cudaMemcpy(sys.p, hsys.data(), sizeof(SysInfo) * nsys, cudaMemcpyHostToDevice));
    cell_key.ensure(static_cast<size_t>(na));
    cell_key_sorted.ensure(static_cast<size_t>(na));
    cell_atoms.ensure(static_cast<size_t>(na));
    xs.ensure(static_cast<size_t>(na));
    atom_iota.ensure(static_cast<size_t>(na));
    cell_start.ensure(static_cast<size_t>(ncell_total) + 1);
    {
      std::vector<int> io(static_cast<size_t>(na));
      for (int a = 0; a < na; ++a) io[static_cast<size_t>(a)] = a;
      RXCU(cudaMemcpy(atom_iota.p, io.data(), sizeof(int) * na, cudaMemcpyHostToDevice));
    }
    key_bits = 1;
    while ((1LL << key_bits) <= ncell_total) ++key_bits;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, cell_key.p, cell_key_sorted.p, atom_iota.p, cell_atoms.p, na, 0, key_bits, stream);
    cub_tmp.ensure(tmp);
    const double expect = 4.0 / 3.0 * M_PI * rc0 * rc0 * rc0 * max_density;
    const int want_ncap = static_cast<int>(std::ceil((expect * 1.3 + 32) / 32.0)) * 32;
    if (ncap < want_ncap) ncap = want_ncap;
    const double expect_v = 4.0 / 3.0 * M_PI * rc * rc * rc * max_density;
    const int want_vcap = static_cast<int>(std::ceil((expect_v * 1.3 + 32) / 32.0)) * 32;
    if (vcap < want_vcap) vcap = want_vcap;
    const double rn = ctl.bond_cut + skin, ra = ctl.hbond_cut + skin;
    const int want_near = static_cast<int>(std::ceil((4.0 / 3.0 * M_PI * rn * rn * rn * max_density * 1.3 + 32) / 32.0)) * 32;
    if (ncap_near < want_near) ncap_near = want_near;
    // acceptors are a fraction of the atoms; the estimate takes half of them and grows on overflow
    const int want_acc = static_cast<int>(std::ceil((4.0 / 3.0 * M_PI * ra * ra * ra * max_density * 0.5 + 32) / 32.0)) * 32;
    if (ncap_acc < want_acc) ncap_acc = want_acc;
    if (bcap < 16) bcap = 16;
    alloc_atoms();
    alloc_lists();
    force_rebuild();
  }

  void alloc_atoms() {
    const size_t n = static_cast<size_t>(na);
    Deltap.ensure(n); Deltap_boc.ensure(n); cdtot.ensure(n); W.ensure(n); eatom.ensure(n * kTerms);
    dDp_self.ensure(n); fown.ensure(n); fdb.ensure(n); fnb.ensure(n); grad.ensure(n);
    aq.ensure(n); census.ensure(n * kCensus);
    nbr_cnt.ensure(n); bcnt.ensure(n); near_cnt.ensure(n); acc_cnt.ensure(n); vcnt.ensure(n); xref.ensure(n);
    sys_flag.ensure(static_cast<size_t>(nsys)); cg_nref.ensure(1); cg_brk.ensure(static_cast<size_t>(nsys));
    energies.ensure(static_cast<size_t>(nsys) * kTerms);
    virial.ensure(static_cast<size_t>(nsys) * kVir);
    {
      int maxn = 1;
      for (const auto& si : hsys) maxn = std::max(maxn, si.natoms);
      echunks = (maxn + 255) / 256;
      epart.ensure(static_cast<size_t>(nsys) * echunks * (kTerms + kVir));
    }
    vir.ensure(n * kVir);
    vir_nb.ensure(n * kVir); vir_h.ensure(n * kVir); vir_t.ensure(n * kVir);
    fown_h.ensure(n); fown_t.ensure(n); fix_h.ensure(3 * n); pe_fix.ensure(n);
    cg_x.ensure(n); cg_df.ensure(n); cg_b.ensure(n); cg_r.ensure(n); cg_d.ensure(n); cg_p.ensure(n); cg_q.ensure(n); cg_eta.ensure(n);
    cg_iters.ensure(2 * static_cast<size_t>(nsys)); cg_rel.ensure(2 * static_cast<size_t>(nsys));
    cg_sys.ensure(nsys); cg_rb0.ensure(n); cg_rb1.ensure(n); cg_nlive.ensure(2);
    cg_part.ensure(16 * static_cast<size_t>(std::max(nsm, 1)) * 32);
  }

  void alloc_lists() {
    drop_graph();
    const size_t n = static_cast<size_t>(na);
    vrow.ensure(n * vcap);
    nbr.ensure(n * ncap);
    hhi.ensure(n * ncap);
    hlo.ensure(n * ncap);
    near.ensure(n * ncap_near);
    acc.ensure(n * ncap_acc);
    const size_t nb = n * bcap;
    bcode.ensure(nb); bsym.ensure(nb);
    bdv.ensure(nb); bBO.ensure(nb); bdBOp.ensure(nb); bdlnpi.ensure(nb); bdlnpi2.ensure(nb);
    bC0.ensure(nb); bC1.ensure(nb); bC2.ensure(nb); bacc.ensure(nb); bfn.ensure(nb);
    bcdbo_h.ensure(nb); bfn_h.ensure(nb); bacc_t.ensure(nb); bfn_t.ensure(nb);
    Tl.ensure(nb * bcap);
    Ti.ensure(nb * bcap);
    Tsum.ensure(2 * nb);
    Tvir.ensure(nb * kVir);
    tflag.ensure(nb);
    tor_list.ensure(nb);
    tor_n.ensure(1);
  }

  Dev dev() {
    Dev d{};
    d.na = na; d.nsys = nsys; d.sys = sys.p; d.sys_of = sys_of.p; d.x = x.p; d.type = type.p; d.tag = tag.p; d.q = q.p;
    d.cell_key = cell_key.p; d.cell_atoms = cell_atoms.p; d.xs = xs.p; d.cell_start = cell_start.p; d.ncell_total = ncell_total;
    d.ncap = ncap; d.nbr = nbr.p; d.nbr_cnt = nbr_cnt.p; d.hhi = hhi.p; d.hlo = hlo.p;
    d.vcap = vcap; d.vrow = vrow.p; d.vcnt = vcnt.p; d.xref = xref.p; d.sys_flag = sys_flag.p;
    d.rv2 = (ff.nonb_cut + skin) * (ff.nonb_cut + skin);
    d.half_skin2 = 0.25 * skin * skin;
    d.abits = abits; d.amask = (abits >= 32) ? 0xffffffffu : ((1u << abits) - 1u); d.smax = smax; d.S = S;
    d.shifts = shifts.p; d.ncap_near = ncap_near; d.near = near.p; d.near_cnt = near_cnt.p;
    d.ncap_acc = ncap_acc; d.acc = acc.p; d.acc_cnt = acc_cnt.p;
    {  // the short Verlet rows (rebuilt with the Verlet rows): supersets of the consumers' exact sqrt(r2) <= cut tests for
       // every position until the next rebuild (each atom moves less than skin/2 meanwhile)
      const double rn = (ctl.bond_cut + skin) * (1.0 + 1e-9), ra = (ctl.hbond_cut + skin) * (1.0 + 1e-9);
      d.rnear2 = rn * rn;
      d.racc2 = ra * ra;
    }
    d.bcap = bcap; d.bcode = bcode.p; d.bsym = bsym.p; d.bcnt = bcnt.p; d.bdv = bdv.p; d.bBO = bBO.p; d.bdBOp = bdBOp.p;
    d.bdlnpi = bdlnpi.p; d.bdlnpi2 = bdlnpi2.p; d.bC0 = bC0.p; d.bC1 = bC1.p; d.bC2 = bC2.p; d.bacc = bacc.p; d.bfn = bfn.p; d.Tl = Tl.p; d.Ti = Ti.p; d.Tsum = Tsum.p; d.Tvir = Tvir.p;
    d.tflag = tflag.p; d.tor_list = tor_list.p; d.tor_n = tor_n.p;
    d.Deltap = Deltap.p; d.Deltap_boc = Deltap_boc.p; d.dDp_self = dDp_self.p; d.aq = aq.p; d.fown = fown.p; d.cdtot = cdtot.p;
    d.W = W.p; d.fdb = fdb.p; d.fnb = fnb.p; d.grad = grad.p; d.eatom = eatom.p; d.vir = vir.p; d.vir_nb = vir_nb.p; d.vir_h = vir_h.p; d.vir_t = vir_t.p;
    d.fown_h = fown_h.p; d.fown_t = fown_t.p; d.fix_h = fix_h.p; d.pe_fix = pe_fix.p; d.pe_on = pe_on; d.bcdbo_h = bcdbo_h.p; d.bfn_h = bfn_h.p; d.bacc_t = bacc_t.p; d.bfn_t = bfn_t.p; d.census = census.p; d.status = status.p;
    d.counters = counters.p;
    return d;
  }

  // ------------------------------------------------------------------ timing
  void tic(int k, const char* name) {
    if (!timing) return;
    while (static_cast<int>(phases.size()) <= k) {
      Phase p{name, nullptr, nullptr, 0.0};
      cudaEventCreate(&p.a);
      cudaEventCreate(&p.b);
      phases.push_back(p);
    }
    phases[static_cast<size_t>(k)].name = name;
    cudaEventRecord(phases[static_cast<size_t>(k)].a, stream);
  }
  void toc(int k) {
    if (!timing) return;
    cudaEventRecord(phases[static_cast<size_t>(k)].b, stream);
  }
  void collect_times() {
    if (!timing) return;
    for (auto& p : phases) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) p.ms += ms;
    }
  }

  // ------------------------------------------------------------------ the force evaluation
  static unsigned blocks(long long n, int per) { return static_cast<unsigned>((n + per - 1) / per); }

  // every system's Verlet rows are rebuilt at the next evaluation (new positions, capacities or cut-offs)
  void force_rebuild() {
    if (nsys > 0) RXCU(cudaMemsetAsync(sys_flag.p, 1, sizeof(int) * nsys, stream));
  }

  // Verlet maintenance + this evaluation's rows (neighbor rows, charge matrix, near rows). The wrap/bin, sort and
  // cell-start kernels run every evaluation but do work only for systems whose flag is set; k_neighbors likewise.
  // While an evaluation is being captured, the rebuild kernels go into the body of a graph conditional that
  // k_rebuild_flag opens only when some system's flag is set: an evaluation that rebuilds nothing skips them (and the
  // radix sort) altogether. Launched one by one (timing, or a runtime without conditionals), they run every
  // evaluation and do work only for the flagged systems.
  bool cond_ok = true;
  void launch_rebuild(const Dev& d, cudaStream_t st) {
    launches += 4;
    k_wrap_bin<<<blocks(na, 256), 256, 0, st>>>(d);
    size_t tmp = cub_tmp.n;
    RXCU(cub::DeviceRadixSort::SortPairs(cub_tmp.p, tmp, cell_key.p, cell_key_sorted.p, atom_iota.p, cell_atoms.p, na, 0, key_bits, st));
    k_cell_start<<<blocks(na + 1, 256), 256, 0, st>>>(d, cell_key_sorted.p);
    k_neighbors<<<blocks(static_cast<long long>(na) * 32, 128), 128, 0, st>>>(d, dff);
  }
  void build_lists(const Dev& d) {
    build_rows(d);
    launch_pairs(d);
  }
  // the Verlet check and, where some system is flagged, the rebuild of its rows (the bonded chain needs only these)
  void build_rows(const Dev& d) {
    tic(0, "neighbors");
    ++launches;
    k_nbr_check<<<blocks(na, 256), 256, 0, stream>>>(d);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cond_ok && !timing) RXCU(cudaStreamIsCapturing(stream, &cs));
    if (cs == cudaStreamCaptureStatusActive) {
      cudaGraph_t g = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      RXCU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, &deps, &nd));
      cudaGraphConditionalHandle h;
      RXCU(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
      ++launches;
      k_rebuild_flag<<<1, 256, 0, stream>>>(d, h);
      RXCU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, &deps, &nd));
      cudaGraphNodeParams p{};
      p.type = cudaGraphNodeTypeConditional;
      p.conditional.handle = h;
      p.conditional.type = cudaGraphCondTypeIf;
      p.conditional.size = 1;
      cudaGraphNode_t node = nullptr;
      RXCU(cudaGraphAddNode(&node, g, deps, nd, &p));
      RXCU(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
      RXCU(cudaStreamBeginCaptureToGraph(side_c, p.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      launch_rebuild(d, side_c);
      cudaGraph_t body = nullptr;
      RXCU(cudaStreamEndCapture(side_c, &body));
    } else {
      launch_rebuild(d, stream);
    }
  }
  // the per-step exact filter of the Verlet rows into the neighbor rows and the charge matrix
  void launch_pairs(const Dev& d) {
    ++launches;
    k_pairs<<<blocks(static_cast<long long>(na) * 32, tune.tpb_pairs), tune.tpb_pairs, 0, stream>>>(d, dff, qp);
    toc(0);
  }

  CgArgs cg_args() {
    CgArgs a{};
    a.imax = qeq_imax; a.tol = qeq_tol;
    a.x = cg_x.p; a.b = cg_b.p; a.r = cg_r.p; a.d = cg_d.p; a.p = cg_p.p; a.q = cg_q.p; a.df = cg_df.p; a.eta = cg_eta.p; a.part = cg_part.p;
    a.out_iters = cg_iters.p; a.out_rel = cg_rel.p; a.out_nref = cg_nref.p; a.out_brk = cg_brk.p; a.write_q = 1;
    return a;
  }

  // Launch shapes (atoms per block of the warp-per-atom and thread-per-atom kernels, the size above which a lone
  // system takes the single-system CG): none changes a result bit, so rx_autotune may pick them by measurement.
  struct Tune {
    int tpb_pairs = 128, tpb_nb = 128, tpb_hb = 128, tpb_bonds = 128, tpb_atom = 64;
    int lone_grid_min = 4096;
    int overlap = 1;   // bonded chain beside the charge solve
    // threads per SM of the single-system CG in units of 256 (1-4; 0: four), launched as one block per SM. Two leave
    // half of every SM to the bonded terms that run beside the solve: on the 24,000-atom water step the solve alone
    // is slower, the step faster. One block per SM rather than several smaller ones halves the blocks that meet at
    // each grid barrier. The setting changes the CG's summation order, so it is one value for every solve of the
    // context.
    int cg_per_sm = 2;
  } tune;
  int grid_occ[5] = {0, 0, 0, 0, 0}, seg_per_sm = 0;
  void launch_cg(const Dev& d, CgArgs a) {
    if (nsys == 1 && na > tune.lone_grid_min) {   // one large system: all SMs on its rows, block partials in block order
      const int units = tune.cg_per_sm > 0 ? std::min(tune.cg_per_sm, 4) : 4;
      const int threads = 256 * units;
      if (!grid_occ[units]) RXCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid_occ[units], k_cg_grid, threads, 0));
      if (grid_occ[units] < 1) throw Error(RX_ERR_CUDA, "the single-system CG block does not fit on an SM");
      int grid = std::max(1, std::min(nsm, (na + (threads / 32) - 1) / (threads / 32)));
      a.begin = 0;
      a.n = na;
      void* args[] = {const_cast<Dev*>(&d), &a};
      ++launches;
      RXCU(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cg_grid), dim3(grid), dim3(threads), args, 0, stream));
    } else {   // a batch (or one small system): every row of every system on all SMs, per-system fixed-order sums
      const int threads = 256;
      if (!seg_per_sm) RXCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&seg_per_sm, k_cg_seg, threads, 0));
      int grid = std::max(1, std::min(seg_per_sm * nsm, (na + (threads / 32) - 1) / (threads / 32)));
      grid = std::min(grid, nsm * 32);
      a.sc = cg_sys.p; a.rb0 = cg_rb0.p; a.rb1 = cg_rb1.p; a.nlive = cg_nlive.p;
      RXCU(cudaMemsetAsync(cg_sys.p, 0, sizeof(SysCg) * nsys, stream));
      RXCU(cudaMemsetAsync(cg_nlive.p, 0, 2 * sizeof(int), stream));
      void* args[] = {const_cast<Dev*>(&d), &a};
      ++launches;
      RXCU(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cg_seg), dim3(grid), dim3(threads), args, 0, stream));
    }
  }

  // charges: guesses from the histories, the CG, q, and the history shift (skipped by the kernel after a failure)
  void launch_qeq(const Dev& d) {
    tic(1, "qeq");
    CgArgs a = cg_args();
    ++launches;
    k_qeq_prepare<<<blocks(na, 256), 256, 0, stream>>>(d, dff, a, s_hist.p, t_hist.p);
    launch_cg(d, a);
    ++launches;
    k_qeq_history<<<blocks(na, 256), 256, 0, stream>>>(d, cg_x.p, s_hist.p, t_hist.p, qeq_strict);
    toc(1);
  }

  // After the Verlet check and rebuild, the bonded chain (bond orders, then k_bonded_atom, with the H-bonds on `side_h`
  // and the torsions on `side_t`, then the bonded gathers k_fold and k_dbond) needs neither the neighbor rows nor the
  // charges, so with tune.overlap it runs on `side` next to the row filter and the charge solve; the non-bonded pairs follow the charges on `stream`, and k_force_final joins both. Each branch writes its own arrays (fnb, vir_nb; bacc/bfn/fown; *_h; *_t, Tl), and
  // all join before the gathers, which add them in fixed order, so the schedule changes no result bit. With timing
  // on, every branch runs on `stream`, one after the other, so each phase is timed alone.
  void launch_bonded(const Dev& d) {
    const bool conc = !timing;
    cudaStream_t bs = conc ? side : stream, hs = conc ? side_h : stream, ts = conc ? side_t : stream;
    if (conc) {
      RXCU(cudaEventRecord(ev_fork, stream));
      RXCU(cudaStreamWaitEvent(side, ev_fork, 0));
    }
    tic(2, "bond_orders");
    launches += 4;
    k_bonds<<<blocks(static_cast<long long>(na) * 32, tune.tpb_bonds), tune.tpb_bonds, 0, bs>>>(d, dff, ctl);
    k_bond_sym<<<blocks(static_cast<long long>(na) * bcap, 256), 256, 0, bs>>>(d);
    k_bo_correct<<<blocks(static_cast<long long>(na) * bcap, 256), 256, 0, bs>>>(d, dff, ctl);
    k_atom_quantities<<<blocks(na, 128), 128, 0, bs>>>(d, dff);
    toc(2);
    if (conc) {
      RXCU(cudaEventRecord(ev_fork2, bs));
      RXCU(cudaStreamWaitEvent(side_h, ev_fork2, 0));
      RXCU(cudaStreamWaitEvent(side_t, ev_fork2, 0));
    }
    tic(3, "bonded_terms");
    launches += 2;
    k_bonded_atom<<<blocks(na, tune.tpb_atom), tune.tpb_atom, 0, bs>>>(d, dff, ctl);
    k_hbond<<<blocks(static_cast<long long>(na) * 32, tune.tpb_hb), tune.tpb_hb, 0, hs>>>(d, dff, ctl);
    toc(3);
    tic(4, "torsion");
    ++launches;
    // at most one listed slot per bond (the tag-order end): half the slots bound the list
    k_torsion<<<blocks((static_cast<long long>(na) * bcap + 1) / 2, tune.tpb_atom), tune.tpb_atom, 0, ts>>>(d, dff, ctl);
    toc(4);
    // the bonded gathers need the H-bond and torsion branches but no charge or non-bonded result: they stay on the
    // bonded branch, so only k_force_final follows the non-bonded pairs
    if (conc) {
      RXCU(cudaEventRecord(ev_join_h, side_h));
      RXCU(cudaEventRecord(ev_join_t, side_t));
      RXCU(cudaStreamWaitEvent(bs, ev_join_h, 0));
      RXCU(cudaStreamWaitEvent(bs, ev_join_t, 0));
    }
    tic(6, "gather");
    launches += 2;
    k_fold<<<blocks(na, 128), 128, 0, bs>>>(d);
    k_dbond<<<blocks(na, 128), 128, 0, bs>>>(d);
    toc(6);
    if (conc) RXCU(cudaEventRecord(ev_join, bs));
  }

  void launch_nonbonded(const Dev& d) {
    tic(5, "nonbonded");
    ++launches;
    // each pair once (the partner's share through the fixed-point accumulator), except when the per-atom split of
    // energies and virials is wanted
    if (pe_on) k_nonbonded<<<blocks(static_cast<long long>(na) * 32, tune.tpb_nb), tune.tpb_nb, 0, stream>>>(d, dff);
    else k_nonbonded_half<<<blocks(static_cast<long long>(na) * 32, tune.tpb_nb), tune.tpb_nb, 0, stream>>>(d, dff);
    if (acks2_on) {
      ++launches;
      k_acks2<<<blocks(static_cast<long long>(na) * 32, 128), 128, 0, stream>>>(d, dff, s_kin.p);
    }
    toc(5);
  }

  void launch_gathers(const Dev& d) {
    if (!timing) RXCU(cudaStreamWaitEvent(stream, ev_join, 0));
    tic(7, "force_final");
    ++launches;
    k_force_final<<<blocks(na, 128), 128, 0, stream>>>(d);
    toc(7);
  }

  // One evaluation of every system, enqueued without any host synchronisation: kernels after a failure (a list
  // overflow) return at once; the host reads the status word when it next synchronises. Without tune.overlap the
  // bonded chain is forked after the charges instead (the non-bonded pairs then run beside it).
  void enqueue_eval(bool do_qeq) {
    const Dev d = dev();
    build_rows(d);
    if (tune.overlap && !timing) {
      // the bonded chain forks off before the row filter: it reads only the short rows and the positions
      launch_bonded(d);
      launch_pairs(d);
      if (do_qeq) launch_qeq(d);
    } else if (tune.overlap) {
      launch_pairs(d);
      launch_bonded(d);
      if (do_qeq) launch_qeq(d);
    } else {
      launch_pairs(d);
      if (do_qeq) launch_qeq(d);
      launch_bonded(d);
    }
    launch_nonbonded(d);
    launch_gathers(d);
  }

  // grow the capacities from a status word with overflow bits; false if nothing overflowed
  bool grow_from_status(const int* st, int attempt) {
    if (!(st[0] & (ST_NBR_OVERFLOW | ST_BOND_OVERFLOW | ST_NEAR_OVERFLOW | ST_VERLET_OVERFLOW | ST_ACC_OVERFLOW))) return false;
    if (attempt >= 4) throw Error(RX_ERR_CAPACITY, "list capacity still exceeded after 4 grow attempts");
    if (st[0] & ST_NBR_OVERFLOW) ncap = ((st[1] * 5 / 4) + 31) / 32 * 32;
    if (st[0] & ST_NEAR_OVERFLOW) ncap_near = ((st[3] * 5 / 4) + 31) / 32 * 32;
    if (st[0] & ST_ACC_OVERFLOW) ncap_acc = ((st[5] * 5 / 4) + 31) / 32 * 32;
    if (st[0] & ST_VERLET_OVERFLOW) vcap = ((st[4] * 5 / 4) + 31) / 32 * 32;
    if (st[0] & ST_BOND_OVERFLOW) bcap = std::max(bcap, ((st[2] * 5 / 4) + 3) / 4 * 4);
    alloc_lists();
    return true;
  }

  void check_status(const int* st, bool do_qeq) {
    if (st[0] & ST_SHIFT_RANGE) throw Error(RX_ERR_INVALID, "a periodic image outside the shift encoding was requested");
    if (st[0] & ST_NONFINITE) throw Error(RX_ERR_INVALID, "non-finite coordinate");
    if (st[0] & ST_NONPERIODIC_ESCAPE)
      throw Error(RX_ERR_INVALID, "an atom left the extent laid out for a non-periodic direction; set the positions again");
    if (st[0] & ST_SYM_MISSING) throw Error(RX_ERR_INVALID, "inconsistent bond list (a bond without its reverse)");
    if (do_qeq) {
      if (st[0] & ST_CG_BREAKDOWN) throw Error(RX_ERR_NOT_CONVERGED, "charge equilibration: CG breakdown");
      if (qeq_strict && (st[0] & ST_CG_NOTCONV))
        throw Error(RX_ERR_NOT_CONVERGED, "charge equilibration did not converge within " + std::to_string(qeq_imax) + " iterations");
      finish_qeq();
    }
  }

  void fetch_qeq_counts() {
    last_iters.resize(2 * static_cast<size_t>(nsys));
    last_rel.resize(2 * static_cast<size_t>(nsys));
    RXCU(cudaMemcpyAsync(last_iters.data(), cg_iters.p, sizeof(int) * 2 * nsys, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaMemcpyAsync(last_rel.data(), cg_rel.p, sizeof(double) * 2 * nsys, cudaMemcpyDeviceToHost, stream));
  }

  // One force evaluation of every system, with grow-and-retry of the list capacities (neighbor.cpp:362-374,
  // bonded_device.cpp:117-190). With `do_qeq` the charges are equilibrated first and the histories advanced on success.
  void evaluate(bool do_qeq) { evaluate_with(do_qeq, [] {}); }

  // `tail` enqueues work ordered after the evaluation (result sums and copies into pinned memory); it is repeated with
  // the evaluation when the lists are regrown, and the one synchronisation waits for both
  template <class Tail>
  void evaluate_with(bool do_qeq, Tail&& tail) {
    require_ff();
    require_sys();
    if (!have_pos) throw Error(RX_ERR_STATE, "no positions set");
    const size_t n2 = 2 * static_cast<size_t>(nsys);
    char* sm = small_stage(sizeof(int) * (kStatusWords + n2) + sizeof(double) * n2);
    int* st = reinterpret_cast<int*>(sm);
    int* it = st + kStatusWords;
    double* rl = reinterpret_cast<double*>(sm + sizeof(int) * (kStatusWords + n2));
    for (int attempt = 0;; ++attempt) {
      RXCU(cudaMemsetAsync(status.p, 0, sizeof(int) * kStatusWords, stream));
      const int gi = do_qeq ? 1 : 0;
      if (graphs_ok && !timing && !eval_graph[gi]) capture_retry(eval_graph[gi], eval_launches[gi], [&] { enqueue_eval(do_qeq); });
      if (graphs_ok && !timing && eval_graph[gi]) {
        RXCU(cudaGraphLaunch(eval_graph[gi], stream));
        launches += eval_launches[gi];
      } else {
        enqueue_eval(do_qeq);
      }
      if (do_qeq) {
        RXCU(cudaMemcpyAsync(it, cg_iters.p, sizeof(int) * n2, cudaMemcpyDeviceToHost, stream));
        RXCU(cudaMemcpyAsync(rl, cg_rel.p, sizeof(double) * n2, cudaMemcpyDeviceToHost, stream));
      }
      tail();
      RXCU(cudaMemcpyAsync(st, status.p, sizeof(int) * kStatusWords, cudaMemcpyDeviceToHost, stream));
      RXCU(cudaStreamSynchronize(stream));
      RXCU(cudaGetLastError());
      if (do_qeq) {
        last_iters.assign(it, it + n2);
        last_rel.assign(rl, rl + n2);
      }
      if (grow_from_status(st, attempt)) {
        force_rebuild();
        continue;
      }
      check_status(st, do_qeq);
      break;
    }
    forces_valid = true;
    collect_times();
  }

  void finish_qeq() {   // the counts were copied back with the status word
    if (qeq_strict)
      for (size_t k = 0; k < last_rel.size(); ++k)
        if (!(last_rel[k] <= qeq_tol))
          throw Error(RX_ERR_NOT_CONVERGED, "charge equilibration did not converge after " + std::to_string(qeq_imax) +
                                                " iterations (relative residual " + std::to_string(last_rel[k]) + ")");
  }

  bool have_virial = false;
  bool forces_valid = false;   // the gradient buffer holds the forces of the current positions and systems
  void energy_sums() {
    have_virial = true;
    launches += 2;
    const Dev d = dev();
    k_energy_part<<<dim3(nsys, echunks), 256, 0, stream>>>(d, epart.p, echunks);
    k_energy_final<<<nsys, 32 * (kTerms + kVir), 0, stream>>>(d, epart.p, echunks, energies.p, virial.p);
  }

  // ------------------------------------------------------------------ autotuning
  // Times every candidate launch shape of the tunable kernels on the current systems (CUDA events around `reps`
  // launches each, after one full evaluation that makes their inputs current) and keeps the fastest; then evaluates
  // again so that every array is consistent. Returns the chosen shapes.
  void autotune(int reps, int* out) {
    require_ff();
    require_sys();
    if (!have_pos) throw Error(RX_ERR_STATE, "no positions set");
    if (reps < 1) reps = 3;
    const bool tm = timing;
    timing = false;
    evaluate(true);
    const Dev d = dev();
    cudaEvent_t a, b;
    RXCU(cudaEventCreate(&a));
    RXCU(cudaEventCreate(&b));
    auto time_it = [&](auto&& launch) {
      launch();   // warm
      RXCU(cudaEventRecord(a, stream));
      for (int r = 0; r < reps; ++r) launch();
      RXCU(cudaEventRecord(b, stream));
      RXCU(cudaEventSynchronize(b));
      float ms = 0.f;
      RXCU(cudaEventElapsedTime(&ms, a, b));
      return ms;
    };
    const long long nw = static_cast<long long>(na) * 32;
    auto pick = [&](int* slot, std::initializer_list<int> cands, auto&& launch_with) {
      float best = 1e30f;
      int arg = *slot;
      for (int t : cands) {
        const float ms = time_it([&] { launch_with(t); });
        if (ms < best) { best = ms; arg = t; }
      }
      *slot = arg;
    };
    pick(&tune.tpb_pairs, {64, 128, 256}, [&](int t) { k_pairs<<<blocks(nw, t), t, 0, stream>>>(d, dff, qp); });
    pick(&tune.tpb_bonds, {64, 128, 256}, [&](int t) { k_bonds<<<blocks(nw, t), t, 0, stream>>>(d, dff, ctl); });
    pick(&tune.tpb_nb, {64, 128, 256}, [&](int t) {   // the non-bonded kernel the evaluations take
      if (pe_on) k_nonbonded<<<blocks(nw, t), t, 0, stream>>>(d, dff);
      else k_nonbonded_half<<<blocks(nw, t), t, 0, stream>>>(d, dff);
    });
    pick(&tune.tpb_hb, {64, 128, 256}, [&](int t) { k_hbond<<<blocks(nw, t), t, 0, stream>>>(d, dff, ctl); });
    pick(&tune.tpb_atom, {32, 64, 128}, [&](int t) {
      k_bonded_atom<<<blocks(na, t), t, 0, stream>>>(d, dff, ctl);
      k_torsion<<<blocks((static_cast<long long>(na) * bcap + 1) / 2, t), t, 0, stream>>>(d, dff, ctl);
    });
    RXCU(cudaEventDestroy(a));
    RXCU(cudaEventDestroy(b));
    RXCU(cudaGetLastError());
    drop_graph();
    timing = tm;
    evaluate(true);
    if (out) { out[0] = tune.tpb_pairs; out[1] = tune.tpb_bonds; out[2] = tune.tpb_nb; out[3] = tune.tpb_hb; out[4] = tune.tpb_atom; }
  }

  void set_tuning(int key, int value) {
    auto check = [&](bool ok) { if (!ok) throw Error(RX_ERR_INVALID, "tuning value out of range"); };
    switch (key) {
      case RX_TUNE_PAIRS_TPB: check(value == 64 || value == 128 || value == 256); tune.tpb_pairs = value; break;
      case RX_TUNE_BONDS_TPB: check(value == 64 || value == 128 || value == 256); tune.tpb_bonds = value; break;
      case RX_TUNE_NONBONDED_TPB: check(value == 64 || value == 128 || value == 256); tune.tpb_nb = value; break;
      case RX_TUNE_HBOND_TPB: check(value == 64 || value == 128 || value == 256); tune.tpb_hb = value; break;
      case RX_TUNE_ATOM_TPB: check(value == 32 || value == 64 || value == 128); tune.tpb_atom = value; break;
      case RX_TUNE_LONE_GRID_MIN: check(value >= 0); tune.lone_grid_min = value; break;
      case RX_TUNE_OVERLAP: check(value == 0 || value == 1); tune.overlap = value; break;
      case RX_TUNE_CG_BLOCKS_PER_SM: check(value >= 0 && value <= 4); tune.cg_per_sm = value; break;
      default: throw Error(RX_ERR_INVALID, "unknown tuning key");
    }
    drop_graph();
  }

  // ------------------------------------------------------------------ state I/O
  // Non-periodic directions (Box::periodic, include/reaxmetal/system.hpp:29): the engine lays the system out in a
  // lattice whose vector along such a direction is stretched to the atoms' extent plus rc + skin + kNpPad on both
  // sides, so that no periodic image along it comes within the cut-offs, and atoms are never wrapped along it. An atom
  // that later leaves that extent stops the evaluation (set the positions again to re-fit).
  static constexpr double kNpPad = 50.0;
  void fit_nonperiodic(const double* xin, int sys_from = 0) {
    bool any = false;
    for (int sy = sys_from; sy < nsys; ++sy) {
      const SysInfo& u = huser[static_cast<size_t>(sy)];
      SysInfo& si = hsys[static_cast<size_t>(sy)];
      if (u.per[0] && u.per[1] && u.per[2]) continue;
      any = true;
      // fractional coordinates in the caller's lattice
      const double* L = u.L;
      double R[9];
      {
        const double* a = L; const double* b = L + 3; const double* c = L + 6;
        const double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
        const double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
        const double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
        if (!(det > 0) || !std::isfinite(det)) throw Error(RX_ERR_INVALID, "box must be right-handed and non-degenerate");
        for (int k = 0; k < 3; ++k) { R[k] = bc[k] / det; R[3 + k] = ca[k] / det; R[6 + k] = ab[k] / det; }
        const double hk[3] = {det / std::sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]), det / std::sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]),
                              det / std::sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2])};
        for (int c2 = 0; c2 < 3; ++c2) si.origin[c2] = u.origin[c2];
        for (int c2 = 0; c2 < 9; ++c2) si.L[c2] = u.L[c2];
        const double reach = ff.nonb_cut + skin + kNpPad;
        for (int k = 0; k < 3; ++k) {
          if (u.per[k]) continue;
          double fmin = HUGE_VAL, fmax = -HUGE_VAL;
          for (int a2 = u.begin; a2 < u.begin + u.natoms; ++a2) {
            const double* r = xin + 3 * static_cast<size_t>(a2);
            const double f = R[3 * k] * (r[0] - u.origin[0]) + R[3 * k + 1] * (r[1] - u.origin[1]) + R[3 * k + 2] * (r[2] - u.origin[2]);
            if (!std::isfinite(f)) throw Error(RX_ERR_INVALID, "non-finite coordinate");
            fmin = std::min(fmin, f);
            fmax = std::max(fmax, f);
          }
          const double m = reach / hk[k];                 // margin in the caller's fractional units
          const double scale = (fmax - fmin) + 2.0 * m;   // new length along k in units of the caller's vector
          const double t = fmin - m;
          for (int c2 = 0; c2 < 3; ++c2) {
            si.origin[c2] += t * L[3 * k + c2];
            si.L[3 * k + c2] = scale * L[3 * k + c2];
          }
        }
      }
    }
    if (any) layout_systems();
  }

  // a caller array in page-locked memory is copied from and into directly (the layout change runs on the device);
  // pageable arrays go through the context's own pinned staging buffer
  static bool is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
      (void)cudaGetLastError();
      return false;
    }
    return at.type == cudaMemoryTypeHost;
  }
  DBuf<double> xyz3;   // device scratch in the caller's 3-per-atom layout

  void set_positions(const double* xin) {
    require_sys();
    fit_nonperiodic(xin);
    if (is_pinned(xin)) {
      xyz3.ensure(3 * static_cast<size_t>(na));
      RXCU(cudaMemcpyAsync(xyz3.p, xin, sizeof(double) * 3 * na, cudaMemcpyHostToDevice, stream));
      ++launches;
      k_unpack3<<<blocks(na, 256), 256, 0, stream>>>(na, xyz3.p, x.p);
    } else {
      double4* h = stage(static_cast<size_t>(na));
      for (int a = 0; a < na; ++a) h[a] = make_double4(xin[3 * a], xin[3 * a + 1], xin[3 * a + 2], 0.0);
      RXCU(cudaMemcpyAsync(x.p, h, sizeof(double4) * na, cudaMemcpyHostToDevice, stream));
    }
    // no forced rebuild: the next evaluation's Verlet check moves every atom to the periodic image of the engine's
    // rows and rebuilds the systems whose atoms moved more than skin/2 (or whose layout fit_nonperiodic changed)
    RXCU(cudaStreamSynchronize(stream));
    have_pos = true;
    forces_valid = false;
  }
  void get_positions(double* xout) {
    require_sys();
    std::vector<double4> h(static_cast<size_t>(na));
    RXCU(cudaMemcpyAsync(h.data(), x.p, sizeof(double4) * na, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaStreamSynchronize(stream));
    for (int a = 0; a < na; ++a) { xout[3 * a] = h[a].x; xout[3 * a + 1] = h[a].y; xout[3 * a + 2] = h[a].z; }
  }

  void compute(int flags, double* e_out, double* g_out, int32_t* cen_out, int64_t* counts) {
    if ((flags & RX_COMPUTE_QEQ) && (flags & RX_COMPUTE_QEQ_COLD)) {   // a fresh single point: CG from s = t = 0
      RXCU(cudaMemsetAsync(s_hist.p, 0, sizeof(double) * 4 * static_cast<size_t>(na), stream));
      RXCU(cudaMemsetAsync(t_hist.p, 0, sizeof(double) * 4 * static_cast<size_t>(na), stream));
    }
    const int want_pe = (flags & RX_COMPUTE_PERATOM) ? 1 : 0;
    if (want_pe != pe_on) {   // the tallies are a kernel argument: a captured evaluation holds the old value
      pe_on = want_pe;
      drop_graph();
    }
    const bool g_pinned = g_out && is_pinned(g_out);
    double4* g = g_out && !g_pinned ? stage(static_cast<size_t>(na)) : nullptr;
    if (g_pinned) xyz3.ensure(3 * static_cast<size_t>(na));
    double* eh = nullptr;
    evaluate_with((flags & RX_COMPUTE_QEQ) != 0, [&] {
      // the gradient's layout change and copy run on `side` (idle once the evaluation has joined) while `stream` sums
      // the energies and copies them; `stream` waits for the copy before the status word is read
      const bool fork = g || g_pinned;
      cudaStream_t gs = fork ? side : stream;
      if (fork) {
        RXCU(cudaEventRecord(ev_tail, stream));
        RXCU(cudaStreamWaitEvent(side, ev_tail, 0));
      }
      if (g) RXCU(cudaMemcpyAsync(g, grad.p, sizeof(double4) * na, cudaMemcpyDeviceToHost, gs));
      if (g_pinned) {
        ++launches;
        k_pack3<<<blocks(na, 256), 256, 0, gs>>>(na, grad.p, xyz3.p);
        RXCU(cudaMemcpyAsync(g_out, xyz3.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, gs));
      }
      energy_sums();
      if (e_out) {
        eh = energy_stage(static_cast<size_t>(kTerms) * nsys);
        RXCU(cudaMemcpyAsync(eh, energies.p, sizeof(double) * kTerms * nsys, cudaMemcpyDeviceToHost, stream));
      }
      if (fork) {
        RXCU(cudaEventRecord(ev_tail_done, side));
        RXCU(cudaStreamWaitEvent(stream, ev_tail_done, 0));
      }
    });
    have_peratom = pe_on != 0;
    if (e_out) std::copy(eh, eh + static_cast<size_t>(kTerms) * nsys, e_out);
    if (cen_out) RXCU(cudaMemcpyAsync(cen_out, census.p, sizeof(int) * kCensus * na, cudaMemcpyDeviceToHost, stream));
    std::vector<int> nb, bc;
    if (counts) {
      nb.resize(static_cast<size_t>(na));
      bc.resize(static_cast<size_t>(na));
      RXCU(cudaMemcpyAsync(nb.data(), nbr_cnt.p, sizeof(int) * na, cudaMemcpyDeviceToHost, stream));
      RXCU(cudaMemcpyAsync(bc.data(), bcnt.p, sizeof(int) * na, cudaMemcpyDeviceToHost, stream));
    }
    if (cen_out || counts) RXCU(cudaStreamSynchronize(stream));
    if (g)
      for (int a = 0; a < na; ++a) { g_out[3 * a] = g[a].x; g_out[3 * a + 1] = g[a].y; g_out[3 * a + 2] = g[a].z; }
    if (counts) {
      long long sb = 0, sn = 0;
      for (int a = 0; a < na; ++a) { sb += bc[a]; sn += nb[a]; }
      std::vector<int> cen(static_cast<size_t>(kCensus) * na);
      RXCU(cudaMemcpy(cen.data(), census.p, sizeof(int) * kCensus * na, cudaMemcpyDeviceToHost));
      long long pairs = 0, hb = 0;
      for (int a = 0; a < na; ++a) { pairs += cen[4 * static_cast<size_t>(na) + a]; hb += cen[3 * static_cast<size_t>(na) + a]; }
      counts[0] = sb / 2;
      counts[1] = pairs;
      counts[2] = sn;
      counts[3] = hb;
    }
  }

  // the pair side of fix acks2/reaxff: kinetic potentials per atom (NULL switches the terms off)
  bool acks2_on = false;
  DBuf<double> s_kin;
  void set_acks2(const double* sk) {
    require_sys();
    drop_graph();
    acks2_on = sk != nullptr;
    if (!sk) return;
    s_kin.ensure(static_cast<size_t>(na));
    RXCU(cudaMemcpy(s_kin.p, sk, sizeof(double) * na, cudaMemcpyHostToDevice));
  }

  void qeq_reset() {
    require_sys();
    RXCU(cudaMemsetAsync(s_hist.p, 0, sizeof(double) * 4 * static_cast<size_t>(na), stream));
    RXCU(cudaMemsetAsync(t_hist.p, 0, sizeof(double) * 4 * static_cast<size_t>(na), stream));
    RXCU(cudaStreamSynchronize(stream));
  }

  // per-atom energies (the reference's tally rules, src/cpu/bonded.cpp:210-710, nonbonded.cpp:50-76) and per-atom
  // virials (the virial of every interaction kept by the atom it is centred on: pairs and bonds half each) of the last
  // rx_compute with RX_COMPUTE_PERATOM
  bool have_peratom = false;
  void get_peratom(double* eatom_out, double* vatom_out) {
    require_sys();
    if (!have_peratom) throw Error(RX_ERR_STATE, "no evaluation with RX_COMPUTE_PERATOM yet");
    if (eatom_out) {
      std::vector<unsigned long long> h(static_cast<size_t>(na));
      RXCU(cudaMemcpy(h.data(), pe_fix.p, sizeof(unsigned long long) * na, cudaMemcpyDeviceToHost));
      for (int a = 0; a < na; ++a) eatom_out[a] = static_cast<double>(static_cast<long long>(h[static_cast<size_t>(a)])) / 4294967296.0;
    }
    if (vatom_out) {
      const size_t m = static_cast<size_t>(na) * kVir;
      std::vector<double> v1(m), v2(m), v3(m), v4(m);
      RXCU(cudaMemcpy(v1.data(), vir.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
      RXCU(cudaMemcpy(v2.data(), vir_h.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
      RXCU(cudaMemcpy(v3.data(), vir_t.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
      RXCU(cudaMemcpy(v4.data(), vir_nb.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < m; ++k) vatom_out[k] = ((v1[k] + v2[k]) + v3[k]) + v4[k];
    }
  }

  // the bond table of the last evaluation (BondTable, include/reaxmetal/bonded.hpp:32-37): bonds of atom a at
  // [start[a], start[a+1]), partner owner index and lattice shift, corrected bond order; total bond order and lone pairs
  // per atom. Returns the number of bonds (the capacity needed when `cap` is too small).
  long long get_bonds(int* start, int* partner, int* shift3, double* bo, double* total_bo, double* nlp, long long cap) {
    require_sys();
    if (!forces_valid) throw Error(RX_ERR_STATE, "no force evaluation of the current positions");
    const size_t n = static_cast<size_t>(na), nb = n * bcap;
    std::vector<int> cnt(n);
    RXCU(cudaMemcpy(cnt.data(), bcnt.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    long long total = 0;
    for (size_t a = 0; a < n; ++a) total += std::min(cnt[a], bcap);
    if (!start || total > cap) return total;
    std::vector<unsigned> code(nb);
    std::vector<double4> bov(nb);
    std::vector<AtomQ> aqh(n);
    RXCU(cudaMemcpy(code.data(), bcode.p, sizeof(unsigned) * nb, cudaMemcpyDeviceToHost));
    RXCU(cudaMemcpy(bov.data(), bBO.p, sizeof(double4) * nb, cudaMemcpyDeviceToHost));
    RXCU(cudaMemcpy(aqh.data(), aq.p, sizeof(AtomQ) * n, cudaMemcpyDeviceToHost));
    const unsigned amask = (abits >= 32) ? 0xffffffffu : ((1u << abits) - 1u);
    long long k = 0;
    for (size_t a = 0; a < n; ++a) {
      start[a] = static_cast<int>(k);
      for (int s2 = 0; s2 < std::min(cnt[a], bcap); ++s2, ++k) {
        const unsigned c = code[a * bcap + s2];
        if (partner) partner[k] = static_cast<int>(c & amask);
        if (shift3) {
          const int sidx = static_cast<int>(c >> abits);
          shift3[3 * k] = sidx / (S * S) - smax;
          shift3[3 * k + 1] = (sidx / S) % S - smax;
          shift3[3 * k + 2] = sidx % S - smax;
        }
        if (bo) bo[k] = bov[a * bcap + s2].x;
      }
      if (total_bo) total_bo[a] = aqh[a].total_bo;
      if (nlp) nlp[a] = aqh[a].nlp;
    }
    start[n] = static_cast<int>(k);
    return total;
  }

  void get_gradient(double* g_out) {
    require_sys();
    if (!have_virial) throw Error(RX_ERR_STATE, "no force evaluation yet");
    double4* g = stage(static_cast<size_t>(na));
    RXCU(cudaMemcpyAsync(g, grad.p, sizeof(double4) * na, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaStreamSynchronize(stream));
    for (int a = 0; a < na; ++a) { g_out[3 * a] = g[a].x; g_out[3 * a + 1] = g[a].y; g_out[3 * a + 2] = g[a].z; }
  }

  void get_virial(double* out) {
    require_sys();
    if (!have_virial) throw Error(RX_ERR_STATE, "no force evaluation yet");
    RXCU(cudaMemcpy(out, virial.p, sizeof(double) * kVir * nsys, cudaMemcpyDeviceToHost));
  }

  void qeq_solve(int* iters, double* rel) {
    require_ff();
    require_sys();
    if (!have_pos) throw Error(RX_ERR_STATE, "no positions set");
    for (int attempt = 0;; ++attempt) {
      RXCU(cudaMemsetAsync(status.p, 0, sizeof(int) * kStatusWords, stream));
      const Dev d = dev();
      build_lists(d);
      launch_qeq(d);
      fetch_qeq_counts();
      int st[kStatusWords];
      RXCU(cudaMemcpyAsync(st, status.p, sizeof st, cudaMemcpyDeviceToHost, stream));
      RXCU(cudaStreamSynchronize(stream));
      RXCU(cudaGetLastError());
      if (grow_from_status(st, attempt)) {
        force_rebuild();
        continue;
      }
      check_status(st, true);
      break;
    }
    if (iters) std::copy(last_iters.begin(), last_iters.end(), iters);
    if (rel) std::copy(last_rel.begin(), last_rel.end(), rel);
  }

  // mtl::Context::qeq_solve: the charge matrix of the current positions (compute_H), then the CG of both systems for
  // the caller's right-hand sides from the caller's guesses; charges and histories are left alone.
  void qeq_cg(const double* b, const double* x0, double* x_out, int* iters, double* rel, int* stat) {
    require_ff();
    require_sys();
    if (!have_pos) throw Error(RX_ERR_STATE, "no positions set");
    if (!b || !x_out) throw Error(RX_ERR_INVALID, "rx_qeq_cg: null b or x_out");
    rows_only();
    const size_t n2 = 2 * static_cast<size_t>(na);
    DBuf<double> bd, xd;
    bd.ensure(n2);
    RXCU(cudaMemcpyAsync(bd.p, b, sizeof(double) * n2, cudaMemcpyHostToDevice, stream));
    if (x0) {
      xd.ensure(n2);
      RXCU(cudaMemcpyAsync(xd.p, x0, sizeof(double) * n2, cudaMemcpyHostToDevice, stream));
    }
    RXCU(cudaMemsetAsync(status.p, 0, sizeof(int) * kStatusWords, stream));
    const Dev d = dev();
    CgArgs a = cg_args();
    a.write_q = 0;
    ++launches;
    k_qeq_prepare_given<<<blocks(na, 256), 256, 0, stream>>>(d, dff, a, bd.p, x0 ? xd.p : nullptr);
    launch_cg(d, a);
    fetch_qeq_counts();
    std::vector<double2> xh(static_cast<size_t>(na));
    std::vector<int> brk(static_cast<size_t>(nsys));
    RXCU(cudaMemcpyAsync(xh.data(), cg_x.p, sizeof(double2) * na, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaMemcpyAsync(brk.data(), cg_brk.p, sizeof(int) * nsys, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaStreamSynchronize(stream));
    RXCU(cudaGetLastError());
    for (int i = 0; i < na; ++i) { x_out[i] = xh[static_cast<size_t>(i)].x; x_out[na + i] = xh[static_cast<size_t>(i)].y; }
    for (int sy = 0; sy < nsys; ++sy)
      for (int k = 0; k < 2; ++k) {
        const size_t j = 2 * static_cast<size_t>(sy) + k;
        if (iters) iters[j] = last_iters[j];
        if (rel) rel[j] = last_rel[j];
        if (stat) stat[j] = brk[static_cast<size_t>(sy)] ? 2 : (last_rel[j] <= qeq_tol ? 1 : 3);
      }
  }

  // rows and charge matrix of the current positions, with grow-and-retry (no charge solve, no forces)
  void rows_only() {
    for (int attempt = 0;; ++attempt) {
      RXCU(cudaMemsetAsync(status.p, 0, sizeof(int) * kStatusWords, stream));
      build_lists(dev());
      int st[kStatusWords];
      RXCU(cudaMemcpyAsync(st, status.p, sizeof st, cudaMemcpyDeviceToHost, stream));
      RXCU(cudaStreamSynchronize(stream));
      RXCU(cudaGetLastError());
      if (grow_from_status(st, attempt)) {
        force_rebuild();
        continue;
      }
      check_status(st, false);
      break;
    }
  }

  void qeq_matvec(const double* vin, double* yout) {
    require_ff();
    require_sys();
    if (!have_pos) throw Error(RX_ERR_STATE, "no positions set");
    rows_only();
    std::vector<double2> h(static_cast<size_t>(na));
    for (int a = 0; a < na; ++a) h[static_cast<size_t>(a)] = make_double2(vin[a], 0.0);
    RXCU(cudaMemcpyAsync(cg_d.p, h.data(), sizeof(double2) * na, cudaMemcpyHostToDevice, stream));
    ++launches;
    k_qeq_matvec<<<blocks(static_cast<long long>(na) * 32, 128), 128, 0, stream>>>(dev(), dff, cg_d.p, cg_q.p);
    RXCU(cudaMemcpyAsync(h.data(), cg_q.p, sizeof(double2) * na, cudaMemcpyDeviceToHost, stream));
    RXCU(cudaStreamSynchronize(stream));
    for (int a = 0; a < na; ++a) yout[a] = h[static_cast<size_t>(a)].x;
  }

  // ------------------------------------------------------------------ MD
  void md_setup(const double* mass_in, double dt, double t0, double t1, double tdamp, int chain) {
    require_ff();
    require_sys();
    if (!(dt > 0) || !(t0 > 0) || !(t1 > 0) || !(tdamp > 0) || chain < 0 || chain > kMaxChain)
      throw Error(RX_ERR_INVALID, "md_setup: need dt, temperatures, damping > 0 and 0 <= chain <= 8");
    mass.ensure(static_cast<size_t>(ff.nt));
    RXCU(cudaMemcpy(mass.p, mass_in, sizeof(double) * ff.nt, cudaMemcpyHostToDevice));
    v.ensure(static_cast<size_t>(na));
    md_layout(dt, t0, t1, tdamp, chain);
    RXCU(cudaMemset(xi.p, 0, sizeof(double) * nsys * kMaxChain));
    RXCU(cudaMemset(vxi.p, 0, sizeof(double) * nsys * kMaxChain));
    RXCU(cudaMemset(v.p, 0, sizeof(double4) * na));
    md_step = 0;
  }

  // the per-system integrator arrays of the current systems (velocities and chain state are left to the caller)
  void md_layout(double dt, double t0, double t1, double tdamp, int chain) {
    v.ensure(static_cast<size_t>(na));
    ke.ensure(static_cast<size_t>(nsys)); temp.ensure(static_cast<size_t>(nsys)); scale.ensure(static_cast<size_t>(nsys));
    xi.ensure(static_cast<size_t>(nsys) * kMaxChain); vxi.ensure(static_cast<size_t>(nsys) * kMaxChain);
    std::vector<int> first(static_cast<size_t>(nsys) + 1, 0), csys;
    for (int s = 0; s < nsys; ++s) {
      const int nc = (hsys[s].natoms + kKeChunk - 1) / kKeChunk;
      first[s + 1] = first[s] + nc;
      for (int k = 0; k < nc; ++k) csys.push_back(s);
    }
    const int nchunks = first[nsys];
    kpart.ensure(std::max(nchunks, 1)); kfirst.ensure(first.size()); ksys.ensure(std::max(nchunks, 1));
    RXCU(cudaMemcpy(kfirst.p, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
    if (nchunks > 0) RXCU(cudaMemcpy(ksys.p, csys.data(), sizeof(int) * csys.size(), cudaMemcpyHostToDevice));
    ramp.ensure(2);
    RXCU(cudaMemset(ramp.p, 0, sizeof(double) * 2));
    md = MdDev{v.p, mass.p, ke.p, temp.p, scale.p, xi.p, vxi.p, dt, t0, t1, tdamp, chain, kpart.p, kfirst.p, ksys.p, nchunks, ramp.p,
               nullptr, nullptr};
    md_ready = true;
    drop_graph();
  }

  // Continuous batching: the systems become `nkeep` of the current ones (keep[k] = current index, in their new order)
  // followed by `nnew` new ones. Kept systems carry their positions, velocities, charges, charge histories and chain
  // state; new systems take x_new / v_new. Every system's rows are rebuilt at the next evaluation.
  void update_systems(int nkeep, const int* keep, int nnew, const int* natoms, const double* origin, const double* box,
                      const int* periodic, const int* types, const int64_t* tags, const double* x_new, const double* v_new) {
    require_ff();
    if (host_only) throw Error(RX_ERR_STATE, "host-only context (created with device < 0)");
    if (nkeep < 0 || nnew < 0 || nkeep + nnew <= 0) throw Error(RX_ERR_INVALID, "update_systems: no systems");
    if (nkeep > 0 && (!keep || nsys == 0)) throw Error(RX_ERR_INVALID, "update_systems: nothing to keep");
    if (nnew > 0 && (!natoms || !origin || !box || !types || !tags || !x_new)) throw Error(RX_ERR_INVALID, "update_systems: null input");
    std::vector<char> seen(static_cast<size_t>(nsys), 0);
    for (int k = 0; k < nkeep; ++k) {
      if (keep[k] < 0 || keep[k] >= nsys || seen[static_cast<size_t>(keep[k])]) throw Error(RX_ERR_INVALID, "update_systems: bad keep list");
      seen[static_cast<size_t>(keep[k])] = 1;
    }
    const int ns = nkeep + nnew;
    std::vector<int> nat(static_cast<size_t>(ns)), per(3 * static_cast<size_t>(ns), 1), ty;
    std::vector<double> org(3 * static_cast<size_t>(ns)), bx(9 * static_cast<size_t>(ns));
    std::vector<int64_t> tg;
    std::vector<int> src;   // new atom -> old atom (kept systems)
    for (int k = 0; k < nkeep; ++k) {
      const SysInfo& o = hsys[static_cast<size_t>(keep[k])];
      nat[static_cast<size_t>(k)] = o.natoms;
      for (int c = 0; c < 3; ++c) org[3 * k + c] = o.origin[c];
      for (int c = 0; c < 9; ++c) bx[9 * k + c] = o.L[c];
      for (int c = 0; c < 3; ++c) per[3 * k + c] = o.per[c];
      for (int a = 0; a < o.natoms; ++a) {
        src.push_back(o.begin + a);
        ty.push_back(htype[static_cast<size_t>(o.begin + a)]);
        tg.push_back(htag[static_cast<size_t>(o.begin + a)]);
      }
    }
    const size_t nkept_atoms = src.size();
    long long nadd = 0;
    for (int k = 0; k < nnew; ++k) {
      nat[static_cast<size_t>(nkeep + k)] = natoms[k];
      for (int c = 0; c < 3; ++c) org[3 * (nkeep + k) + c] = origin[3 * k + c];
      for (int c = 0; c < 9; ++c) bx[9 * (nkeep + k) + c] = box[9 * k + c];
      if (periodic)
        for (int c = 0; c < 3; ++c) per[3 * (nkeep + k) + c] = periodic[3 * k + c];
      if (natoms[k] <= 0) throw Error(RX_ERR_INVALID, "every system needs at least one atom");
      nadd += natoms[k];
    }
    ty.insert(ty.end(), types, types + nadd);
    tg.insert(tg.end(), tags, tags + nadd);
    // the state to carry, before the buffers are resized
    const int old_na = na, old_nsys = nsys;
    const bool had_md = md_ready;
    const MdDev md_old = md;
    DBuf<double4> ox, ov;
    DBuf<double> oq, osh, oth;
    std::vector<double> oxi, ovxi;
    if (nkeep > 0) {
      ox.ensure(static_cast<size_t>(old_na)); oq.ensure(static_cast<size_t>(old_na));
      osh.ensure(4 * static_cast<size_t>(old_na)); oth.ensure(4 * static_cast<size_t>(old_na));
      RXCU(cudaMemcpy(ox.p, x.p, sizeof(double4) * old_na, cudaMemcpyDeviceToDevice));
      RXCU(cudaMemcpy(oq.p, q.p, sizeof(double) * old_na, cudaMemcpyDeviceToDevice));
      RXCU(cudaMemcpy(osh.p, s_hist.p, sizeof(double) * 4 * old_na, cudaMemcpyDeviceToDevice));
      RXCU(cudaMemcpy(oth.p, t_hist.p, sizeof(double) * 4 * old_na, cudaMemcpyDeviceToDevice));
      if (had_md) {
        ov.ensure(static_cast<size_t>(old_na));
        RXCU(cudaMemcpy(ov.p, v.p, sizeof(double4) * old_na, cudaMemcpyDeviceToDevice));
        oxi.resize(static_cast<size_t>(old_nsys) * kMaxChain);
        ovxi.resize(oxi.size());
        RXCU(cudaMemcpy(oxi.data(), xi.p, sizeof(double) * oxi.size(), cudaMemcpyDeviceToHost));
        RXCU(cudaMemcpy(ovxi.data(), vxi.p, sizeof(double) * ovxi.size(), cudaMemcpyDeviceToHost));
      }
    }
    const bool had_forces = forces_valid;
    DBuf<double4> og;
    if (nkeep > 0 && had_forces) {
      og.ensure(static_cast<size_t>(old_na));
      RXCU(cudaMemcpy(og.p, grad.p, sizeof(double4) * old_na, cudaMemcpyDeviceToDevice));
    }
    set_systems(ns, nat.data(), org.data(), bx.data(), per.data(), ty.data(), tg.data());
    if (nadd > 0) {   // new systems start with cold charge histories
      RXCU(cudaMemset(s_hist.p + 4 * nkept_atoms, 0, sizeof(double) * 4 * nadd));
      RXCU(cudaMemset(t_hist.p + 4 * nkept_atoms, 0, sizeof(double) * 4 * nadd));
    }
    {   // new systems with non-periodic directions are laid out around their own atoms
      std::vector<double> xall(3 * static_cast<size_t>(na), 0.0);
      std::copy(x_new, x_new + 3 * nadd, xall.begin() + 3 * static_cast<long long>(nkept_atoms));
      fit_nonperiodic(xall.data(), nkeep);
    }
    // positions: new systems from the caller, kept ones gathered from the saved state
    {
      std::vector<double4> h(static_cast<size_t>(nadd));
      for (long long a = 0; a < nadd; ++a) h[static_cast<size_t>(a)] = make_double4(x_new[3 * a], x_new[3 * a + 1], x_new[3 * a + 2], 0.0);
      if (nadd > 0) RXCU(cudaMemcpy(x.p + nkept_atoms, h.data(), sizeof(double4) * nadd, cudaMemcpyHostToDevice));
    }
    DBuf<int> srcd;
    if (nkept_atoms > 0) {
      srcd.ensure(nkept_atoms);
      RXCU(cudaMemcpy(srcd.p, src.data(), sizeof(int) * nkept_atoms, cudaMemcpyHostToDevice));
      ++launches;
      k_gather_state<<<blocks(static_cast<long long>(nkept_atoms), 256), 256, 0, stream>>>(
          static_cast<int>(nkept_atoms), srcd.p, ox.p, oq.p, osh.p, oth.p, x.p, q.p, s_hist.p, t_hist.p);
    }
    if (had_forces && nkeep > 0 && nadd == 0) {   // only removals: the kept systems' forces stay valid
      ++launches;
      k_gather_vel<<<blocks(static_cast<long long>(nkept_atoms), 256), 256, 0, stream>>>(static_cast<int>(nkept_atoms), srcd.p, og.p, grad.p);
    }
    if (had_md) {
      md_layout(md_old.dt, md_old.t_start, md_old.t_stop, md_old.t_damp, md_old.chain);
      RXCU(cudaMemsetAsync(v.p, 0, sizeof(double4) * na, stream));
      if (nkept_atoms > 0) {
        ++launches;
        k_gather_vel<<<blocks(static_cast<long long>(nkept_atoms), 256), 256, 0, stream>>>(static_cast<int>(nkept_atoms), srcd.p, ov.p, v.p);
      }
      if (v_new && nadd > 0) {
        std::vector<double4> h(static_cast<size_t>(nadd));
        for (long long a = 0; a < nadd; ++a) h[static_cast<size_t>(a)] = make_double4(v_new[3 * a], v_new[3 * a + 1], v_new[3 * a + 2], 0.0);
        RXCU(cudaMemcpyAsync(v.p + nkept_atoms, h.data(), sizeof(double4) * nadd, cudaMemcpyHostToDevice, stream));
      }
      std::vector<double> nxi(static_cast<size_t>(nsys) * kMaxChain, 0.0), nvxi(nxi.size(), 0.0);
      for (int k = 0; k < nkeep; ++k)
        for (int c = 0; c < kMaxChain; ++c) {
          nxi[static_cast<size_t>(k) * kMaxChain + c] = oxi[static_cast<size_t>(keep[k]) * kMaxChain + c];
          nvxi[static_cast<size_t>(k) * kMaxChain + c] = ovxi[static_cast<size_t>(keep[k]) * kMaxChain + c];
        }
      RXCU(cudaMemcpyAsync(xi.p, nxi.data(), sizeof(double) * nxi.size(), cudaMemcpyHostToDevice, stream));
      RXCU(cudaMemcpyAsync(vxi.p, nvxi.data(), sizeof(double) * nvxi.size(), cudaMemcpyHostToDevice, stream));
    }
    RXCU(cudaStreamSynchronize(stream));
    RXCU(cudaGetLastError());
    have_pos = true;
    forces_valid = had_forces && nkeep > 0 && nadd == 0;
    force_rebuild();
    RXCU(cudaStreamSynchronize(stream));
  }

  // per-system targets and activity (serving); NULL restores the common ramp / all active
  DBuf<double> t_sys_buf;
  DBuf<int> active_buf;
  void md_targets(const double* t_target, const int* active) {
    if (!md_ready) throw Error(RX_ERR_STATE, "call rx_md_setup first");
    if (t_target) {
      for (int s = 0; s < nsys; ++s)
        if (!(t_target[s] > 0.0)) throw Error(RX_ERR_INVALID, "target temperatures must be positive");
      t_sys_buf.ensure(static_cast<size_t>(nsys));
      RXCU(cudaMemcpy(t_sys_buf.p, t_target, sizeof(double) * nsys, cudaMemcpyHostToDevice));
    }
    if (active) {
      active_buf.ensure(static_cast<size_t>(nsys));
      RXCU(cudaMemcpy(active_buf.p, active, sizeof(int) * nsys, cudaMemcpyHostToDevice));
    }
    const double* ts = t_target ? t_sys_buf.p : nullptr;
    const int* ac = active ? active_buf.p : nullptr;
    if (ts != md.t_sys || ac != md.active) drop_graph();   // a captured step holds the pointers, not the values
    md.t_sys = ts;
    md.active = ac;
  }

  void set_velocities(const double* vin) {
    if (!md_ready) throw Error(RX_ERR_STATE, "call rx_md_setup first");
    std::vector<double4> h(static_cast<size_t>(na));
    for (int a = 0; a < na; ++a) h[static_cast<size_t>(a)] = make_double4(vin[3 * a], vin[3 * a + 1], vin[3 * a + 2], 0.0);
    RXCU(cudaMemcpy(v.p, h.data(), sizeof(double4) * na, cudaMemcpyHostToDevice));
  }
  void get_velocities(double* vout) {
    if (!md_ready) throw Error(RX_ERR_STATE, "call rx_md_setup first");
    std::vector<double4> h(static_cast<size_t>(na));
    RXCU(cudaMemcpy(h.data(), v.p, sizeof(double4) * na, cudaMemcpyDeviceToHost));
    for (int a = 0; a < na; ++a) { vout[3 * a] = h[a].x; vout[3 * a + 1] = h[a].y; vout[3 * a + 2] = h[a].z; }
  }

  // the kinetic energy of the velocities as they stand, into md.ke (the chain's first half of a step starts from it)
  void kinetic_now() {
    launches += 2;
    k_md_kinetic_part<<<md.nchunks, 256, 0, stream>>>(md, sys.p, type.p);
    k_md_kinetic_sum<<<blocks(nsys, 64), 64, 0, stream>>>(md, nsys);
  }

  // one velocity-Verlet step with the chain applied for dt/2 on each side (see md_kernels.cu), enqueued only. First
  // half: the chain from the kinetic energy the previous half left in md.ke, then scale, kick and drift in one kernel;
  // second half: kick and the kinetic-energy partials in one kernel, the chain, the scale (and the ramp's step).
  bool md_qeq = true;   // charges re-equilibrated at every step of rx_md_run
  void enqueue_step() {
    launches += 2;
    k_md_chain<<<blocks(nsys, 64), 64, 0, stream>>>(md, sys.p, nsys, 1);
    k_md_scale_kick<<<blocks(na, 256), 256, 0, stream>>>(md, type.p, sys_of.p, grad.p, x.p, na);
    enqueue_eval(md_qeq);
    launches += 3;
    k_md_kick_kinetic<<<md.nchunks, 256, 0, stream>>>(md, sys.p, type.p, sys_of.p, grad.p);
    k_md_chain<<<blocks(nsys, 64), 64, 0, stream>>>(md, sys.p, nsys, 0);
    k_md_scale<<<blocks(na, 256), 256, 0, stream>>>(md, sys_of.p, na, 1);
  }

  // Capture the launches `fn` enqueues into a CUDA graph (every kernel argument is fixed at capture; what changes
  // from call to call lives in device memory). On failure graphs are switched off for this context and the launches
  // go out one by one.
  template <class F>
  bool capture(cudaGraphExec_t& exec, long long& count, F&& fn) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      (void)cudaGetLastError();
      graphs_ok = false;
      return false;
    }
    const long long l0 = launches;
    bool ok = true;
    try {
      fn();
    } catch (const Error&) {
      ok = false;
    }
    count = launches - l0;
    launches = l0;   // the capture itself launched nothing
    const cudaError_t e = cudaStreamEndCapture(stream, &g);
    ok = ok && e == cudaSuccess && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      exec = nullptr;
      (void)cudaGetLastError();
      graphs_ok = false;
    }
    return ok;
  }
  // a capture that fails with the rebuild conditional is repeated once without it
  template <class F>
  bool capture_retry(cudaGraphExec_t& exec, long long& count, F&& fn) {
    if (capture(exec, count, fn)) return true;
    if (!cond_ok) return false;
    cond_ok = false;
    graphs_ok = true;
    return capture(exec, count, fn);
  }
  long long step_launches = 0;   // this engine's kernels in one captured MD step
  bool capture_step() { return capture_retry(md_graph, step_launches, [&] { enqueue_step(); }); }

  // state that a chunk of steps changes, saved before the chunk so that an overflow (lists grown, chunk repeated)
  // restarts from it
  DBuf<double4> snap_x, snap_v, snap_g;
  DBuf<double> snap_q, snap_sh, snap_th, snap_xi, snap_vxi, snap_ramp;
  void snapshot(bool save) {
    const size_t n = static_cast<size_t>(na), nc = static_cast<size_t>(nsys) * kMaxChain;
    if (save) {
      snap_x.ensure(n); snap_v.ensure(n); snap_g.ensure(n); snap_q.ensure(n); snap_sh.ensure(4 * n); snap_th.ensure(4 * n);
      snap_xi.ensure(nc); snap_vxi.ensure(nc); snap_ramp.ensure(2);
    }
    auto cp = [&](void* dst_snap, void* live, size_t bytes) {
      if (save) RXCU(cudaMemcpyAsync(dst_snap, live, bytes, cudaMemcpyDeviceToDevice, stream));
      else RXCU(cudaMemcpyAsync(live, dst_snap, bytes, cudaMemcpyDeviceToDevice, stream));
    };
    cp(snap_x.p, x.p, sizeof(double4) * n);
    cp(snap_v.p, v.p, sizeof(double4) * n);
    cp(snap_g.p, grad.p, sizeof(double4) * n);
    cp(snap_q.p, q.p, sizeof(double) * n);
    cp(snap_sh.p, s_hist.p, sizeof(double) * 4 * n);
    cp(snap_th.p, t_hist.p, sizeof(double) * 4 * n);
    cp(snap_xi.p, xi.p, sizeof(double) * nc);
    cp(snap_vxi.p, vxi.p, sizeof(double) * nc);
    cp(snap_ramp.p, ramp.p, sizeof(double) * 2);
  }

  static constexpr int kChunk = 50;   // steps between host synchronisations of rx_md_run

  // Steps are enqueued in chunks without any host synchronisation (from a captured graph when possible); the host reads
  // the status word once per chunk. A list overflow inside a chunk restores the state saved before it, grows the
  // lists and repeats the chunk; any other failure is reported.
  void md_run(int nsteps, double* e_out, double* t_out, long long total_steps_hint) {
    if (!md_ready) throw Error(RX_ERR_STATE, "call rx_md_setup first");
    if (nsteps < 0) throw Error(RX_ERR_INVALID, "negative step count");
    const long long span = total_steps_hint > 0 ? total_steps_hint : nsteps;
    const double rh[2] = {0.0, static_cast<double>(span)};
    RXCU(cudaMemcpyAsync(ramp.p, rh, sizeof rh, cudaMemcpyHostToDevice, stream));
    if (!forces_valid) evaluate(md_qeq);   // forces of the initial configuration
    int done = 0;
    while (done < nsteps) {
      const int chunk = std::min(nsteps - done, kChunk);
      for (int attempt = 0;; ++attempt) {
        snapshot(true);
        kinetic_now();   // md.ke of the chunk's starting velocities (set by the caller or restored by a repeat)
        RXCU(cudaMemsetAsync(status.p, 0, sizeof(int) * kStatusWords, stream));
        const bool use_graph = graphs_ok && !timing;
        if (use_graph && !md_graph) capture_step();
        for (int k = 0; k < chunk; ++k) {
          if (use_graph && md_graph) {
            RXCU(cudaGraphLaunch(md_graph, stream));
            launches += step_launches;
          } else {
            enqueue_step();
            if (timing) {
              RXCU(cudaStreamSynchronize(stream));
              collect_times();
            }
          }
        }
        if (md_qeq) fetch_qeq_counts();
        int st[kStatusWords];
        RXCU(cudaMemcpyAsync(st, status.p, sizeof st, cudaMemcpyDeviceToHost, stream));
        RXCU(cudaStreamSynchronize(stream));
        RXCU(cudaGetLastError());
        if (grow_from_status(st, attempt)) {
          snapshot(false);
          force_rebuild();
          continue;
        }
        check_status(st, md_qeq);
        break;
      }
      done += chunk;
      md_step += chunk;
    }
    energy_sums();
    if (e_out) RXCU(cudaMemcpyAsync(e_out, energies.p, sizeof(double) * kTerms * nsys, cudaMemcpyDeviceToHost, stream));
    if (t_out) {
      launches += 2;
      k_md_kinetic_part<<<md.nchunks, 256, 0, stream>>>(md, sys.p, type.p);
      k_md_kinetic_sum<<<blocks(nsys, 64), 64, 0, stream>>>(md, nsys);
      std::vector<double> kk(static_cast<size_t>(nsys));
      RXCU(cudaMemcpyAsync(kk.data(), ke.p, sizeof(double) * nsys, cudaMemcpyDeviceToHost, stream));
      RXCU(cudaStreamSynchronize(stream));
      for (int s = 0; s < nsys; ++s) t_out[s] = 2.0 * kk[s] / ((3.0 * hsys[s].natoms - 3.0) * 0.0019872067);
    }
    RXCU(cudaStreamSynchronize(stream));
  }
};

}  // namespace rx

// ======================================================================================================== C ABI
struct rx_context {
  std::unique_ptr<rx::Context> c;
  std::string err;
};

namespace {
thread_local std::string g_create_error;

template <class F>
int guarded(rx_context* ctx, F&& f) {
  if (!ctx || !ctx->c) return RX_ERR_STATE;
  try {
    if (!ctx->c->host_only) cudaSetDevice(ctx->c->device);
    f(*ctx->c);
    ctx->err.clear();
    return RX_OK;
  } catch (const rx::Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return RX_ERR_INVALID;
  }
}
}  // namespace

extern "C" {

rx_context* rx_create(int device) {
  try {
    auto* ctx = new rx_context;
    ctx->c = std::make_unique<rx::Context>(device);
    g_create_error.clear();
    return ctx;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return nullptr;
  }
}

void rx_destroy(rx_context* ctx) { delete ctx; }

void* rx_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0 || cudaMallocHost(&p, bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return p;
}

void rx_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

const char* rx_last_error(const rx_context* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int rx_set_forcefield(rx_context* ctx, const char* text, int lgvdw) {
  return guarded(ctx, [&](rx::Context& c) { c.set_forcefield(text, lgvdw); });
}

long rx_forcefield_dump(rx_context* ctx, int portable, char* out, long outlen) {
  long result = -1;
  const int rc = guarded(ctx, [&](rx::Context& c) {
    c.require_ff();
    const std::string s = c.ff.canonical_dump(portable != 0);
    if (out && outlen > 0) {
      const size_t m = std::min<size_t>(s.size(), static_cast<size_t>(outlen - 1));
      std::memcpy(out, s.data(), m);
      out[m] = 0;
    }
    result = static_cast<long>(s.size());
  });
  return rc == RX_OK ? result : -1;
}

int rx_forcefield_params(rx_context* ctx, int* ntypes, double* chi, double* eta, double* gamma, double* mass) {
  return guarded(ctx, [&](rx::Context& c) {
    c.require_ff();
    if (ntypes) *ntypes = c.ff.nt;
    for (int t = 0; t < c.ff.nt; ++t) {
      if (chi) chi[t] = c.ff.s(t, rx::SB_CHI);
      if (eta) eta[t] = c.ff.s(t, rx::SB_ETA);
      if (gamma) gamma[t] = c.ff.s(t, rx::SB_GAMMA);
      if (mass) mass[t] = c.ff.s(t, rx::SB_MASS);
    }
  });
}

int rx_forcefield_element(rx_context* ctx, const char* symbol) {
  int out = -1;
  const int rc = guarded(ctx, [&](rx::Context& c) {
    c.require_ff();
    if (!symbol) throw rx::Error(RX_ERR_INVALID, "null element symbol");
    std::string key;
    for (const char* p = symbol; *p && key.size() < 3; ++p) key.push_back(static_cast<char>(toupper(static_cast<unsigned char>(*p))));
    for (size_t k = 0; k < c.ff.names.size(); ++k)
      if (c.ff.names[k] == key) { out = static_cast<int>(k); break; }
  });
  return rc == RX_OK ? out : -1;
}

int rx_set_control(rx_context* ctx, double bond_cut, double hbond_cut, double thb_cut, double thb_cutsq, int enobonds) {
  return guarded(ctx, [&](rx::Context& c) { c.set_control(bond_cut, hbond_cut, thb_cut, thb_cutsq, enobonds); });
}

int rx_set_systems(rx_context* ctx, int nsys, const int* natoms, const double* origin, const double* box, const int* periodic,
                   const int* type, const int64_t* tag) {
  return guarded(ctx, [&](rx::Context& c) { c.set_systems(nsys, natoms, origin, box, periodic, type, tag); });
}

int rx_num_atoms(const rx_context* ctx) { return (ctx && ctx->c) ? ctx->c->na : 0; }

// The LAMMPS pair-style energy vector of `pair_style reaxff` (src/core/energy_terms.cpp:35-50 mirrors
// pair_reaxff.cpp:501-514): 14 slots eb, ea (over + under), elp, emol (0), ev, epen, ecoa, ehb, et, eco, ew, ep, efi (0),
// eqeq (polarization); eng_vdwl = every term but Coulomb and polarization, eng_coul = Coulomb + polarization
// (pair_reaxff_metal.cpp:515-519).
int rx_pvector(const double* e, double* pv, double* eng_vdwl, double* eng_coul) {
  if (!e) return RX_ERR_INVALID;
  using namespace rx;
  if (pv) {
    const double v[14] = {e[E_BOND], e[E_OV] + e[E_UN], e[E_LP], 0.0, e[E_ANG], e[E_PEN], e[E_COA], e[E_HB], e[E_TOR],
                          e[E_CON], e[E_VDW], e[E_ELE], 0.0, e[E_POL]};
    for (int k = 0; k < 14; ++k) pv[k] = v[k];
  }
  if (eng_vdwl)
    *eng_vdwl = e[E_BOND] + e[E_OV] + e[E_UN] + e[E_LP] + e[E_ANG] + e[E_PEN] + e[E_COA] + e[E_HB] + e[E_TOR] + e[E_CON] + e[E_VDW];
  if (eng_coul) *eng_coul = e[E_ELE] + e[E_POL];
  return RX_OK;
}

int rx_qeq_refinements(rx_context* ctx) {
  if (!ctx || !ctx->c || ctx->c->host_only || !ctx->c->cg_nref.p) return -1;
  int v = 0;
  if (cudaMemcpy(&v, ctx->c->cg_nref.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return v;
}

int rx_qeq_last(const rx_context* ctx, int32_t* iters, double* rel) {
  if (!ctx || !ctx->c) return RX_ERR_STATE;
  const rx::Context& c = *ctx->c;
  if (c.last_iters.empty()) return RX_ERR_STATE;
  if (iters) std::copy(c.last_iters.begin(), c.last_iters.end(), iters);
  if (rel) std::copy(c.last_rel.begin(), c.last_rel.end(), rel);
  return RX_OK;
}

int rx_set_capacities(rx_context* ctx, int nbr_entries, int bonds, int near_entries) {
  return guarded(ctx, [&](rx::Context& c) {
    c.require_sys();
    if (nbr_entries < 1 || bonds < 1 || near_entries < 1) throw rx::Error(RX_ERR_INVALID, "capacities must be >= 1");
    c.ncap = (nbr_entries + 31) / 32 * 32;
    c.bcap = bonds;
    c.ncap_near = (near_entries + 31) / 32 * 32;
    c.alloc_lists();
    c.force_rebuild();
  });
}

int rx_get_capacities(const rx_context* ctx, int* out3) {
  if (!ctx || !ctx->c || !out3) return RX_ERR_INVALID;
  out3[0] = ctx->c->ncap;
  out3[1] = ctx->c->bcap;
  out3[2] = ctx->c->ncap_near;
  return RX_OK;
}

int rx_set_positions(rx_context* ctx, const double* x) {
  return guarded(ctx, [&](rx::Context& c) {
    if (!x) throw rx::Error(RX_ERR_INVALID, "null positions");
    c.set_positions(x);
  });
}
int rx_get_positions(rx_context* ctx, double* x) { return guarded(ctx, [&](rx::Context& c) { c.get_positions(x); }); }

int rx_set_charges(rx_context* ctx, const double* q) {
  return guarded(ctx, [&](rx::Context& c) {
    c.require_sys();
    RXCU(cudaMemcpy(c.q.p, q, sizeof(double) * c.na, cudaMemcpyHostToDevice));
  });
}
int rx_get_charges(rx_context* ctx, double* q) {
  return guarded(ctx, [&](rx::Context& c) {
    c.require_sys();
    RXCU(cudaMemcpy(q, c.q.p, sizeof(double) * c.na, cudaMemcpyDeviceToHost));
  });
}

int rx_set_qeq(rx_context* ctx, double swa, double swb, double tol, int imax, int strict) {
  return guarded(ctx, [&](rx::Context& c) {
    c.set_qeq(swa, swb, tol, imax, strict);
    if (c.have_ff && c.nsys > 0) c.layout_systems();
  });
}
int rx_qeq_solve(rx_context* ctx, int* iters, double* rel) { return guarded(ctx, [&](rx::Context& c) { c.qeq_solve(iters, rel); }); }
int rx_qeq_cg(rx_context* ctx, const double* b, const double* x0, double* x_out, int* iters, double* rel, int* status) {
  return guarded(ctx, [&](rx::Context& c) { c.qeq_cg(b, x0, x_out, iters, rel, status); });
}
int rx_qeq_matvec(rx_context* ctx, const double* v, double* y) { return guarded(ctx, [&](rx::Context& c) { c.qeq_matvec(v, y); }); }

int rx_compute(rx_context* ctx, int flags, double* energies, double* grad, int32_t* census, int64_t* counts) {
  return guarded(ctx, [&](rx::Context& c) { c.compute(flags, energies, grad, census, counts); });
}

int rx_md_setup(rx_context* ctx, const double* mass, double dt, double t_start, double t_stop, double t_damp, int chain) {
  return guarded(ctx, [&](rx::Context& c) { c.md_setup(mass, dt, t_start, t_stop, t_damp, chain); });
}
int rx_set_velocities(rx_context* ctx, const double* v) { return guarded(ctx, [&](rx::Context& c) { c.set_velocities(v); }); }
int rx_get_velocities(rx_context* ctx, double* v) { return guarded(ctx, [&](rx::Context& c) { c.get_velocities(v); }); }
int rx_md_run(rx_context* ctx, int nsteps, double* energies, double* temperature) {
  return guarded(ctx, [&](rx::Context& c) { c.md_run(nsteps, energies, temperature, 0); });
}

int rx_autotune(rx_context* ctx, int reps, int* chosen) {
  return guarded(ctx, [&](rx::Context& c) { c.autotune(reps, chosen); });
}
int rx_set_tuning(rx_context* ctx, int key, int value) {
  return guarded(ctx, [&](rx::Context& c) { c.set_tuning(key, value); });
}

int rx_qeq_reset(rx_context* ctx) { return guarded(ctx, [&](rx::Context& c) { c.qeq_reset(); }); }

int rx_set_acks2(rx_context* ctx, const double* s_kin) {
  return guarded(ctx, [&](rx::Context& c) { c.set_acks2(s_kin); });
}

int rx_set_neighbor(rx_context* ctx, double skin) {
  return guarded(ctx, [&](rx::Context& c) { c.set_neighbor(skin); });
}

int rx_get_peratom(rx_context* ctx, double* eatom, double* vatom) {
  return guarded(ctx, [&](rx::Context& c) { c.get_peratom(eatom, vatom); });
}

long long rx_get_bonds(rx_context* ctx, int* start, int* partner, int* shift, double* bo, double* total_bo, double* nlp,
                       long long cap) {
  long long out = -1;
  const int rc = guarded(ctx, [&](rx::Context& c) { out = c.get_bonds(start, partner, shift, bo, total_bo, nlp, cap); });
  return rc == RX_OK ? out : -1;
}

int rx_get_gradient(rx_context* ctx, double* grad) {
  return guarded(ctx, [&](rx::Context& c) {
    if (!grad) throw rx::Error(RX_ERR_INVALID, "null gradient array");
    c.get_gradient(grad);
  });
}

int rx_get_virial(rx_context* ctx, double* virial) {
  return guarded(ctx, [&](rx::Context& c) {
    if (!virial) throw rx::Error(RX_ERR_INVALID, "null virial array");
    c.get_virial(virial);
  });
}

int rx_update_systems(rx_context* ctx, int nkeep, const int* keep, int nnew, const int* natoms, const double* origin,
                      const double* box, const int* periodic, const int* type, const int64_t* tag, const double* x,
                      const double* v) {
  return guarded(ctx, [&](rx::Context& c) { c.update_systems(nkeep, keep, nnew, natoms, origin, box, periodic, type, tag, x, v); });
}

int rx_md_charges(rx_context* ctx, int on) {
  return guarded(ctx, [&](rx::Context& c) {
    c.md_qeq = on != 0;
    c.drop_graph();
  });
}

int rx_md_targets(rx_context* ctx, const double* t_target, const int* active) {
  return guarded(ctx, [&](rx::Context& c) { c.md_targets(t_target, active); });
}

int64_t rx_kernel_launches(const rx_context* ctx) { return (ctx && ctx->c) ? ctx->c->launches : 0; }

void* rx_stream(rx_context* ctx) { return (ctx && ctx->c) ? reinterpret_cast<void*>(ctx->c->stream) : nullptr; }

int rx_set_timing(rx_context* ctx, int on) {
  return guarded(ctx, [&](rx::Context& c) {
    c.timing = on != 0;
    c.drop_graph();
    for (auto& p : c.phases) p.ms = 0.0;
  });
}

int rx_phase_times(rx_context* ctx, char* names_out, long names_len, double* ms, int max_phases) {
  if (!ctx || !ctx->c) return 0;
  std::string names;
  int n = 0;
  for (auto& p : ctx->c->phases) {
    if (n >= max_phases) break;
    if (ms) ms[n] = p.ms;
    names += p.name;
    names += "\n";
    ++n;
  }
  if (names_out && names_len > 0) {
    const size_t m = std::min<size_t>(names.size(), static_cast<size_t>(names_len - 1));
    std::memcpy(names_out, names.data(), m);
    names_out[m] = 0;
  }
  return n;
}

}  // extern "C"
