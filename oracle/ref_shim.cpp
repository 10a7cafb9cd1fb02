// TEST INFRASTRUCTURE ONLY. A C entry point over the reference's own FP64 `cpu64` engine, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libreaxref.so. Tests and the CPU-baseline leg of the
// benchmark use it to pin the C restatement (oracle/rx_oracle.c) and the CUDA engine; nothing in the product
// links it.
//
// It runs the same sequence as the reference's CLI driver tools/energy_tool.cpp:21-142:
//   read_force_field_file -> expand_images -> AtomSet::validate -> build_far_list -> compute_bonded_core
//   -> compute_nonbonded_core (when charges are given) -> census -> gradient folded onto owners.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "reaxmetal/acks2.hpp"
#include "reaxmetal/bonded.hpp"
#include "reaxmetal/energy_terms.hpp"
#include "reaxmetal/forcefield.hpp"
#include "reaxmetal/neighbor.hpp"
#include "reaxmetal/nonbonded.hpp"

using namespace reaxmetal;

namespace {
void set_err(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) {
    std::snprintf(err, static_cast<std::size_t>(errlen), "%s", msg);
  }
}
}  // namespace

extern "C" {

// Canonical, sorted table dump of the parsed force field (src/io/table_dump.cpp:20). Returns the length
// needed (excluding the NUL); writes at most outlen bytes. Negative on a parse error (message in out).
long ref_table_dump(const char* ffield_text, int portable, char* out, long outlen) {
  try {
    const ForceField ff = parse_force_field(ffield_text, "ffield");
    const std::string s = canonical_table_dump(ff, portable != 0);
    if (out && outlen > 0) {
      const std::size_t m = std::min<std::size_t>(s.size(), static_cast<std::size_t>(outlen - 1));
      std::memcpy(out, s.data(), m);
      out[m] = 0;
    }
    return static_cast<long>(s.size());
  } catch (const std::exception& e) {
    set_err(out, static_cast<int>(outlen), e.what());
    return -1;
  }
}

// One single point of the cpu64 engine.
//   box9: lattice vectors a, b, c (row-major); origin3; periodic3 (0/1)
//   x: 3n owned coordinates, type: n force-field type indices (0-based), tag: n atom ids
//   lgvdw: 1 reads and evaluates the force field as `pair_style reaxff lgvdw yes`
//   s_kin: NULL, or n kinetic potentials of fix acks2/reaxff (its s[N + i]): the ACKS2 pair terms are added
//   q: n charges or NULL (NULL: the non-bonded terms are skipped, as energy_tool does without charges)
//   e13: energies in EnergyTerm order (bond, over, under, lone_pair, valence, penalty, coalition, hbond,
//        torsion, conjugation, vdw, coulomb, polarization), kcal/mol
//   grad: 3n, dE/dx folded onto the owners (ghost gradient added to its owner)
//   census: 7n int32 (bonds, angle_sets, torsions, hbonds, nonbonded, sbo_region, lp_trunc) or NULL
//   counts: [undirected bonds incl. ghost rows, counted non-bonded pairs, nall, far-list entries]
//   virial6: NULL or LAMMPS's fdotr virial of the owned + ghost forces the pair style hands LAMMPS
//            (pair_reaxff_metal.cpp:500-504 then virial_fdotr_compute, :523): sum over nall of x_a f_b in the
//            order xx, yy, zz, xy, xz, yz, f = -grad
int ref_single_point(const char* ffield_text, const double* origin3, const double* box9, const int* periodic3, int n,
                     const double* x, const int* type, const long long* tag, const double* q, double bond_cut,
                     double hbond_cut, double shell, int enobonds, int lgvdw, const double* s_kin, double* e13,
                     double* grad, int* census, long long* counts, double* virial6, char* err, int errlen) {
  try {
    FfieldOptions fo;
    fo.lgvdw = lgvdw != 0;
    const ForceField ff = parse_force_field(ffield_text, "ffield", fo);
    ControlParams ctl;
    ctl.bond_cut = bond_cut;
    ctl.hbond_cut = hbond_cut;
    NeighborCutoffs cut;
    cut.nonb = ff.file_control().nonb_cut;
    cut.bond = ctl.bond_cut;
    cut.hbond = ctl.hbond_cut;
    Box box;
    for (int c = 0; c < 3; ++c) box.origin[static_cast<std::size_t>(c)] = origin3[c];
    for (int v = 0; v < 3; ++v)
      for (int c = 0; c < 3; ++c) box.vectors[static_cast<std::size_t>(v)][static_cast<std::size_t>(c)] = box9[3 * v + c];
    for (int d = 0; d < 3; ++d) box.periodic[static_cast<std::size_t>(d)] = periodic3[d] != 0;
    std::vector<double> xs(x, x + 3 * static_cast<std::size_t>(n));
    std::vector<int> ty(type, type + n);
    std::vector<std::int64_t> tg(tag, tag + n);
    ExpandOptions eo;
    eo.shell = shell > 0 ? shell : cut.required_shell();
    const AtomSet a = expand_images(box, xs, ty, tg, eo);
    a.validate(box);
    const FarList f = build_far_list(a, cut);
    BondedOptions bo;
    bo.enobonds = enobonds != 0;
    bo.census = census != nullptr;
    const BondedResult r = compute_bonded_core(ff, ctl, a, f, bo);
    NonbondedResult nb;
    if (q) {
      NonbondedOptions no;
      no.census = census != nullptr;
      no.lgvdw = lgvdw != 0;
      std::vector<double> qv(q, q + n);
      nb = compute_nonbonded_core(ff, cut, a, f, qv, no);
      if (s_kin) {   // the pair side of fix acks2/reaxff, as pair_reaxff_metal.cpp:492 adds it for cpu64
        std::vector<double> sk(a.nall());
        for (std::size_t i = 0; i < a.nall(); ++i) sk[i] = s_kin[a.owner[i]];
        add_acks2_terms(ff, cut, a, f, qv, sk.data(), nb);
      }
    }
    for (std::size_t t = 0; t < kEnergyTermCount; ++t) e13[t] = r.e.e[t] + nb.e.e[t];
    std::vector<double> g(3 * static_cast<std::size_t>(n), 0.0);
    for (std::size_t i = 0; i < a.nall(); ++i)
      for (std::size_t c = 0; c < 3; ++c)
        g[3 * static_cast<std::size_t>(a.owner[i]) + c] += r.grad[3 * i + c] + (nb.grad.empty() ? 0.0 : nb.grad[3 * i + c]);
    std::memcpy(grad, g.data(), g.size() * sizeof(double));
    if (virial6) {
      for (int c = 0; c < 6; ++c) virial6[c] = 0.0;
      for (std::size_t i = 0; i < a.nall(); ++i) {
        double f[3], xi[3];
        for (std::size_t c = 0; c < 3; ++c) {
          f[c] = -(r.grad[3 * i + c] + (nb.grad.empty() ? 0.0 : nb.grad[3 * i + c]));
          xi[c] = a.x[3 * i + c];
        }
        virial6[0] += f[0] * xi[0]; virial6[1] += f[1] * xi[1]; virial6[2] += f[2] * xi[2];
        virial6[3] += f[1] * xi[0]; virial6[4] += f[2] * xi[0]; virial6[5] += f[2] * xi[1];
      }
    }
    if (census) {
      const std::vector<std::int32_t>* cols[7] = {&r.census.bonds, &r.census.angle_sets, &r.census.torsions, &r.census.hbonds,
                                                 &nb.census_nonbonded, &r.census.sbo_region, &r.census.lp_trunc};
      for (int k = 0; k < 7; ++k)
        for (int i = 0; i < n; ++i)
          census[static_cast<std::size_t>(k) * static_cast<std::size_t>(n) + static_cast<std::size_t>(i)] =
              cols[k]->empty() ? 0 : (*cols[k])[static_cast<std::size_t>(i)];
    }
    if (counts) {
      counts[0] = static_cast<long long>(r.stats.bonds);
      counts[1] = static_cast<long long>(nb.pairs);
      counts[2] = static_cast<long long>(a.nall());
      counts[3] = static_cast<long long>(f.entries());
    }
    return 0;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return 1;
  }
}

// The per-atom tallies and the bond table of the cpu64 engine (BondedOptions::per_atom / bond_table,
// NonbondedOptions::per_atom): eatom[n] and vatom[6n] folded from owned + ghost atoms onto the owners (the reverse
// communication of LAMMPS); the bond table of the owned atoms with the partners mapped to their owners
// (bond_start[n+1], bond_partner / bond_bo of at most bond_cap bonds, total_bo[n], nlp[n]). Returns the number of bonds,
// or -1 with a message in err.
long long ref_peratom(const char* ffield_text, const double* origin3, const double* box9, const int* periodic3, int n,
                      const double* x, const int* type, const long long* tag, const double* q, double shell, double* eatom,
                      double* vatom, int* bond_start, int* bond_partner, double* bond_bo, long long bond_cap, double* total_bo,
                      double* nlp, char* err, int errlen) {
  try {
    const ForceField ff = parse_force_field(ffield_text, "ffield");
    ControlParams ctl;
    NeighborCutoffs cut;
    cut.nonb = ff.file_control().nonb_cut;
    cut.bond = ctl.bond_cut;
    cut.hbond = ctl.hbond_cut;
    Box box;
    for (int c = 0; c < 3; ++c) box.origin[static_cast<std::size_t>(c)] = origin3[c];
    for (int v = 0; v < 3; ++v)
      for (int c = 0; c < 3; ++c) box.vectors[static_cast<std::size_t>(v)][static_cast<std::size_t>(c)] = box9[3 * v + c];
    for (int d = 0; d < 3; ++d) box.periodic[static_cast<std::size_t>(d)] = periodic3[d] != 0;
    std::vector<double> xs(x, x + 3 * static_cast<std::size_t>(n));
    std::vector<int> ty(type, type + n);
    std::vector<std::int64_t> tg(tag, tag + n);
    ExpandOptions eo;
    eo.shell = shell > 0 ? shell : cut.required_shell();
    const AtomSet a = expand_images(box, xs, ty, tg, eo);
    const FarList f = build_far_list(a, cut);
    BondedOptions bo;
    bo.per_atom = true;
    bo.bond_table = true;
    const BondedResult r = compute_bonded_core(ff, ctl, a, f, bo);
    NonbondedOptions no;
    no.per_atom = true;
    std::vector<double> qv(q, q + n);
    const NonbondedResult nb = compute_nonbonded_core(ff, cut, a, f, qv, no);
    for (int i = 0; i < n; ++i) eatom[i] = 0.0;
    for (int i = 0; i < 6 * n; ++i) vatom[i] = 0.0;
    for (std::size_t i = 0; i < a.nall(); ++i) {
      const std::size_t o = static_cast<std::size_t>(a.owner[i]);
      eatom[o] += r.eatom[i] + nb.eatom[i];
      for (std::size_t c = 0; c < 6; ++c) vatom[6 * o + c] += r.vatom[i][c] + nb.vatom[i][c];
    }
    const BondTable& t = r.table;
    const long long nbonds = t.start.empty() ? 0 : t.start.back();
    if (bond_start && nbonds <= bond_cap) {
      for (int i = 0; i <= n; ++i) bond_start[i] = t.start[static_cast<std::size_t>(i)];
      for (long long k = 0; k < nbonds; ++k) {
        bond_partner[k] = a.owner[static_cast<std::size_t>(t.nbr[static_cast<std::size_t>(k)])];
        bond_bo[k] = t.bo[static_cast<std::size_t>(k)];
      }
      for (int i = 0; i < n; ++i) { total_bo[i] = t.total_bo[static_cast<std::size_t>(i)]; nlp[i] = t.nlp[static_cast<std::size_t>(i)]; }
    }
    return nbonds;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return -1;
  }
}

// to_lammps_pvector (src/core/energy_terms.cpp:64-72) of 13 energies in EnergyTerm order.
void ref_pvector(const double* e13, double* out14) {
  EnergyBreakdown b;
  for (std::size_t t = 0; t < kEnergyTermCount; ++t) b.e[t] = e13[t];
  const auto pv = to_lammps_pvector(b);
  for (std::size_t k = 0; k < kPvectorSize; ++k) out14[k] = pv[k];
}

}  // extern "C"
