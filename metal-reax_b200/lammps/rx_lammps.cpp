// The LAMMPS side of the CUDA backend (see rx_lammps.hpp).
#include "rx_lammps.hpp"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace rx_lammps {

void lattice_of(const LammpsBox& b, double origin[3], double box9[9]) {
  for (int d = 0; d < 3; ++d) origin[d] = b.boxlo[d];
  const double lx = b.boxhi[0] - b.boxlo[0], ly = b.boxhi[1] - b.boxlo[1], lz = b.boxhi[2] - b.boxlo[2];
  const double v[9] = {lx, 0.0, 0.0, b.xy, ly, 0.0, b.xz, b.yz, lz};
  std::memcpy(box9, v, sizeof v);
}

RxLammps::RxLammps(int device) {
  ctx_ = rx_create(device);
  if (!ctx_) throw std::runtime_error(std::string("CUDA backend: ") + rx_last_error(nullptr));
}

RxLammps::~RxLammps() { rx_destroy(ctx_); }

void RxLammps::check(int rc) const {
  if (rc != RX_OK) throw std::runtime_error(std::string("CUDA backend: ") + rx_last_error(ctx_));
}

void RxLammps::coeff(const std::string& text, const std::vector<std::string>& type_elements, bool lgvdw) {
  check(rx_set_forcefield(ctx_, text.c_str(), lgvdw ? 1 : 0));
  map_.assign(type_elements.size(), -1);
  for (size_t t = 0; t < type_elements.size(); ++t) {
    if (type_elements[t] == "NULL") continue;
    const int k = rx_forcefield_element(ctx_, type_elements[t].c_str());
    if (k < 0) throw std::runtime_error("Non-existent ReaxFF type");
    map_[t] = k;
  }
  if (std::all_of(map_.begin(), map_.end(), [](int k) { return k < 0; }))
    throw std::runtime_error("Incorrect args for pair coefficients");
  tags_.clear();   // the next compute lays the system out again
}

void RxLammps::control(double bond_cut, double hbond_cut, double thb_cut, double thb_cutsq, bool enobonds) {
  check(rx_set_control(ctx_, bond_cut, hbond_cut, thb_cut, thb_cutsq, enobonds ? 1 : 0));
}

void RxLammps::qeq(double swa, double swb, double tol, int maxiter, bool strict) {
  check(rx_set_qeq(ctx_, swa, swb, tol, maxiter, strict ? 1 : 0));
}

// The engine's system: the handled owned atoms in LAMMPS's local order. A new atom set (after re-neighbouring atoms may
// migrate or be reordered) is handed over again with rx_set_systems, which keeps each atom's charge warm start by
// tag; positions alone go through rx_set_positions.
void RxLammps::layout(int nlocal, const double* const* x, const int* type, const int64_t* tag, const LammpsBox& box) {
  if (map_.empty()) throw std::runtime_error("CUDA backend: pair_coeff first");
  std::vector<int> sel;
  std::vector<int64_t> tg;
  std::vector<int> ty;
  sel.reserve(static_cast<size_t>(nlocal));
  for (int i = 0; i < nlocal; ++i) {
    if (type[i] < 1 || static_cast<size_t>(type[i]) > map_.size()) throw std::runtime_error("CUDA backend: atom type out of range");
    const int k = map_[static_cast<size_t>(type[i] - 1)];
    if (k < 0) continue;
    sel.push_back(i);
    tg.push_back(tag[i]);
    ty.push_back(k);
  }
  if (sel.empty()) throw std::runtime_error("CUDA backend: no atom of a handled type");
  double origin[3], box9[9];
  lattice_of(box, origin, box9);
  const bool same = tg == tags_ && ty == types_ && std::memcmp(origin, origin_, sizeof origin) == 0 &&
                    std::memcmp(box9, box9_, sizeof box9) == 0 && std::memcmp(box.periodic, periodic_, sizeof periodic_) == 0;
  xbuf_.resize(3 * sel.size());
  for (size_t a = 0; a < sel.size(); ++a)
    for (int c = 0; c < 3; ++c) xbuf_[3 * a + static_cast<size_t>(c)] = x[sel[a]][c];
  if (!same) {
    const int natoms = static_cast<int>(sel.size());
    check(rx_set_systems(ctx_, 1, &natoms, origin, box9, box.periodic, ty.data(), tg.data()));
    sel_ = std::move(sel);
    tags_ = std::move(tg);
    types_ = std::move(ty);
    std::memcpy(origin_, origin, sizeof origin);
    std::memcpy(box9_, box9, sizeof box9);
    std::memcpy(periodic_, box.periodic, sizeof periodic_);
  }
  check(rx_set_positions(ctx_, xbuf_.data()));
}

void RxLammps::compute(int nlocal, const double* const* x, const int* type, const int64_t* tag, const double* q, const LammpsBox& box,
                       double* const* f, Result& out, double* eatom, double (*vatom)[6]) {
  layout(nlocal, x, type, tag, box);
  const size_t n = sel_.size();
  qbuf_.resize(n);
  for (size_t a = 0; a < n; ++a) qbuf_[a] = q[sel_[a]];
  check(rx_set_charges(ctx_, qbuf_.data()));
  double e13[13];
  gbuf_.resize(3 * n);
  const bool pa = eatom || vatom;
  check(rx_compute(ctx_, pa ? RX_COMPUTE_PERATOM : 0, e13, gbuf_.data(), nullptr, nullptr));
  for (size_t a = 0; a < n; ++a)
    for (int c = 0; c < 3; ++c) f[sel_[a]][c] -= gbuf_[3 * a + static_cast<size_t>(c)];   // as pair_reaxff_metal.cpp:500-504
  check(rx_pvector(e13, out.pvector, &out.eng_vdwl, &out.eng_coul));
  check(rx_get_virial(ctx_, out.virial));
  if (pa) {
    std::vector<double> ea(n), va(6 * n);
    check(rx_get_peratom(ctx_, ea.data(), va.data()));
    for (size_t a = 0; a < n; ++a) {
      if (eatom) eatom[sel_[a]] += ea[a];
      if (vatom)
        for (int c = 0; c < 6; ++c) vatom[sel_[a]][c] += va[6 * a + static_cast<size_t>(c)];
    }
  }
}

std::pair<int, int> RxLammps::equilibrate(int nlocal, const double* const* x, const int* type, const int64_t* tag,
                                          const LammpsBox& box, double* q) {
  layout(nlocal, x, type, tag, box);
  int it[2];
  double rel[2];
  check(rx_qeq_solve(ctx_, it, rel));
  qbuf_.resize(sel_.size());
  check(rx_get_charges(ctx_, qbuf_.data()));
  for (size_t a = 0; a < sel_.size(); ++a) q[sel_[a]] = qbuf_[a];
  return {it[0], it[1]};
}

}  // namespace rx_lammps
