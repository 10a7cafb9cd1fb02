// The LAMMPS side of `pair_style reaxff/metal NULL backend cuda` and `fix qeq/reaxff/metal`: everything the
// reference's adapter does between LAMMPS's arrays and its engine (plugin/adapter/pair_reaxff_metal.cpp:103-160,
// 412-524; plugin/adapter/fix_qeq_reaxff_metal.cpp:65-124), written against this engine's C ABI (include/rxcuda.h)
// and plain arrays, so that the pair style and the fix keep only their LAMMPS bookkeeping:
//
//   pair_coeff * * ffield C H O NULL   -> RxLammps::coeff(text, {"C","H","O","NULL"}, lgvdw)
//   PairReaxFFMetal::compute           -> RxLammps::compute(...) with atom->x/type/tag/q/f, domain box, flags
//   FixQEqReaxFFMetal::pre_force / CG  -> RxLammps::equilibrate(...) (both CG systems, charges into atom->q)
//
// Atoms of a NULL type are not handled by the style (no force, no energy), as pair reaxff. The engine takes the owned
// atoms only: periodic images live in its neighbor rows, so LAMMPS's ghost atoms are not passed, forces come back
// folded onto the owned atoms, and the pair's virial is set from the engine (the pair style turns virial_fdotr off).
// One RxLammps per MPI rank (each rank's owned atoms are independent periodic systems only when a single rank owns
// the box: the engine does not exchange halos).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

#include "../../include/rxcuda.h"

namespace rx_lammps {

// LAMMPS's box: boxlo/boxhi, tilt factors xy, xz, yz, and per-direction periodicity (domain->periodicity)
struct LammpsBox {
  double boxlo[3], boxhi[3];
  double xy = 0.0, xz = 0.0, yz = 0.0;
  int periodic[3] = {1, 1, 1};
};

// lattice vectors (rows a, b, c) and origin of a LAMMPS box (a = (lx,0,0), b = (xy,ly,0), c = (xz,yz,lz))
void lattice_of(const LammpsBox& b, double origin[3], double box9[9]);

struct Result {
  double pvector[14];      // pair->pvector (eb, ea, elp, emol, ev, epen, ecoa, ehb, et, eco, ew, ep, efi, eqeq)
  double eng_vdwl, eng_coul;
  double virial[6];        // pair->virial (xx, yy, zz, xy, xz, yz)
};

// An array exchanged with the engine every step (positions in, gradient out), in page-locked memory from
// rx_host_alloc, which rx_set_positions and rx_compute copy from and into directly; in ordinary memory where
// page-locked memory cannot be had (the engine then copies through its own staging buffer).
class HostBuf {
 public:
  HostBuf() = default;
  ~HostBuf() { release(); }
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  void resize(size_t n) {
    if (n <= cap_ && p_) { n_ = n; return; }
    release();
    const size_t bytes = (n > 0 ? n : 1) * sizeof(double);
    void* p = rx_host_alloc(bytes);
    pinned_ = p != nullptr;
    if (!p) p = std::malloc(bytes);
    if (!p) throw std::bad_alloc();
    p_ = static_cast<double*>(p);
    cap_ = n > 0 ? n : 1;
    n_ = n;
  }
  double* data() { return p_; }
  double& operator[](size_t i) { return p_[i]; }
  size_t size() const { return n_; }

 private:
  void release() {
    if (p_) {
      if (pinned_) rx_host_free(p_);
      else std::free(p_);
    }
    p_ = nullptr;
    cap_ = n_ = 0;
  }
  double* p_ = nullptr;
  size_t cap_ = 0, n_ = 0;
  bool pinned_ = false;
};

class RxLammps {
 public:
  explicit RxLammps(int device);
  ~RxLammps();
  RxLammps(const RxLammps&) = delete;
  RxLammps& operator=(const RxLammps&) = delete;

  // pair_coeff: the force-field text and the element of every LAMMPS type (index 0 = type 1; "NULL" = not handled).
  // Throws std::runtime_error with the engine's message ("Non-existent ReaxFF type" for an unknown element).
  void coeff(const std::string& ffield_text, const std::vector<std::string>& type_elements, bool lgvdw);
  // pair_style keywords: cut-offs and enobonds; fix qeq/reaxff/metal: taper, tolerance, maxiter, strict
  void control(double bond_cut, double hbond_cut, double thb_cut, double thb_cutsq, bool enobonds);
  void qeq(double swa, double swb, double tol, int maxiter, bool strict);
  int type_element(int lammps_type) const { return map_.at(static_cast<size_t>(lammps_type - 1)); }

  // PairReaxFFMetal::compute: the owned atoms (x[nlocal][3], 1-based types, tags, charges) of this rank; forces are
  // ADDED to f[nlocal][3] (f -= dE/dx); per-atom energies/virials are added when the arrays are given.
  void compute(int nlocal, const double* const* x, const int* type, const int64_t* tag, const double* q, const LammpsBox& box,
               double* const* f, Result& out, double* eatom = nullptr, double (*vatom)[6] = nullptr);
  // FixQEqReaxFFMetal (resident): both CG systems from the engine's warm starts for the current positions; the charges
  // go to q[nlocal] (atoms of a NULL type keep theirs). Returns the iteration counts (s, t).
  std::pair<int, int> equilibrate(int nlocal, const double* const* x, const int* type, const int64_t* tag, const LammpsBox& box,
                                  double* q);

  rx_context* context() { return ctx_; }

 private:
  void layout(int nlocal, const double* const* x, const int* type, const int64_t* tag, const LammpsBox& box);
  void check(int rc) const;

  rx_context* ctx_ = nullptr;
  std::vector<int> map_;            // LAMMPS type - 1 -> force-field type index, -1 = NULL
  std::vector<int> sel_;            // engine atom -> LAMMPS local index
  std::vector<int64_t> tags_;       // tags of the engine atoms (a changed set means re-laying out the system)
  std::vector<int> types_;
  double origin_[3] = {0, 0, 0}, box9_[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int periodic_[3] = {1, 1, 1};
  HostBuf xbuf_, gbuf_;              // positions in, gradient out: every step
  std::vector<double> qbuf_;
};

}  // namespace rx_lammps
