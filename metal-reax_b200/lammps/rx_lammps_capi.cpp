// A flat C entry to the LAMMPS-side bridge (rx_lammps.hpp) for hosts that drive it without C++ (LAMMPS's Python
// module, a Fortran caller, the tests): LAMMPS-layout arrays in, forces added into f, pair energy vector and virial out.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rx_lammps.hpp"

namespace {
thread_local std::string g_err;
template <class F>
int guard(F&& f) {
  try {
    f();
    g_err.clear();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
// the bridge behind a handle; a null handle (rxl_create failed, e.g. no usable GPU) is an error, not a crash
rx_lammps::RxLammps* obj(void* h) {
  if (!h) throw std::runtime_error("CUDA backend: null bridge handle (rxl_create failed)");
  return static_cast<rx_lammps::RxLammps*>(h);
}
}  // namespace

extern "C" {

const char* rxl_last_error() { return g_err.c_str(); }

void* rxl_create(int device) {
  void* out = nullptr;
  guard([&] { out = new rx_lammps::RxLammps(device); });
  return out;
}

void rxl_destroy(void* h) { delete static_cast<rx_lammps::RxLammps*>(h); }

// elements: ntypes symbols separated by spaces ("C H O NULL"), as on the pair_coeff line
int rxl_coeff(void* h, const char* ffield_text, const char* elements, int lgvdw) {
  return guard([&] {
    std::vector<std::string> el;
    std::string cur;
    for (const char* p = elements; ; ++p) {
      if (*p == ' ' || *p == 0) {
        if (!cur.empty()) el.push_back(cur);
        cur.clear();
        if (*p == 0) break;
      } else {
        cur.push_back(*p);
      }
    }
    obj(h)->coeff(ffield_text, el, lgvdw != 0);
  });
}

int rxl_type_element(void* h, int lammps_type) {
  int out = -2;
  guard([&] { out = obj(h)->type_element(lammps_type); });
  return out;
}

int rxl_lattice(const double* boxlo, const double* boxhi, double xy, double xz, double yz, double* origin3, double* box9) {
  rx_lammps::LammpsBox b;
  for (int d = 0; d < 3; ++d) { b.boxlo[d] = boxlo[d]; b.boxhi[d] = boxhi[d]; }
  b.xy = xy; b.xz = xz; b.yz = yz;
  rx_lammps::lattice_of(b, origin3, box9);
  return 0;
}

// x and f as flat nlocal x 3 arrays (LAMMPS's x[0] / f[0]); out14 the pair energy vector, out2 = (eng_vdwl, eng_coul),
// virial6; eatom (nlocal) may be NULL
int rxl_compute(void* h, int nlocal, const double* x, const int* type, const int64_t* tag, const double* q, const double* boxlo,
                const double* boxhi, const double* tilt3, const int* periodic, double* f, double* out14, double* out2,
                double* virial6, double* eatom) {
  return guard([&] {
    std::vector<const double*> xp(static_cast<size_t>(nlocal));
    std::vector<double*> fp(static_cast<size_t>(nlocal));
    for (int i = 0; i < nlocal; ++i) { xp[static_cast<size_t>(i)] = x + 3 * static_cast<size_t>(i); fp[static_cast<size_t>(i)] = f + 3 * static_cast<size_t>(i); }
    rx_lammps::LammpsBox b;
    for (int d = 0; d < 3; ++d) { b.boxlo[d] = boxlo[d]; b.boxhi[d] = boxhi[d]; b.periodic[d] = periodic ? periodic[d] : 1; }
    if (tilt3) { b.xy = tilt3[0]; b.xz = tilt3[1]; b.yz = tilt3[2]; }
    rx_lammps::Result r;
    obj(h)->compute(nlocal, xp.data(), type, tag, q, b, fp.data(), r, eatom);
    if (out14) std::memcpy(out14, r.pvector, sizeof r.pvector);
    if (out2) { out2[0] = r.eng_vdwl; out2[1] = r.eng_coul; }
    if (virial6) std::memcpy(virial6, r.virial, sizeof r.virial);
  });
}

int rxl_equilibrate(void* h, int nlocal, const double* x, const int* type, const int64_t* tag, const double* boxlo,
                    const double* boxhi, const double* tilt3, const int* periodic, double* q, int* iters2) {
  return guard([&] {
    std::vector<const double*> xp(static_cast<size_t>(nlocal));
    for (int i = 0; i < nlocal; ++i) xp[static_cast<size_t>(i)] = x + 3 * static_cast<size_t>(i);
    rx_lammps::LammpsBox b;
    for (int d = 0; d < 3; ++d) { b.boxlo[d] = boxlo[d]; b.boxhi[d] = boxhi[d]; b.periodic[d] = periodic ? periodic[d] : 1; }
    if (tilt3) { b.xy = tilt3[0]; b.xz = tilt3[1]; b.yz = tilt3[2]; }
    const auto it = obj(h)->equilibrate(nlocal, xp.data(), type, tag, b, q);
    if (iters2) { iters2[0] = it.first; iters2[1] = it.second; }
  });
}

}  // extern "C"
