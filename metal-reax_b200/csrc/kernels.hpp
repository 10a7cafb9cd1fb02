// Kernel entry points and their argument structs (shared by the kernel files and the host engine).
#pragma once
#include "device.cuh"
#include "ffield.hpp"

namespace rx {

constexpr int SB_N = SB_NFIELDS;
constexpr int TB_N = TB_NFIELDS;

struct QeqParams {
  double swa, swb;
  double tap[8];   // taper coefficients on [swa, swb]
};

// per-system state of the segmented (batched) CG
struct SysCg {
  double sig_s, sig_t, bnorm_s, bnorm_t, alpha_s, alpha_t, beta_s, beta_t;
  int act_s, act_t, it_s, it_t, live, breakdown;
  unsigned counter;   // rows of this system that have arrived in the current pass
};

struct CgArgs {
  int begin, n, imax;
  double tol;
  double2* x;      // (s, t)
  double2* b;
  double2* r;
  double2* d;
  double2* p;
  double2* q;
  float2* df;     // FP32 copy of d, gathered by the single-precision-matrix iterations (single-system CG)
  double* eta;
  double* part;    // 2 * 8 * gridDim.x partial sums (double-buffered)
  int* out_iters;
  double* out_rel;
  int* out_nref;   // FP64 residual passes of the last single-system solve (may be null)
  int* out_brk;    // per system: 1 after a breakdown (a step length that is not finite)
  int write_q;     // 1: calculate_Q into the charges (the fix's solve); 0: solutions only
  // segmented CG only
  SysCg* sc;       // nsys
  double2* rb0;    // per-row dot-product terms (fixed-order per-system sums)
  double2* rb1;
  int* nlive;      // [2]: systems still iterating, by iteration parity
};

__global__ void k_wrap_bin(Dev d);
__global__ void k_cell_start(Dev d, const int* sorted_keys);
__global__ void k_nbr_check(Dev d);
__global__ void k_rebuild_flag(Dev d, cudaGraphConditionalHandle h);
__global__ void k_neighbors(Dev d, DevFF ff);
__global__ void k_pairs(Dev d, DevFF ff, QeqParams qp);
__global__ void k_nonbonded(Dev d, DevFF ff);
__global__ void k_nonbonded_half(Dev d, DevFF ff);
__global__ void k_acks2(Dev d, DevFF ff, const double* s_kin);
__global__ void k_cg_grid(Dev d, CgArgs a);
__global__ void k_cg_seg(Dev d, CgArgs a);
__global__ void k_qeq_prepare(Dev d, DevFF ff, CgArgs a, const double* s_hist, const double* t_hist);
__global__ void k_qeq_prepare_given(Dev d, DevFF ff, CgArgs a, const double* b, const double* x0);
__global__ void k_qeq_history(Dev d, const double2* x, double* s_hist, double* t_hist, int strict);
__global__ void k_qeq_matvec(Dev d, DevFF ff, const double2* v, double2* y);
__global__ void k_energy_part(Dev d, double* part, int nchunk);
__global__ void k_energy_final(Dev d, const double* part, int nchunk, double* out, double* out_vir);

__global__ void k_bonds(Dev d, DevFF ff, DevCtl ctl);
__global__ void k_bond_sym(Dev d);
__global__ void k_bo_correct(Dev d, DevFF ff, DevCtl ctl);
__global__ void k_atom_quantities(Dev d, DevFF ff);
__global__ void k_bonded_atom(Dev d, DevFF ff, DevCtl ctl);
__global__ void k_hbond(Dev d, DevFF ff, DevCtl ctl);
__global__ void k_torsion(Dev d, DevFF ff, DevCtl ctl);
__global__ void k_fold(Dev d);
__global__ void k_dbond(Dev d);
__global__ void k_force_final(Dev d);

}  // namespace rx
