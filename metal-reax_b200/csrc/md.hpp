// Device state and kernels of the NVT integrator (md_kernels.cu).
#pragma once
#include "device.cuh"

namespace rx {

constexpr int kMaxChain = 8;

struct MdDev {
  double4* v;        // velocities (A/fs)
  const double* mass;  // per force-field type (g/mol)
  double* ke;        // per system (kcal/mol)
  double* temp;      // per system (K)
  double* scale;     // per system velocity scale of the last chain half-step
  double* xi;        // nsys * kMaxChain chain positions
  double* vxi;       // nsys * kMaxChain chain velocities
  double dt, t_start, t_stop, t_damp;
  int chain;
  // kinetic energy in fixed chunks of kKeChunk atoms per system (the sum of a system depends only on its atoms)
  double* kpart;            // one partial per chunk
  const int* kchunk_first;  // nsys + 1: first chunk of each system
  const int* kchunk_sys;    // system of each chunk
  int nchunks;
  // temperature ramp of the current run (device-resident, so a captured step takes no per-step argument):
  // ramp[0] = steps done in this run, ramp[1] = steps of the run; T = t_start + (done / steps) (t_stop - t_start)
  double* ramp;
  // serving: per-system target temperature (null: the ramp above for every system) and per-system activity
  // (null: all active; 0: the system is frozen - its atoms and its chain are not advanced)
  const double* t_sys;
  const int* active;
};

constexpr int kKeChunk = 1024;

__global__ void k_md_kinetic_part(MdDev m, const SysInfo* sys, const int* type);
__global__ void k_md_kinetic_sum(MdDev m, int nsys);
__global__ void k_md_chain(MdDev m, const SysInfo* sys, int nsys, int from_ke);
__global__ void k_md_scale_kick(MdDev m, const int* type, const int* sys_of, const double4* grad, double4* x, int na);
__global__ void k_md_kick_kinetic(MdDev m, const SysInfo* sys, const int* type, const int* sys_of, const double4* grad);
__global__ void k_md_scale(MdDev m, const int* sys_of, int na, int advance);

__global__ void k_gather_state(int n, const int* src, const double4* ox, const double* oq, const double* osh,
                               const double* oth, double4* x, double* q, double* sh, double* th);
__global__ void k_gather_vel(int n, const int* src, const double4* ov, double4* v);
__global__ void k_unpack3(int n, const double* in3, double4* out);
__global__ void k_pack3(int n, const double4* in, double* out3);

}  // namespace rx
