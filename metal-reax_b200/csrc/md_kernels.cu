// Velocity Verlet with a Nose-Hoover chain thermostat (NVT), per system; chain length 0 is plain NVE.
//
// The reference leaves time integration to LAMMPS (`fix nvt temp Tstart Tstop Tdamp`). This is the
// Martyna-Tuckerman-Klein chain (Mol. Phys. 87, 1117 (1996)) applied for dt/2 before the first velocity half-kick
// and after the second, with chain masses Q_1 = Nf kT tau^2 and Q_k = kT tau^2 (tau = Tdamp), Nf = 3N - 3.
// Units LAMMPS `real`: v in A/fs, forces kcal/mol/A, masses g/mol.
#include "device.cuh"
#include "md.hpp"

namespace rx {

namespace {
constexpr double kFtm2v = 1.0 / 48.88821291 / 48.88821291;   // (kcal/mol/A)/(g/mol) -> A/fs^2
constexpr double kMvv2e = 48.88821291 * 48.88821291;         // (g/mol) A^2/fs^2 -> kcal/mol
constexpr double kBoltz = 0.0019872067;                      // kcal/mol/K
}  // namespace

// kinetic energy: one block per chunk of kKeChunk atoms of a system, a fixed-shape tree per chunk
__global__ void k_md_kinetic_part(MdDev m, const SysInfo* sys, const int* type) {
  const int c = blockIdx.x;
  const int s = m.kchunk_sys[c];
  const SysInfo& si = sys[s];
  const int a0 = si.begin + (c - m.kchunk_first[s]) * kKeChunk;
  const int a1 = min(a0 + kKeChunk, si.begin + si.natoms);
  __shared__ double sh[256];
  double v2 = 0.0;
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const double4 v = m.v[a];
    v2 += m.mass[type[a]] * (v.x * v.x + v.y * v.y + v.z * v.z);
  }
  sh[threadIdx.x] = v2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) m.kpart[c] = sh[0];
}

// kinetic energy (kcal/mol) of a system from its chunk partials, in chunk order
__device__ inline double system_ke(const MdDev& m, int s) {
  double t = 0.0;
  for (int c = m.kchunk_first[s]; c < m.kchunk_first[s + 1]; ++c) t += m.kpart[c];
  return 0.5 * kMvv2e * t;
}

__global__ void k_md_kinetic_sum(MdDev m, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) m.ke[s] = system_ke(m, s);
}

// one thread per system: advance the chain by dt/2 and produce the velocity scale factor. The kinetic energy is the
// chunk partials' sum (from_ke 0) or m.ke (from_ke 1: the value the previous half step left, s^2 times the energy it
// scaled, which is the kinetic energy of the velocities as they stand)
__global__ void k_md_chain(MdDev m, const SysInfo* sys, int nsys, int from_ke) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  if (m.active && !m.active[s]) {
    m.scale[s] = 1.0;
    return;
  }
  const int M = m.chain;
  if (M == 0) {   // NVE: no thermostat; the current kinetic energy and temperature only
    const double nf0 = 3.0 * sys[s].natoms - 3.0;
    const double ke = from_ke ? m.ke[s] : system_ke(m, s);
    m.scale[s] = 1.0;
    m.ke[s] = ke;
    m.temp[s] = nf0 > 0.0 ? 2.0 * ke / (nf0 * kBoltz) : 0.0;
    return;
  }
  const double step_frac = m.ramp[1] > 0.0 ? m.ramp[0] / m.ramp[1] : 0.0;
  double* xi = m.xi + s * kMaxChain;
  double* vx = m.vxi + s * kMaxChain;
  const double T = m.t_sys ? m.t_sys[s] : m.t_start + step_frac * (m.t_stop - m.t_start);
  const double kT = kBoltz * T;
  const double nf = 3.0 * sys[s].natoms - 3.0;
  const double tau2 = m.t_damp * m.t_damp;
  double Q[kMaxChain];
  Q[0] = nf * kT * tau2;
  for (int k = 1; k < M; ++k) Q[k] = kT * tau2;
  const double dt = m.dt, dt2 = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  double ke2 = 2.0 * (from_ke ? m.ke[s] : system_ke(m, s));
  auto G = [&](int k) { return k == 0 ? (ke2 - nf * kT) / Q[0] : (Q[k - 1] * vx[k - 1] * vx[k - 1] - kT) / Q[k]; };
  vx[M - 1] += G(M - 1) * dt4;
  for (int k = M - 2; k >= 0; --k) {
    const double e = exp(-vx[k + 1] * dt8);
    vx[k] *= e;
    vx[k] += G(k) * dt4;
    vx[k] *= e;
  }
  const double scale = exp(-vx[0] * dt2);
  ke2 *= scale * scale;
  for (int k = 0; k < M; ++k) xi[k] += vx[k] * dt2;
  for (int k = 0; k < M - 1; ++k) {
    const double e = exp(-vx[k + 1] * dt8);
    vx[k] *= e;
    vx[k] += G(k) * dt4;
    vx[k] *= e;
  }
  vx[M - 1] += G(M - 1) * dt4;
  m.scale[s] = scale;
  m.ke[s] = 0.5 * ke2;
  m.temp[s] = ke2 / (nf * kBoltz);
}

// velocities times their system's chain scale; with `advance` (the second half of a step) the ramp's step count too
__global__ void k_md_scale(MdDev m, const int* sys_of, int na, int advance) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (advance && a == 0) m.ramp[0] += 1.0;
  if (a >= na) return;
  const double sc = m.scale[sys_of[a]];
  double4 v = m.v[a];
  v.x *= sc; v.y *= sc; v.z *= sc;
  m.v[a] = v;
}

// first half of a step, fused: v *= the chain's scale, v += dt/2 F/m (F = -grad), x += dt v
__global__ void k_md_scale_kick(MdDev m, const int* type, const int* sys_of, const double4* grad, double4* x, int na) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= na) return;
  const int s = sys_of[a];
  if (m.active && !m.active[s]) return;
  const double sc = m.scale[s];
  const double c = 0.5 * m.dt * kFtm2v / m.mass[type[a]];
  const double4 g = grad[a];
  double4 v = m.v[a];
  v.x *= sc; v.y *= sc; v.z *= sc;
  v.x -= c * g.x; v.y -= c * g.y; v.z -= c * g.z;
  m.v[a] = v;
  double4 p = x[a];
  p.x += m.dt * v.x; p.y += m.dt * v.y; p.z += m.dt * v.z;
  x[a] = p;
}

// second half of a step, fused: v += dt/2 F/m for the atoms of one kinetic-energy chunk, then the chunk's sum of
// m v^2 in the fixed order of k_md_kinetic_part
__global__ void k_md_kick_kinetic(MdDev m, const SysInfo* sys, const int* type, const int* sys_of, const double4* grad) {
  const int c = blockIdx.x;
  const int s = m.kchunk_sys[c];
  const SysInfo& si = sys[s];
  const int a0 = si.begin + (c - m.kchunk_first[s]) * kKeChunk;
  const int a1 = min(a0 + kKeChunk, si.begin + si.natoms);
  const bool act = !(m.active && !m.active[s]);
  __shared__ double sh[256];
  double v2 = 0.0;
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const double mass = m.mass[type[a]];
    double4 v = m.v[a];
    if (act) {
      const double cf = 0.5 * m.dt * kFtm2v / mass;
      const double4 g = grad[a];
      v.x -= cf * g.x; v.y -= cf * g.y; v.z -= cf * g.z;
      m.v[a] = v;
    }
    v2 += mass * (v.x * v.x + v.y * v.y + v.z * v.z);
  }
  sh[threadIdx.x] = v2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) m.kpart[c] = sh[0];
}

// continuous batching: carry the state of kept atoms (new index a, old index src[a]) into the re-laid-out arrays
__global__ void k_gather_state(int n, const int* src, const double4* ox, const double* oq, const double* osh,
                               const double* oth, double4* x, double* q, double* sh, double* th) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int o = src[a];
  x[a] = ox[o];
  q[a] = oq[o];
  for (int k = 0; k < 4; ++k) {
    sh[4 * static_cast<size_t>(a) + k] = osh[4 * static_cast<size_t>(o) + k];
    th[4 * static_cast<size_t>(a) + k] = oth[4 * static_cast<size_t>(o) + k];
  }
}

__global__ void k_gather_vel(int n, const int* src, const double4* ov, double4* v) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  v[a] = ov[src[a]];
}

// host layout (3 doubles per atom) <-> device layout (double4), for copies straight from and into pinned caller memory
__global__ void k_unpack3(int n, const double* in3, double4* out) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  out[a] = make_double4(in3[3 * static_cast<size_t>(a)], in3[3 * static_cast<size_t>(a) + 1], in3[3 * static_cast<size_t>(a) + 2], 0.0);
}
__global__ void k_pack3(int n, const double4* in, double* out3) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const double4 v = in[a];
  out3[3 * static_cast<size_t>(a)] = v.x;
  out3[3 * static_cast<size_t>(a) + 1] = v.y;
  out3[3 * static_cast<size_t>(a) + 2] = v.z;
}

}  // namespace rx
