// Cell lists, full neighbor rows with the charge matrix, non-bonded forces, charge-equilibration CG, energy sums.
#include <cooperative_groups.h>

#include "device.cuh"
#include "kernels.hpp"

namespace cg = cooperative_groups;

namespace rx {

// ------------------------------------------------------------------------------------------------ Verlet check
// A system's Verlet rows stay valid while no atom of it has moved more than skin/2 since they were built (no pair can
// then have come from beyond nonb_cut + skin to within nonb_cut). Sets the system's rebuild flag otherwise.
__global__ void k_nbr_check(Dev d) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  // this evaluation's H-bond acceptor accumulators and per-atom energy tallies start from zero (the first kernel of an
  // evaluation: the bonded branch may start before the row filter)
  for (int c = 0; c < 3; ++c) d.fix_h[3 * static_cast<size_t>(a) + c] = 0ull;
  if (d.pe_on) d.pe_fix[a] = 0ull;
  const int s = d.sys_of[a];
  const double4 x = d.x[a];
  if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z))) {
    atomicOr(d.status, ST_NONFINITE);
    return;
  }
  if (*reinterpret_cast<volatile const int*>(d.sys_flag + s)) return;
  const double4 r = d.xref[a];
  double dx = x.x - r.x, dy = x.y - r.y, dz = x.z - r.z;
  {   // positions handed in by a caller may sit in another periodic image than the engine's own (wrapped at the last
      // rebuild): the atom moves to the image nearest its reference position, so that the rows' lattice shifts hold
    const SysInfo& sy = d.sys[s];
    double n[3];
    bool shift = false;
    for (int k = 0; k < 3; ++k) {
      n[k] = sy.per[k] ? rint(sy.R[3 * k] * dx + sy.R[3 * k + 1] * dy + sy.R[3 * k + 2] * dz) : 0.0;
      shift = shift || n[k] != 0.0;
    }
    if (shift) {
      double4 y = x;
      y.x -= n[0] * sy.L[0] + n[1] * sy.L[3] + n[2] * sy.L[6];
      y.y -= n[0] * sy.L[1] + n[1] * sy.L[4] + n[2] * sy.L[7];
      y.z -= n[0] * sy.L[2] + n[1] * sy.L[5] + n[2] * sy.L[8];
      d.x[a] = y;
      dx = y.x - r.x; dy = y.y - r.y; dz = y.z - r.z;
    }
  }
  if (dx * dx + dy * dy + dz * dz > d.half_skin2) atomicOr(d.sys_flag + s, 1);
}

// ------------------------------------------------------------------------------------------------ wrap + bin
// Atoms of systems being rebuilt are wrapped into the primary cell first (expand_images with wrap_owned,
// src/neighbor/neighbor.cpp:45-61), then binned into a uniform grid over the fractional coordinates of their system.
// Between rebuilds positions are never re-wrapped: the lattice shifts in the rows are relative to the positions of
// the last rebuild.
__global__ void k_wrap_bin(Dev d) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.na) return;
  const int sy = d.sys_of[a];
  if (!d.sys_flag[sy]) return;   // the atom keeps its key: its system's cells are not used this evaluation
  const SysInfo s = d.sys[sy];
  double4 x = d.x[a];
  double r[3] = {x.x, x.y, x.z};
  double f[3];
  for (int k = 0; k < 3; ++k) f[k] = s.R[3 * k] * (r[0] - s.origin[0]) + s.R[3 * k + 1] * (r[1] - s.origin[1]) + s.R[3 * k + 2] * (r[2] - s.origin[2]);
  bool moved = false;
  for (int k = 0; k < 3; ++k) {
    const double fl = floor(f[k]);
    if (fl != 0.0) {
      if (!s.per[k]) {   // never wrapped: the atom has left the extent the engine laid out for this direction
        atomicOr(d.status, ST_NONPERIODIC_ESCAPE);
        continue;
      }
      for (int c = 0; c < 3; ++c) r[c] -= fl * s.L[3 * k + c];
      moved = true;
    }
  }
  if (moved) {
    for (int k = 0; k < 3; ++k) f[k] = s.R[3 * k] * (r[0] - s.origin[0]) + s.R[3 * k + 1] * (r[1] - s.origin[1]) + s.R[3 * k + 2] * (r[2] - s.origin[2]);
    x.x = r[0]; x.y = r[1]; x.z = r[2];
    d.x[a] = x;
  }
  d.xref[a] = x;
  if (!(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]))) atomicOr(d.status, ST_NONFINITE);
  int c[3];
  for (int k = 0; k < 3; ++k) {
    int v = static_cast<int>(floor(f[k] * s.nc[k]));
    v = v < 0 ? 0 : (v >= s.nc[k] ? s.nc[k] - 1 : v);
    c[k] = v;
  }
  d.cell_key[a] = s.cell_begin + (c[2] * s.nc[1] + c[1]) * s.nc[0] + c[0];
}

// Sets the captured evaluation's rebuild conditional: 1 when any system's Verlet rows are to be rebuilt (its flag set
// by k_nbr_check or by the host), 0 otherwise, so that the wrap/bin, sort, cell-start and row kernels are skipped.
__global__ void k_rebuild_flag(Dev d, cudaGraphConditionalHandle h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  int mine = 0;
  for (int s = threadIdx.x; s < d.nsys; s += blockDim.x) mine |= d.sys_flag[s];
  if (mine) atomicOr(&any, 1);
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// cell_start[c] = first position in the sorted order whose key is >= c; positions gathered into cell order, relative to
// their system's origin and rounded to single precision (the candidate scan of the Verlet rows reads only these)
__global__ void k_cell_start(Dev d, const int* sorted_keys) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > d.na) return;
  const int prev = p == 0 ? -1 : sorted_keys[p - 1];
  const int cur = p == d.na ? d.ncell_total : sorted_keys[p];
  for (int c = prev + 1; c <= cur; ++c) d.cell_start[c] = p;
  if (p < d.na) {
    const int a = d.cell_atoms[p];
    const double4 x = d.x[a];
    const double* o = d.sys[d.sys_of[a]].origin;
    d.xs[p] = make_float4(static_cast<float>(x.x - o[0]), static_cast<float>(x.y - o[1]), static_cast<float>(x.z - o[2]),
                          static_cast<float>(d.type[a]));
  }
}

// ------------------------------------------------------------------------------------------------ neighbor rows
__device__ inline void taper_horner(const double* c, double r, double& Tap, double& dTap) {
  double t = c[7] * r + c[6];
  t = t * r + c[5]; t = t * r + c[4]; t = t * r + c[3]; t = t * r + c[2]; t = t * r + c[1]; t = t * r + c[0];
  double g = 7 * c[7] * r + 6 * c[6];
  g = g * r + 5 * c[5]; g = g * r + 4 * c[4]; g = g * r + 3 * c[3]; g = g * r + 2 * c[2];
  g += c[1] / r;
  Tap = t;
  dTap = g;
}

// Verlet rows, one warp per atom of a system being rebuilt: every image within nonb_cut + skin (a superset of the
// owned-row cut-off of build_far_list, src/neighbor/neighbor.cpp:180-212). The cells within `range` of the atom's cell
// are visited as runs of consecutive cells along x (one contiguous range of the cell-ordered atoms per run and periodic
// image), so the candidate loads are coalesced. Entries are written through a warp ballot in visiting order
// (deterministic). Rows only need to be supersets (every consumer re-tests its entries exactly in FP64 on the current
// positions), so candidates are tested in single precision against the system's thresholds SysInfo::vthr, which add
// the largest rounding error of that r^2 to the FP64 radii. The loops carry the wrapped cell and image of each row
// incrementally and prune with precomputed reciprocals: no division per run.
__global__ void __launch_bounds__(128, 6) k_neighbors(Dev d, DevFF ff) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  const int i = warp;
  const int sy = d.sys_of[i];
  if (!d.sys_flag[sy]) return;
  const SysInfo& s = d.sys[sy];
  const int nc0 = s.nc[0], nc1 = s.nc[1], nc2 = s.nc[2];
  const int key = d.cell_key[i] - s.cell_begin;
  const int cx = key % nc0, cy = (key / nc0) % nc1, cz = key / (nc0 * nc1);
  const double4 xi = d.x[i];
  int count = 0, count_near = 0, count_acc = 0;
  const unsigned lt = (1u << lane) - 1u;
  const int center = (d.S * d.S * d.S - 1) / 2;
  const size_t rowbase = static_cast<size_t>(i) * d.vcap;
  const bool hb_i = static_cast<int>(ff.sb[d.type[i] * SB_N + SB_P_HBOND]) == 1;
  const float tv = s.vthr[0], tn = s.vthr[1], ta = s.vthr[2];
  const int smax = d.smax, S = d.S, sbase = s.shift_base;
  const double oxi = xi.x - s.origin[0], oyi = xi.y - s.origin[1], ozi = xi.z - s.origin[2];
  // fractional coordinates of i: lower bounds of the distance to a cell slab prune whole runs and clip the x range
  double fi[3];
  for (int k = 0; k < 3; ++k) fi[k] = s.R[3 * k] * oxi + s.R[3 * k + 1] * oyi + s.R[3 * k + 2] * ozi;
  const double rc = sqrt(d.rv2) * (1.0 + 1e-9) + 1e-9;
  auto slab_gap = [&](int k, int c) {   // distance from i to the slab of cell index c (unwrapped) along direction k
    const double lo = static_cast<double>(c) * s.inv_nc[k], hi = static_cast<double>(c + 1) * s.inv_nc[k];
    const double g = fmax(0.0, fmax(lo - fi[k], fi[k] - hi));
    return fmax(0.0, g * s.h[k] - 1e-9 * s.h[k]);
  };
  auto advance = [](int& w, int& sh, int n) { if (++w == n) { w = 0; ++sh; } };
  int shz = floor_div(cz - s.range[2], nc2), wz = cz - s.range[2] - shz * nc2;
  const int shy0 = floor_div(cy - s.range[1], nc1), wy0 = cy - s.range[1] - shy0 * nc1;
  for (int zz = cz - s.range[2]; zz <= cz + s.range[2]; ++zz, advance(wz, shz, nc2)) {
    const double gz = slab_gap(2, zz);
    if (gz > rc) continue;
    int shy = shy0, wy = wy0;
    for (int yy = cy - s.range[1]; yy <= cy + s.range[1]; ++yy, advance(wy, shy, nc1)) {
      const double gy = slab_gap(1, yy);
      double rx;
      if (s.ortho) {
        const double g2 = gy * gy + gz * gz;
        if (g2 > rc * rc) continue;
        // single-precision square root widened past its rounding error: the x range only needs to be a superset
        rx = static_cast<double>(sqrtf(static_cast<float>(rc * rc - g2)) * 1.000001f) + 1e-6;
      } else {
        if (gy > rc) continue;
        rx = rc;
      }
      const int rowcell = s.cell_begin + (wz * nc1 + wy) * nc0;
      const double dfx = rx * s.inv_h[0];
      int xx = max(cx - s.range[0], static_cast<int>(floor((fi[0] - dfx) * nc0)));
      const int xend = min(cx + s.range[0], static_cast<int>(floor((fi[0] + dfx) * nc0)));
      if (xx > xend) continue;
      // wrapped cell and image of the first run; each further run starts a new image at cell 0
      int shx = __float2int_rd(static_cast<float>(xx) * s.inv_ncf0), wx0 = xx - shx * nc0;
      if (wx0 < 0) { wx0 += nc0; --shx; } else if (wx0 >= nc0) { wx0 -= nc0; ++shx; }
      for (; xx <= xend; wx0 = 0, ++shx) {
        const int len = min(nc0 - wx0, xend - xx + 1);
        xx += len;
        if (shx < -smax || shx > smax || shy < -smax || shy > smax || shz < -smax || shz > smax) {
          if (lane == 0) atomicOr(d.status, ST_SHIFT_RANGE);
          continue;
        }
        const int sidx = ((shx + smax) * S + (shy + smax)) * S + (shz + smax);
        const int c0 = d.cell_start[rowcell + wx0], c1 = d.cell_start[rowcell + wx0 + len];
        if (c0 >= c1) continue;
        // the run's image: separation = xs[p] + cimg, cimg = L s - (x_i - origin) in FP64 rounded once
        const double4 sh = d.shifts[sbase + sidx];
        const float3 cimg = make_float3(static_cast<float>(sh.x - oxi), static_cast<float>(sh.y - oyi), static_cast<float>(sh.z - ozi));
        for (int base = c0; base < c1; base += 32) {
          const int p = base + lane;
          bool ok = false;
          int j = 0;
          float r2 = 0.f, tj = 0.f;
          if (p < c1) {
            j = d.cell_atoms[p];
            const float4 xj = d.xs[p];
            tj = xj.w;
            if (!(j == i && sidx == center)) {
              const float dx = xj.x + cimg.x, dy = xj.y + cimg.y, dz = xj.z + cimg.z;
              r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
              ok = r2 <= tv;
            }
          }
          const unsigned code = static_cast<unsigned>(j) | (static_cast<unsigned>(sidx) << d.abits);
          const unsigned m = __ballot_sync(0xffffffffu, ok);
          if (ok) {
            const int pos = count + __popc(m & lt);
            if (pos < d.vcap) d.vrow[rowbase + pos] = code;
          }
          count += __popc(m);
          // the short Verlet rows of the bond and H-bond kernels (their own exact tests run on every evaluation)
          const bool nr = ok && r2 <= tn;
          const unsigned mn = __ballot_sync(0xffffffffu, nr);
          if (nr) {
            const int posn = count_near + __popc(mn & lt);
            if (posn < d.ncap_near) d.near[static_cast<size_t>(i) * d.ncap_near + posn] = code;
          }
          count_near += __popc(mn);
          if (hb_i) {   // warp-uniform
            const bool ac = ok && r2 <= ta && static_cast<int>(ff.sb[static_cast<int>(tj) * SB_N + SB_P_HBOND]) == 2;
            const unsigned ma = __ballot_sync(0xffffffffu, ac);
            if (ac) {
              const int posa = count_acc + __popc(ma & lt);
              if (posa < d.ncap_acc) d.acc[static_cast<size_t>(i) * d.ncap_acc + posa] = code;
            }
            count_acc += __popc(ma);
          }
        }
      }
    }
  }
  if (lane == 0) {
    d.vcnt[i] = count;
    if (count > d.vcap) {
      atomicOr(d.status, ST_VERLET_OVERFLOW);
      atomicMax(d.status + 4, count);
    }
    d.near_cnt[i] = count_near;
    if (count_near > d.ncap_near) {
      atomicOr(d.status, ST_NEAR_OVERFLOW);
      atomicMax(d.status + 3, count_near);
    }
    d.acc_cnt[i] = count_acc;
    if (count_acc > d.ncap_acc) {
      atomicOr(d.status, ST_ACC_OVERFLOW);
      atomicMax(d.status + 5, count_acc);
    }
  }
}

// The rows of this evaluation, one warp per atom: the entries of the Verlet row within nonb_cut, in Verlet-row order,
// with the exact FP64 distance test of build_far_list (every cut-off decision is the reference's). Fused: the
// charge-matrix entry H = 14.4 Tap(r) / cbrt(r^3 + (gamma_i gamma_j)^-1.5) for r <= swb (ENGINE_SPEC 7; fix_qeq_reaxff
// compute_H) stored as hi + lo single-precision parts. Also clears the per-system rebuild flags for the next evaluation.
__global__ void __launch_bounds__(256) k_pairs(Dev d, DevFF ff, QeqParams qp) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid < d.nsys) d.sys_flag[gid] = 0;
  const int warp = gid >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  if (lists_failed(d)) return;
  const int i = warp;
  const SysInfo s = d.sys[d.sys_of[i]];
  const double rc2 = ff.nonb_cut * ff.nonb_cut;
  const double4 xi = d.x[i];
  const int ti = d.type[i];
  const double* shld_i = ff.shld + static_cast<size_t>(ti) * ff.nt;
  int count = 0;
  const unsigned lt = (1u << lane) - 1u;
  const size_t vbase = static_cast<size_t>(i) * d.vcap, rowbase = static_cast<size_t>(i) * d.ncap;
  const int nv = min(d.vcnt[i], d.vcap);
  for (int base = 0; base < nv; base += 32) {
    const int e = base + lane;
    bool ok = false;
    unsigned code = 0;
    int j = 0;
    double r2 = 0.0;
    if (e < nv) {
      code = d.vrow[vbase + e];
      j = static_cast<int>(code & d.amask);
      double dv[3];
      pair_dvec_x(d, s, i, j, static_cast<int>(code >> d.abits), xi, d.x[j], dv);
      r2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
      ok = r2 <= rc2;
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      const int pos = count + __popc(m & lt);
      if (pos < d.ncap) {
        d.nbr[rowbase + pos] = code;
        const double r = sqrt(r2);
        double h = 0.0;
        if (r <= qp.swb) {
          double Tap, dTap;
          taper_horner(qp.tap, r, Tap, dTap);
          const double a3 = r * r * r + shld_i[d.type[j]];
          // z = a3^(-1/3): single-precision seed, then two Newton steps z <- z + (z/3)(1 - a3 z^3), which
          // square the relative error each (1e-7 -> 1e-14 -> rounding level); no division
          double z = static_cast<double>(rcbrtf(static_cast<float>(a3)));
          for (int k = 0; k < 2; ++k) z = fma(z * (1.0 / 3.0), fma(-a3 * z, z * z, 1.0), z);
          h = Tap * 14.4 * z;
        }
        const float hi = static_cast<float>(h);
        d.hhi[rowbase + pos] = hi;
        d.hlo[rowbase + pos] = static_cast<float>(h - static_cast<double>(hi));
      }
    }
    count += __popc(m);
  }
  if (lane == 0) {
    d.nbr_cnt[i] = count;
    if (count > d.ncap) {
      atomicOr(d.status, ST_NBR_OVERFLOW);
      atomicMax(d.status + 1, count);
    }
  }
}

// ------------------------------------------------------------------------------------------------ non-bonded
// The pair terms of one non-bonded entry at separation dvd (terms::nonbonded_pair, terms.hpp:282-323): returns CE with
// gradient -CE dvd on i and +CE dvd on the partner, and the pair's van der Waals and Coulomb energies.
__device__ __forceinline__ float nb_pair_terms(const DevFF& ff, int ti, int tj, float qi, float qj, const double* dvd,
                                               float p_vdW1, float p_vdW1i, float swa, float inv_dd, float& e_vdW,
                                               float& e_ele) {
  // the exact cut-off test was taken in FP64 when the row was filtered; the pair terms run in FP32, division-free:
  // 1/r from the reciprocal square root, reciprocals of the type-pair constants from the table, exp(a) as the square
  // of exp(a/2), and the Coulomb shielding through the reciprocal cube root z = (r^3 + gamma^-3)^(-1/3), whose cube
  // is 1/(r^3 + gamma^-3)
  const float r2f = static_cast<float>(dvd[0] * dvd[0] + dvd[1] * dvd[1] + dvd[2] * dvd[2]);
  const float inv_r = rsqrtf(r2f);
  const float r = r2f * inv_r;
  const float* pp = ff.nbf + (static_cast<size_t>(ti) * ff.nt + tj) * 12;
  float Tap, dTap;
  {   // taper_stable (include/reaxmetal/terms.hpp:268-272) in t = (r - swa)/(swb - swa)
    const float t = (r - swa) * inv_dd, t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
    Tap = 1.f - t4 * (35.f - 84.f * t + 70.f * t2 - 20.f * t3);
    dTap = (t3 * (-140.f + 420.f * t - 420.f * t2 + 140.f * t3)) * (inv_dd * inv_r);
  }
  const float alpha = pp[0], D = pp[1], inv_rvdw = pp[10];
  float CEvd;
  e_vdW = 0.f;
  if (ff.vdw_type == 1 || ff.vdw_type == 3) {
    const float powr_vdW1 = exp2f(p_vdW1 * __log2f(r));   // r^p and (..)^(1/p) through the fast base-2 pair
    const float sum = powr_vdW1 + pp[3];
    const float fn13 = exp2f(p_vdW1i * __log2f(sum));
    const float exp2 = __expf(0.5f * alpha * (1.f - fn13 * inv_rvdw));
    const float exp1 = exp2 * exp2;
    const float evd = D * (exp1 - 2.f * exp2);
    e_vdW += Tap * evd;
    // (sum)^(1/p - 1) r^(p - 2) = fn13 / sum * powr / r^2
    const float dfn13 = __fdividef(fn13, sum) * (powr_vdW1 * inv_r * inv_r);
    CEvd = dTap * evd - Tap * D * (alpha * inv_rvdw) * (exp1 - exp2) * dfn13;
  } else {
    const float exp2 = __expf(0.5f * alpha * (1.f - r * inv_rvdw));
    const float exp1 = exp2 * exp2;
    const float evd = D * (exp1 - 2.f * exp2);
    e_vdW += Tap * evd;
    CEvd = dTap * evd - Tap * D * (alpha * inv_rvdw) * (exp1 - exp2) * inv_r;
  }
  if (ff.vdw_type == 2 || ff.vdw_type == 3) {
    const float ecore = pp[4], acore = pp[5], inv_rcore = pp[11];
    const float e_core = ecore * __expf(acore * (1.f - r * inv_rcore));
    e_vdW += Tap * e_core;
    const float de_core = -(acore * inv_rcore) * e_core;
    CEvd += dTap * e_core + Tap * de_core * inv_r;
    if (ff.lg) {
      const float r4 = r2f * r2f, r5 = r4 * r, r6 = r4 * r2f, re6 = pp[9];
      const float inv6 = __fdividef(1.f, r6 + re6);
      const float e_lg = -pp[8] * inv6;
      e_vdW += Tap * e_lg;
      const float de_lg = -6.f * e_lg * r5 * inv6;
      CEvd += dTap * e_lg + Tap * de_lg * inv_r;
    }
  }
  const float z = rcbrtf(r2f * r + pp[7]);
  const float cq = 332.06371f * qi * qj;
  e_ele = cq * (Tap * z);
  const float CEclmb = cq * (dTap - Tap * r * (z * z * z)) * z;
  return CEvd + CEclmb;
}

// One warp per atom over its full row (FP32 pair arithmetic, FP64 accumulation). The gradient of atom i collects
// -CE * dvec from every entry of its own row, so no write ever touches another atom. Energies use the reference's
// counted pairs (owner-computes rule, classify_nonbonded_entry, src/neighbor/neighbor.cpp:295-310): an entry counts
// at i if it is owned-owned with j > i, or a periodic image with tag_i < tag_j or, for an image of i itself, the
// positive direction; each counted entry contributes its full pair energy (terms::nonbonded_pair, terms.hpp:282-323).
__global__ void k_nonbonded(Dev d, DevFF ff) {
  if (lists_failed(d)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  const int i = warp;
  const SysInfo s = d.sys[d.sys_of[i]];
  const int ti = d.type[i];
  const int cnt = min(d.nbr_cnt[i], d.ncap);
  const float p_vdW1 = static_cast<float>(ff.gp[28]), p_vdW1i = 1.f / p_vdW1;
  const float swa = static_cast<float>(ff.nonb_low), inv_dd = static_cast<float>(1.0 / (ff.nonb_cut - ff.nonb_low));
  const float qi = static_cast<float>(d.q[i]);
  const long long tag_i = d.tag[i];
  const int center = (d.S * d.S * d.S - 1) / 2;
  double gx = 0, gy = 0, gz = 0, ev = 0, ee = 0, ehalf = 0;
  float v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;   // pair virial, half per directed entry (lane partials)
  int counted = 0;
  const double4 xi4 = d.x[i];
  for (int e = lane; e < cnt; e += 32) {
    const unsigned code = d.nbr[static_cast<size_t>(i) * d.ncap + e];
    const int j = static_cast<int>(code & d.amask);
    const int sidx = static_cast<int>(code >> d.abits);
    double dvd[3];
    pair_dvec_x(d, s, i, j, sidx, xi4, d.x[j], dvd);
    const int tj = d.type[j];
    float e_vdW, e_ele;
    const float CE = nb_pair_terms(ff, ti, tj, qi, static_cast<float>(d.q[j]), dvd, p_vdW1, p_vdW1i, swa, inv_dd, e_vdW, e_ele);
    const float dx = static_cast<float>(dvd[0]), dy = static_cast<float>(dvd[1]), dz = static_cast<float>(dvd[2]);
    gx -= static_cast<double>(CE * dx);
    gy -= static_cast<double>(CE * dy);
    gz -= static_cast<double>(CE * dz);
    {   // the gradient -CE dv on i and +CE dv on the partner: virial -CE dv (x) dv, half of it from each direction
      const float c = -0.5f * CE;
      v0 += c * dx * dx; v1 += c * dy * dy; v2 += c * dz * dz;
      v3 += c * dx * dy; v4 += c * dx * dz; v5 += c * dy * dz;
    }
    // owner-computes counting of the energy
    bool count = false;
    if (sidx == center) count = j > i;
    else {
      const long long tag_j = d.tag[j];
      if (tag_i < tag_j) count = true;
      else if (tag_i == tag_j) {
        const double SMALL = 1e-4;
        if (dvd[2] > SMALL) count = true;
        else if (fabs(dvd[2]) < SMALL) {
          if (dvd[1] > SMALL) count = true;
          else if (fabs(dvd[1]) < SMALL && dvd[0] > SMALL) count = true;
        }
      }
    }
    if (count) {
      ev += static_cast<double>(e_vdW);
      ee += static_cast<double>(e_ele);
      ++counted;
    }
    ehalf += 0.5 * (static_cast<double>(e_vdW) + static_cast<double>(e_ele));   // per-atom tally: half of every pair
  }
  gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz); ev = warp_sum(ev); ee = warp_sum(ee);
  const double w0 = warp_sum(static_cast<double>(v0)), w1 = warp_sum(static_cast<double>(v1)), w2 = warp_sum(static_cast<double>(v2));
  const double w3 = warp_sum(static_cast<double>(v3)), w4 = warp_sum(static_cast<double>(v4)), w5 = warp_sum(static_cast<double>(v5));
  if (d.pe_on) ehalf = warp_sum(ehalf);
  for (int o = 16; o > 0; o >>= 1) counted += __shfl_xor_sync(0xffffffffu, counted, o);
  if (lane == 0) {
    d.fnb[i] = make_double4(gx, gy, gz, 0.0);
    double* vi = d.vir_nb + static_cast<size_t>(i) * kVir;
    vi[0] = w0; vi[1] = w1; vi[2] = w2; vi[3] = w3; vi[4] = w4; vi[5] = w5;
    d.eatom[static_cast<size_t>(i) * kTerms + E_VDW] = ev;
    d.eatom[static_cast<size_t>(i) * kTerms + E_ELE] = ee;
    const double chi = ff.sb[ti * SB_N + SB_CHI], eta = ff.sb[ti * SB_N + SB_ETA], qd = d.q[i];
    d.eatom[static_cast<size_t>(i) * kTerms + E_POL] = 23.02 * (chi * qd + (eta / 2.) * (qd * qd));
    if (d.pe_on) pe_add(d, i, ehalf + 23.02 * (chi * qd + (eta / 2.) * (qd * qd)));
    d.census[4 * d.na + i] = counted;
  }
}

// Each non-bonded pair once: the same terms as k_nonbonded over the counted entries of every row only (the
// owner-computes rule above picks exactly one entry of each pair), with the partner's gradient +CE dv added to its
// fixed-point accumulator (2^32 units: integer additions give the same sum in any order, so the result is
// deterministic). The counted entries of a row are gathered into a per-warp queue in row order, so every lane of a
// batch of 32 has a pair to compute. The pair virial goes whole to the owner; the per-atom split of energies and
// virials (RX_COMPUTE_PERATOM) takes k_nonbonded instead.
__global__ void __launch_bounds__(256) k_nonbonded_half(Dev d, DevFF ff) {
  if (lists_failed(d)) return;
  __shared__ unsigned queue[8][64];
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  if (warp >= d.na) return;
  const int i = warp;
  const SysInfo s = d.sys[d.sys_of[i]];
  const int ti = d.type[i];
  const int cnt = min(d.nbr_cnt[i], d.ncap);
  const float p_vdW1 = static_cast<float>(ff.gp[28]), p_vdW1i = 1.f / p_vdW1;
  const float swa = static_cast<float>(ff.nonb_low), inv_dd = static_cast<float>(1.0 / (ff.nonb_cut - ff.nonb_low));
  const float qi = static_cast<float>(d.q[i]);
  const long long tag_i = d.tag[i];
  const int center = (d.S * d.S * d.S - 1) / 2;
  const unsigned lt = (1u << lane) - 1u;
  double gx = 0, gy = 0, gz = 0, ev = 0, ee = 0;
  float v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;   // pair virials (lane partials)
  int counted = 0;
  const double4 xi4 = d.x[i];
  auto pair = [&](unsigned code) {
    const int j = static_cast<int>(code & d.amask);
    const int sidx = static_cast<int>(code >> d.abits);
    double dvd[3];
    pair_dvec_x(d, s, i, j, sidx, xi4, d.x[j], dvd);
    float e_vdW, e_ele;
    const float CE = nb_pair_terms(ff, ti, d.type[j], qi, static_cast<float>(d.q[j]), dvd, p_vdW1, p_vdW1i, swa, inv_dd,
                                   e_vdW, e_ele);
    const float dx = static_cast<float>(dvd[0]), dy = static_cast<float>(dvd[1]), dz = static_cast<float>(dvd[2]);
    const float fx = CE * dx, fy = CE * dy, fz = CE * dz;
    gx -= static_cast<double>(fx);
    gy -= static_cast<double>(fy);
    gz -= static_cast<double>(fz);
    fix_add(d.fix_h + 3 * static_cast<size_t>(j), static_cast<double>(fx));
    fix_add(d.fix_h + 3 * static_cast<size_t>(j) + 1, static_cast<double>(fy));
    fix_add(d.fix_h + 3 * static_cast<size_t>(j) + 2, static_cast<double>(fz));
    const float c = -CE;   // the pair virial -CE dv (x) dv, whole
    v0 += c * dx * dx; v1 += c * dy * dy; v2 += c * dz * dz;
    v3 += c * dx * dy; v4 += c * dx * dz; v5 += c * dy * dz;
    ev += static_cast<double>(e_vdW);
    ee += static_cast<double>(e_ele);
    ++counted;
  };
  int qn = 0;   // entries waiting in this warp's queue (warp-uniform)
  for (int base = 0; base < cnt; base += 32) {
    const int e = base + lane;
    bool own = false;
    unsigned code = 0;
    if (e < cnt) {
      code = d.nbr[static_cast<size_t>(i) * d.ncap + e];
      const int j = static_cast<int>(code & d.amask);
      const int sidx = static_cast<int>(code >> d.abits);
      if (sidx == center) {
        own = j > i;
      } else {
        const long long tag_j = d.tag[j];
        if (tag_i < tag_j) {
          own = true;
        } else if (tag_i == tag_j) {   // an image of i itself: the positive direction
          double dvd[3];
          pair_dvec_x(d, s, i, j, sidx, xi4, d.x[j], dvd);
          const double SMALL = 1e-4;
          if (dvd[2] > SMALL) own = true;
          else if (fabs(dvd[2]) < SMALL) {
            if (dvd[1] > SMALL) own = true;
            else if (fabs(dvd[1]) < SMALL && dvd[0] > SMALL) own = true;
          }
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, own);
    if (own) queue[wb][qn + __popc(m & lt)] = code;
    qn += __popc(m);
    __syncwarp();
    if (qn >= 32) {   // a full batch: one pair per lane; the rest moves to the front of the queue
      const unsigned mine = queue[wb][lane];
      const unsigned rest = lane + 32 < qn ? queue[wb][lane + 32] : 0u;
      __syncwarp();
      if (lane + 32 < qn) queue[wb][lane] = rest;
      __syncwarp();
      qn -= 32;
      pair(mine);
    }
  }
  if (lane < qn) pair(queue[wb][lane]);
  gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz); ev = warp_sum(ev); ee = warp_sum(ee);
  const double w0 = warp_sum(static_cast<double>(v0)), w1 = warp_sum(static_cast<double>(v1)), w2 = warp_sum(static_cast<double>(v2));
  const double w3 = warp_sum(static_cast<double>(v3)), w4 = warp_sum(static_cast<double>(v4)), w5 = warp_sum(static_cast<double>(v5));
  for (int o = 16; o > 0; o >>= 1) counted += __shfl_xor_sync(0xffffffffu, counted, o);
  if (lane == 0) {
    d.fnb[i] = make_double4(gx, gy, gz, 0.0);
    double* vi = d.vir_nb + static_cast<size_t>(i) * kVir;
    vi[0] = w0; vi[1] = w1; vi[2] = w2; vi[3] = w3; vi[4] = w4; vi[5] = w5;
    d.eatom[static_cast<size_t>(i) * kTerms + E_VDW] = ev;
    d.eatom[static_cast<size_t>(i) * kTerms + E_ELE] = ee;
    const double chi = ff.sb[ti * SB_N + SB_CHI], eta = ff.sb[ti * SB_N + SB_ETA], qd = d.q[i];
    d.eatom[static_cast<size_t>(i) * kTerms + E_POL] = 23.02 * (chi * qd + (eta / 2.) * (qd * qd));
    d.census[4 * d.na + i] = counted;
  }
}

// ------------------------------------------------------------------------------------------------ ACKS2 pair terms
// The pair side of the ACKS2 charge model (src/cpu/acks2.cpp:11-63), FP64, one warp per atom over its full row, with
// the kinetic potentials s_kin of fix acks2/reaxff as input: the polarization coupling 23.02 q_i s_i, and over the
// entries within xcut = (bcut_i + bcut_j)/2 the bond-softness Coulomb E = -23.02/2 bs (s_i - s_j)^2,
// bs = softness d^3 (1 - d)^6, d = r / xcut (softness = gp[34]). The gradient of i takes every entry of its row; the
// energy takes the owner-computes counted entries, as k_nonbonded. Adds to the non-bonded branch's arrays (the same
// stream, after k_nonbonded).
__global__ void k_acks2(Dev d, DevFF ff, const double* s_kin) {
  if (lists_failed(d)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.na) return;
  const int i = warp;
  const SysInfo s = d.sys[d.sys_of[i]];
  const int ti = d.type[i];
  const int cnt = min(d.nbr_cnt[i], d.ncap);
  const double softness = ff.gp[34];
  const double bcut_i = ff.sb[ti * SB_N + SB_BCUT_ACKS2], s_i = s_kin[i];
  const long long tag_i = d.tag[i];
  const int center = (d.S * d.S * d.S - 1) / 2;
  double gx = 0, gy = 0, gz = 0, ee = 0, eh2 = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
  for (int e = lane; e < cnt; e += 32) {
    const unsigned code = d.nbr[static_cast<size_t>(i) * d.ncap + e];
    const int j = static_cast<int>(code & d.amask);
    const int sidx = static_cast<int>(code >> d.abits);
    const double xcut = 0.5 * (bcut_i + ff.sb[d.type[j] * SB_N + SB_BCUT_ACKS2]);
    double dv[3];
    pair_dvec(d, s, i, j, sidx, dv);
    const double dist = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    if (!(dist <= xcut)) continue;
    const double dd = dist / xcut, om = 1.0 - dd, om2 = om * om;
    const double bs = softness * (dd * dd * dd) * (om2 * om2 * om2);
    if (!(bs > 0.0)) continue;
    const double effpot = s_i - s_kin[j];
    double dbs = softness * 3.0 / xcut * (dd * dd) * (om2 * om2 * om) * (1.0 - 3.0 * dd);
    dbs = 23.02 * (-0.5 * dbs * effpot * effpot) / dist;
    gx -= dbs * dv[0]; gy -= dbs * dv[1]; gz -= dbs * dv[2];
    const double c = -0.5 * dbs;
    v0 += c * dv[0] * dv[0]; v1 += c * dv[1] * dv[1]; v2 += c * dv[2] * dv[2];
    v3 += c * dv[0] * dv[1]; v4 += c * dv[0] * dv[2]; v5 += c * dv[1] * dv[2];
    bool count = false;
    if (sidx == center) count = j > i;
    else {
      const long long tag_j = d.tag[j];
      if (tag_i < tag_j) count = true;
      else if (tag_i == tag_j) {
        const double SMALL = 1e-4;
        if (dv[2] > SMALL) count = true;
        else if (fabs(dv[2]) < SMALL) {
          if (dv[1] > SMALL) count = true;
          else if (fabs(dv[1]) < SMALL && dv[0] > SMALL) count = true;
        }
      }
    }
    if (count) ee += -0.5 * 23.02 * bs * effpot * effpot;
    eh2 += 0.5 * (-0.5 * 23.02 * bs * effpot * effpot);
  }
  gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz); ee = warp_sum(ee);
  if (d.pe_on) eh2 = warp_sum(eh2);
  v0 = warp_sum(v0); v1 = warp_sum(v1); v2 = warp_sum(v2); v3 = warp_sum(v3); v4 = warp_sum(v4); v5 = warp_sum(v5);
  if (lane == 0) {
    double4 f = d.fnb[i];
    f.x += gx; f.y += gy; f.z += gz;
    d.fnb[i] = f;
    d.eatom[static_cast<size_t>(i) * kTerms + E_ELE] += ee;
    d.eatom[static_cast<size_t>(i) * kTerms + E_POL] += 23.02 * d.q[i] * s_i;
    if (d.pe_on) pe_add(d, i, eh2 + 23.02 * d.q[i] * s_i);
    double* vi = d.vir_nb + static_cast<size_t>(i) * kVir;
    vi[0] += v0; vi[1] += v1; vi[2] += v2; vi[3] += v3; vi[4] += v4; vi[5] += v5;
  }
}

// ------------------------------------------------------------------------------------------------ QEq CG
// y = (diag(eta) + H) v for one row, both right-hand sides (s, t) at once; warp per row, each lane taking four
// consecutive entries per pass with 16-byte loads (rows start 128-byte aligned: ncap is a multiple of 32); H as
// hi + lo (the FP64 matrix to ~1e-15).
__device__ inline double2 row_mv(const Dev& d, int i, double eta, const double2* v) {
  const int cnt = min(d.nbr_cnt[i], d.ncap);
  const int lane = threadIdx.x & 31;
  const double2 vi = v[i];   // issued before the row so that its latency hides behind it
  double ys = 0.0, yt = 0.0;
  const size_t base = static_cast<size_t>(i) * d.ncap;
  for (int e0 = lane * 4; e0 < cnt; e0 += 128) {
    const uint4 c4 = *reinterpret_cast<const uint4*>(d.nbr + base + e0);
    const float4 h4 = *reinterpret_cast<const float4*>(d.hhi + base + e0);
    const float4 l4 = *reinterpret_cast<const float4*>(d.hlo + base + e0);
    const unsigned cc[4] = {c4.x, c4.y, c4.z, c4.w};
    const float hh[4] = {h4.x, h4.y, h4.z, h4.w}, ll[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (e0 + k < cnt) {
        const double h = static_cast<double>(hh[k]) + static_cast<double>(ll[k]);
        const double2 vj = v[cc[k] & d.amask];
        ys += h * vj.x;
        yt += h * vj.y;
      }
    }
  }
  ys = warp_sum(ys);
  yt = warp_sum(yt);
  return make_double2(eta * vi.x + __shfl_sync(0xffffffffu, ys, 0), eta * vi.y + __shfl_sync(0xffffffffu, yt, 0));
}

// (A v)_i of the single-precision-matrix iterations: FP32 values of the matrix (hhi) times the FP32 copy vf of v,
// products and sums in FP64; the diagonal term takes v_i itself. Gathering 8-byte float2 halves the bytes of the
// gathers (the vector of a 24k-atom system then fits in an SM's L1).
__device__ inline double2 row_mv_f32(const Dev& d, int i, double eta, const double2* v, const float2* vf) {
  const int cnt = min(d.nbr_cnt[i], d.ncap);
  const int lane = threadIdx.x & 31;
  const double2 vi = v[i];
  double ys = 0.0, yt = 0.0;
  const size_t base = static_cast<size_t>(i) * d.ncap;
  for (int e0 = lane * 8; e0 < cnt; e0 += 256) {   // eight entries per lane in flight (rows hold ncap, a multiple of 32)
    const uint4 c4a = *reinterpret_cast<const uint4*>(d.nbr + base + e0);
    const uint4 c4b = *reinterpret_cast<const uint4*>(d.nbr + base + e0 + 4);
    const float4 h4a = *reinterpret_cast<const float4*>(d.hhi + base + e0);
    const float4 h4b = *reinterpret_cast<const float4*>(d.hhi + base + e0 + 4);
    const unsigned cc[8] = {c4a.x, c4a.y, c4a.z, c4a.w, c4b.x, c4b.y, c4b.z, c4b.w};
    const float hh[8] = {h4a.x, h4a.y, h4a.z, h4a.w, h4b.x, h4b.y, h4b.z, h4b.w};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (e0 + k < cnt) {
        const float2 vj = vf[cc[k] & d.amask];
        ys += static_cast<double>(hh[k]) * static_cast<double>(vj.x);
        yt += static_cast<double>(hh[k]) * static_cast<double>(vj.y);
      }
    }
  }
  ys = warp_sum(ys);
  yt = warp_sum(yt);
  return make_double2(eta * vi.x + __shfl_sync(0xffffffffu, ys, 0), eta * vi.y + __shfl_sync(0xffffffffu, yt, 0));
}

// deterministic block sum of NV doubles per thread into out[blockIdx.x * NV + k]
template <int NV>
__device__ inline void block_partials(const double* v, double* out, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid * NV + k] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sh[w * NV + threadIdx.x];
    out[blockIdx.x * NV + threadIdx.x] = t;
  }
  __syncthreads();
}

// Sum of the per-block partials, identical in every block: each thread loads a strided subset in order, then a
// fixed-shape shuffle tree and a fixed-order sum over the warps (the tree depends only on gridDim and blockDim).
template <int NV>
__device__ inline void grid_totals(const double* part, int nblocks, double* tot, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) t += part[b * NV + k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[wid * NV + k] = t;
  }
  __syncthreads();
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sh[w * NV + k];
    tot[k] = t;
  }
  __syncthreads();
}

// Persistent cooperative Jacobi-PCG for one system, s and t solved together: the stock loop of fix qeq/reaxff as
// reproduced in plugin/adapter/fix_qeq_reaxff_metal.cpp:89-123, each right-hand side stopping on its own test
// sqrt(r.M^-1 r)/|b| <= tol with at most imax-1 iterations; then calculate_Q: q = s - (sum s / sum t) t.
// Precision (the resident refinement of src/metal/metal_backend.mm:435-530, in FP64 instead of double-single): the
// iterations multiply the single-precision matrix (hi: 8 bytes per entry with its index) by an FP32 copy of the search
// direction (products and sums in FP64), the vectors and every dot product are FP64, and the residual is recomputed with the FP64 matrix (hi + lo) whenever the iterations have
// converged - or have reduced the residual by kRefineDrop, below which the single-precision matrix stops helping. The
// solve ends only on that FP64 residual, so the tolerance and the reported residuals are those of the FP64 system.
// Rows are distributed over all warps of the grid; reductions are fixed-order (per-block partials summed in block
// order), so the result is bitwise reproducible. Only grid.sync() waits; the kernel is launched cooperatively.
constexpr double kRefineDrop = 1e-6;

__global__ void __launch_bounds__(1024, 1) k_cg_grid(Dev d, CgArgs a) {
  cg::grid_group g = cg::this_grid();
  __shared__ double sh[32 * 4];
  __shared__ double tot_sh[32 * 4];
  const int wpb = blockDim.x >> 5;
  const int gw = blockIdx.x * wpb + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * wpb;
  const int lane = threadIdx.x & 31;
  const int i0 = a.begin, n = a.n;
  double loc[4], tot[4];
  int phase = 0;
  auto partbuf = [&]() { return a.part + static_cast<size_t>(phase & 1) * gridDim.x * 4; };
  double bnorm_s = 0.0, bnorm_t = 0.0, sig_s = 0.0, sig_t = 0.0;
  bool act_s = true, act_t = true, breakdown = false;
  int it_s = 1, it_t = 1, nref = 0;
  for (;;) {
    // ---- FP64 residual: r = b - A x ; p = M^-1 r ; r.p (and |b|^2 on the first pass)
    loc[0] = loc[1] = loc[2] = loc[3] = 0.0;
    for (int r = gw; r < n; r += nwarps) {
      const int i = i0 + r;
      const double eta = a.eta[i];
      const double2 y = row_mv(d, i, eta, a.x);
      if (lane == 0) {
        const double2 b = a.b[i];
        const double2 rr = make_double2(b.x - y.x, b.y - y.y);
        a.r[i] = rr;
        const double2 pp = make_double2(rr.x / eta, rr.y / eta);
        a.p[i] = pp;
        loc[0] += b.x * b.x; loc[1] += b.y * b.y; loc[2] += rr.x * pp.x; loc[3] += rr.y * pp.y;
      }
    }
    block_partials<4>(loc, partbuf(), sh);
    g.sync();
    grid_totals<4>(partbuf(), gridDim.x, tot, tot_sh);
    ++phase;
    ++nref;
    if (nref == 1) { bnorm_s = sqrt(tot[0]); bnorm_t = sqrt(tot[1]); }
    if (act_s) sig_s = tot[2];
    if (act_t) sig_t = tot[3];
    act_s = act_s && (sqrt(sig_s) / bnorm_s > a.tol);
    act_t = act_t && (sqrt(sig_t) / bnorm_t > a.tol);
    if ((!act_s || it_s >= a.imax) && (!act_t || it_t >= a.imax)) break;
    const double stop_s = fmax(a.tol * bnorm_s, kRefineDrop * sqrt(sig_s));
    const double stop_t = fmax(a.tol * bnorm_t, kRefineDrop * sqrt(sig_t));
    // ---- single-precision-matrix iterations from this residual (d = p on entry)
    for (int r = gw * 32 + lane; r < n; r += nwarps * 32) {
      const double2 pp = a.p[i0 + r];
      a.d[i0 + r] = pp;
      a.df[i0 + r] = make_float2(static_cast<float>(pp.x), static_cast<float>(pp.y));
    }
    g.sync();
    for (;;) {
      const bool in_s = act_s && it_s < a.imax && sqrt(sig_s) > stop_s;
      const bool in_t = act_t && it_t < a.imax && sqrt(sig_t) > stop_t;
      if (!in_s && !in_t) break;
      // q = A d ; partial d.q
      loc[0] = loc[1] = 0.0;
      for (int r = gw; r < n; r += nwarps) {
        const int i = i0 + r;
        const double2 y = row_mv_f32(d, i, a.eta[i], a.d, a.df);
        if (lane == 0) {
          a.q[i] = y;
          const double2 dd = a.d[i];
          loc[0] += dd.x * y.x; loc[1] += dd.y * y.y;
        }
      }
      block_partials<2>(loc, partbuf(), sh);
      g.sync();
      grid_totals<2>(partbuf(), gridDim.x, tot, tot_sh);
      ++phase;
      const double alpha_s = in_s ? sig_s / tot[0] : 0.0;
      const double alpha_t = in_t ? sig_t / tot[1] : 0.0;
      if (!(isfinite(alpha_s) && isfinite(alpha_t))) { breakdown = true; break; }
      // x += alpha d ; r -= alpha q ; p = M^-1 r ; partial r.p
      loc[0] = loc[1] = 0.0;
      for (int r = gw * 32 + lane; r < n; r += nwarps * 32) {
        const int i = i0 + r;
        const double2 dd = a.d[i], qq = a.q[i];
        double2 xx = a.x[i], rr = a.r[i];
        xx.x += alpha_s * dd.x; xx.y += alpha_t * dd.y;
        rr.x -= alpha_s * qq.x; rr.y -= alpha_t * qq.y;
        a.x[i] = xx;
        a.r[i] = rr;
        const double eta = a.eta[i];
        const double2 pp = make_double2(rr.x / eta, rr.y / eta);
        a.p[i] = pp;
        loc[0] += rr.x * pp.x; loc[1] += rr.y * pp.y;
      }
      block_partials<2>(loc, partbuf(), sh);
      g.sync();
      grid_totals<2>(partbuf(), gridDim.x, tot, tot_sh);
      ++phase;
      const double beta_s = in_s ? tot[0] / sig_s : 0.0;
      const double beta_t = in_t ? tot[1] / sig_t : 0.0;
      if (in_s) { sig_s = tot[0]; ++it_s; }
      if (in_t) { sig_t = tot[1]; ++it_t; }
      // d = p + beta d (only for the right-hand sides still iterating)
      for (int r = gw * 32 + lane; r < n; r += nwarps * 32) {
        const int i = i0 + r;
        const double2 pp = a.p[i];
        double2 dd = a.d[i];
        if (in_s) dd.x = pp.x + beta_s * dd.x;
        if (in_t) dd.y = pp.y + beta_t * dd.y;
        a.d[i] = dd;
        a.df[i] = make_float2(static_cast<float>(dd.x), static_cast<float>(dd.y));
      }
      g.sync();
    }
    if (breakdown) break;
  }
  // calculate_Q: q = s - (sum s / sum t) t
  loc[0] = loc[1] = 0.0;
  for (int r = gw * 32 + lane; r < n; r += nwarps * 32) {
    const double2 xx = a.x[i0 + r];
    loc[0] += xx.x; loc[1] += xx.y;
  }
  block_partials<2>(loc, partbuf(), sh);
  g.sync();
  grid_totals<2>(partbuf(), gridDim.x, tot, tot_sh);
  ++phase;
  const double u = tot[0] / tot[1];
  if (a.write_q)
    for (int r = gw * 32 + lane; r < n; r += nwarps * 32) {
      const double2 xx = a.x[i0 + r];
      d.q[i0 + r] = xx.x - u * xx.y;
    }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.out_brk) a.out_brk[0] = breakdown ? 1 : 0;
    a.out_iters[0] = it_s;
    a.out_iters[1] = it_t;
    a.out_rel[0] = sqrt(sig_s) / bnorm_s;
    a.out_rel[1] = sqrt(sig_t) / bnorm_t;
    if (a.out_nref) a.out_nref[0] = nref;
    if (breakdown) atomicOr(d.status, ST_CG_BREAKDOWN);
    if (!(a.out_rel[0] <= a.tol && a.out_rel[1] <= a.tol)) atomicOr(d.status, ST_CG_NOTCONV);
  }
}

// Segmented Jacobi-PCG: every system of the batch at once on one cooperative grid, the same algorithm (and the same
// stopping rule per system, s and t separately) as the stock loop of fix qeq/reaxff (fix_qeq_reaxff_metal.cpp:89-123).
// Rows of all systems are spread over all warps of the GPU, so one small system no longer runs on a single block.
// Every dot product is a per-row term written to rb0/rb1; the warp that brings the last row of a system to a pass
// sums that system's terms in row order (lane-strided, then a butterfly), so a system's result depends only on its
// own rows: it is bitwise the same alone and inside any batch. The iteration loop ends when no system is live; the
// live count is kept per iteration parity so that no block can see it change before every block has read it.
__device__ inline double2 sys_sum2(const double2* v, int i0, int n) {
  const int lane = threadIdx.x & 31;
  double sx = 0.0, sy = 0.0;
#pragma unroll 4
  for (int k = lane; k < n; k += 32) {
    const double2 t = __ldcg(v + i0 + k);
    sx += t.x;
    sy += t.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  return make_double2(sx, sy);
}

// lane 0 counts cnt rows of the system in (after every lane's writes are fenced); true in every lane of the warp that
// brought the system's last rows
__device__ inline bool arrive_last(SysCg* sc, int n, int cnt) {
  __threadfence();
  __syncwarp();
  bool last = false;
  if ((threadIdx.x & 31) == 0) last = atomicAdd(&sc->counter, static_cast<unsigned>(cnt)) == static_cast<unsigned>(n - cnt);
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) __threadfence();
  return last;
}

__global__ void __launch_bounds__(256, 4) k_cg_seg(Dev d, CgArgs a) {
  if (lists_failed(d)) return;
  cg::grid_group g = cg::this_grid();
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int nw = gridDim.x * (blockDim.x >> 5);
  const int na = d.na;
  const double tol = a.tol;
  // matrix passes: warp per row, rows dealt round-robin over all warps (a system that is still iterating when most
  // have stopped keeps many warps busy); a warp counts its rows of one system in when it meets a different system
  // ---- r = b - A x, d = M^-1 r; |b|^2 and r.d per system; first stop test
  {
    int cur = -1, cnt = 0;
    auto finish = [&](int s, int c) {
      const SysInfo& si = d.sys[s];
      if (!arrive_last(a.sc + s, si.natoms, c)) return;
      const double2 bb = sys_sum2(a.rb0, si.begin, si.natoms);
      const double2 rd = sys_sum2(a.rb1, si.begin, si.natoms);
      if (lane == 0) {
        SysCg& c2 = a.sc[s];
        c2.counter = 0;
        c2.bnorm_s = sqrt(bb.x);
        c2.bnorm_t = sqrt(bb.y);
        c2.sig_s = rd.x;
        c2.sig_t = rd.y;
        c2.it_s = c2.it_t = 1;
        c2.breakdown = 0;
        c2.act_s = sqrt(c2.sig_s) / c2.bnorm_s > tol;
        c2.act_t = sqrt(c2.sig_t) / c2.bnorm_t > tol;
        c2.live = (c2.act_s || c2.act_t) && a.imax > 1;
        if (c2.live) atomicAdd(a.nlive + 1, 1);
      }
    };
    for (int i = gw; i < na; i += nw) {
      const int s = d.sys_of[i];
      if (s != cur) {
        if (cnt > 0) finish(cur, cnt);
        cur = s;
        cnt = 0;
      }
      const double eta = a.eta[i];
      const double2 y = row_mv(d, i, eta, a.x);
      if (lane == 0) {
        const double2 b = a.b[i];
        const double2 rr = make_double2(b.x - y.x, b.y - y.y);
        a.r[i] = rr;
        const double2 dd = make_double2(rr.x / eta, rr.y / eta);
        a.d[i] = dd;
        a.rb0[i] = make_double2(b.x * b.x, b.y * b.y);
        a.rb1[i] = make_double2(rr.x * dd.x, rr.y * dd.y);
      }
      ++cnt;
    }
    if (cnt > 0) finish(cur, cnt);
  }
  g.sync();
  for (int it = 1; it < a.imax; ++it) {
    if (__ldcg(a.nlive + (it & 1)) == 0) break;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.nlive[(it + 1) & 1] = 0;
    // ---- q = A d, d.q; alpha (or a breakdown, which ends this system)
    {
      int cur = -1, cnt = 0;
      bool live = false;
      auto finish = [&](int s, int c) {
        const SysInfo& si = d.sys[s];
        if (!arrive_last(a.sc + s, si.natoms, c)) return;
        const double2 dq = sys_sum2(a.rb0, si.begin, si.natoms);
        if (lane == 0) {
          SysCg& c2 = a.sc[s];
          c2.counter = 0;
          c2.alpha_s = c2.act_s ? c2.sig_s / dq.x : 0.0;
          c2.alpha_t = c2.act_t ? c2.sig_t / dq.y : 0.0;
          if (!(isfinite(c2.alpha_s) && isfinite(c2.alpha_t))) {
            c2.breakdown = 1;
            c2.live = 0;
          }
        }
      };
      for (int i = gw; i < na; i += nw) {
        const int s = d.sys_of[i];
        if (s != cur) {
          if (cnt > 0) finish(cur, cnt);
          cur = s;
          cnt = 0;
          live = __ldcg(&a.sc[s].live) != 0;
        }
        if (!live) continue;
        const double2 y = row_mv(d, i, a.eta[i], a.d);
        if (lane == 0) {
          a.q[i] = y;
          const double2 dd = a.d[i];
          a.rb0[i] = make_double2(dd.x * y.x, dd.y * y.y);
        }
        ++cnt;
      }
      if (cnt > 0) finish(cur, cnt);
    }
    g.sync();
    // ---- x += alpha d, r -= alpha q, p = M^-1 r, r.p; beta, the counts and the next stop test
    for (int i0 = gw * 32; i0 < na; i0 += nw * 32) {
      const int i = i0 + lane;
      int s = -1;
      bool on = false;
      if (i < na) {
        s = d.sys_of[i];
        on = __ldcg(&a.sc[s].live) != 0;
      }
      if (on) {
        const double alpha_s = __ldcg(&a.sc[s].alpha_s), alpha_t = __ldcg(&a.sc[s].alpha_t);
        const double2 dd = a.d[i], qq = a.q[i];
        double2 xx = a.x[i], rr = a.r[i];
        xx.x += alpha_s * dd.x; xx.y += alpha_t * dd.y;
        rr.x -= alpha_s * qq.x; rr.y -= alpha_t * qq.y;
        a.x[i] = xx;
        a.r[i] = rr;
        const double eta = a.eta[i];
        const double2 pp = make_double2(rr.x / eta, rr.y / eta);
        a.p[i] = pp;
        a.rb0[i] = make_double2(rr.x * pp.x, rr.y * pp.y);
      }
      __threadfence();
      __syncwarp();
      // one arrival per system present in this warp's 32 rows, by the lowest lane of that system
      const unsigned on_mask = __ballot_sync(0xffffffffu, on);
      const unsigned same = __match_any_sync(0xffffffffu, s) & on_mask;
      bool last = false;
      if (on && (__ffs(same) - 1) == lane) {
        const unsigned c = __popc(same);
        last = atomicAdd(&a.sc[s].counter, c) == static_cast<unsigned>(d.sys[s].natoms) - c;
      }
      unsigned m = __ballot_sync(0xffffffffu, last);
      if (m) __threadfence();
      while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1;
        const int ss = __shfl_sync(0xffffffffu, s, l);
        const SysInfo& si = d.sys[ss];
        const double2 rp = sys_sum2(a.rb0, si.begin, si.natoms);
        if (lane == 0) {
          SysCg& c = a.sc[ss];
          c.counter = 0;
          c.beta_s = c.act_s ? rp.x / c.sig_s : 0.0;
          c.beta_t = c.act_t ? rp.y / c.sig_t : 0.0;
          if (c.act_s) { c.sig_s = rp.x; c.it_s = it + 1; }
          if (c.act_t) { c.sig_t = rp.y; c.it_t = it + 1; }
          // the stop test of the next iteration; d below is updated only for the right-hand sides still active
          c.act_s = c.act_s && (sqrt(c.sig_s) / c.bnorm_s > tol);
          c.act_t = c.act_t && (sqrt(c.sig_t) / c.bnorm_t > tol);
          c.live = (c.act_s || c.act_t) && it + 1 < a.imax;
          if (c.live) atomicAdd(a.nlive + ((it + 1) & 1), 1);
        }
      }
    }
    g.sync();
    // ---- d = p + beta d
    for (int i = gw * 32 + lane; i < na; i += nw * 32) {
      const int s = d.sys_of[i];
      if (!__ldcg(&a.sc[s].live)) continue;
      const double beta_s = __ldcg(&a.sc[s].beta_s), beta_t = __ldcg(&a.sc[s].beta_t);
      const int act_s = __ldcg(&a.sc[s].act_s), act_t = __ldcg(&a.sc[s].act_t);
      const double2 pp = a.p[i];
      double2 dd = a.d[i];
      if (act_s) dd.x = pp.x + beta_s * dd.x;
      if (act_t) dd.y = pp.y + beta_t * dd.y;
      a.d[i] = dd;
    }
    g.sync();
  }
// ---- calculate_Q per system (warp per system): q = s - (sum s / sum t) t, the counts and residuals
  for (int s = gw; s < d.nsys; s += nw) {
    const SysInfo& si = d.sys[s];
    const double2 sum = sys_sum2(a.x, si.begin, si.natoms);
    const double u = sum.x / sum.y;
    if (a.write_q)
      for (int k = lane; k < si.natoms; k += 32) {
        const double2 xx = a.x[si.begin + k];
        d.q[si.begin + k] = xx.x - u * xx.y;
      }
    if (lane == 0) {
      const SysCg& c = a.sc[s];
      if (a.out_brk) a.out_brk[s] = c.breakdown;
      a.out_iters[2 * s] = c.it_s;
      a.out_iters[2 * s + 1] = c.it_t;
      a.out_rel[2 * s] = sqrt(c.sig_s) / c.bnorm_s;
      a.out_rel[2 * s + 1] = sqrt(c.sig_t) / c.bnorm_t;
      if (c.breakdown) atomicOr(d.status, ST_CG_BREAKDOWN);
      if (!(a.out_rel[2 * s] <= tol && a.out_rel[2 * s + 1] <= tol)) atomicOr(d.status, ST_CG_NOTCONV);
    }
  }
}


// Initial guesses from the histories (Q-23: s = 4(s0+s2) - (6 s1 + s3), t = t2 + 3(t0 - t1); index 0 = latest),
// right-hand sides b_s = -chi, b_t = -1, and the diagonal eta.
__global__ void k_qeq_prepare(Dev d, DevFF ff, CgArgs a, const double* s_hist, const double* t_hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.na) return;
  const int t = d.type[i];
  const double* sh = s_hist + 4 * static_cast<size_t>(i);
  const double* th = t_hist + 4 * static_cast<size_t>(i);
  a.x[i] = make_double2(4 * (sh[0] + sh[2]) - (6 * sh[1] + sh[3]), th[2] + 3 * (th[0] - th[1]));
  a.b[i] = make_double2(-ff.sb[t * SB_N + SB_CHI], -1.0);
  a.eta[i] = ff.sb[t * SB_N + SB_ETA];
}

// A solve of given right-hand sides from given guesses (mtl::Context::qeq_solve, metal_backend.hpp:84-86): b and x0
// hold the s system for every atom, then the t system.
__global__ void k_qeq_prepare_given(Dev d, DevFF ff, CgArgs a, const double* b, const double* x0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.na) return;
  a.x[i] = x0 ? make_double2(x0[i], x0[d.na + i]) : make_double2(0.0, 0.0);
  a.b[i] = make_double2(b[i], b[d.na + i]);
  a.eta[i] = ff.sb[d.type[i] * SB_N + SB_ETA];
}

// the solve just finished becomes the newest history entry; not after a list overflow (the evaluation is repeated),
// nor after a failed solve (a breakdown, or a system above its tolerance in strict mode): the call then reports an
// error and leaves the histories as they were
__global__ void k_qeq_history(Dev d, const double2* x, double* s_hist, double* t_hist, int strict) {
  if (lists_failed(d)) return;
  const int st = *reinterpret_cast<volatile const int*>(d.status);
  if ((st & ST_CG_BREAKDOWN) || (strict && (st & ST_CG_NOTCONV))) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.na) return;
  double* sh = s_hist + 4 * static_cast<size_t>(i);
  double* th = t_hist + 4 * static_cast<size_t>(i);
  for (int k = 3; k > 0; --k) { sh[k] = sh[k - 1]; th[k] = th[k - 1]; }
  sh[0] = x[i].x;
  th[0] = x[i].y;
}

// y = (diag(eta) + H) v, owned rows (mtl::Context::qeq_matvec)
__global__ void k_qeq_matvec(Dev d, DevFF ff, const double2* v, double2* y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= d.na) return;
  const double eta = ff.sb[d.type[warp] * SB_N + SB_ETA];
  const double2 r = row_mv(d, warp, eta, v);
  if ((threadIdx.x & 31) == 0) y[warp] = r;
}

// ------------------------------------------------------------------------------------------------ energy sums
// Per system: fixed-order sums of the 13 energy terms and the 6 virial components over the system's atoms, in two
// passes. k_energy_part: one block per (system, 256-atom chunk), a thread per atom, each of the 19 quantities summed by
// a fixed shuffle tree per warp and then over the warps in order; k_energy_final: per system, a warp per quantity over
// the chunk partials (lane-strided, then a fixed shuffle tree). Chunks start at the system's first atom, so a system's sums are the same alone or in a
// batch.
constexpr int kESum = kTerms + kVir;
__global__ void __launch_bounds__(256) k_energy_part(Dev d, double* part, int nchunk) {
  const int sidx = blockIdx.x, c = blockIdx.y;   // systems along x: any number of them
  const SysInfo& s = d.sys[sidx];
  if (c * 256 >= s.natoms) return;
  __shared__ double sh[8][kESum];
  const int r = c * 256 + threadIdx.x;
  double v[kESum];
  if (r < s.natoms) {
    const size_t a = static_cast<size_t>(s.begin + r);
#pragma unroll
    for (int t = 0; t < kTerms; ++t) v[t] = d.eatom[a * kTerms + t];
#pragma unroll
    for (int k = 0; k < kVir; ++k) {
      const size_t q = a * kVir + k;
      v[kTerms + k] = ((d.vir[q] + d.vir_h[q]) + d.vir_t[q]) + d.vir_nb[q];
    }
  } else {
#pragma unroll
    for (int t = 0; t < kESum; ++t) v[t] = 0.0;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < kESum; ++t) {
    double x = v[t];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[w][t] = x;
  }
  __syncthreads();
  if (threadIdx.x < kESum) {
    double x = 0.0;
    for (int k = 0; k < 8; ++k) x += sh[k][threadIdx.x];
    part[(static_cast<size_t>(sidx) * nchunk + c) * kESum + threadIdx.x] = x;
  }
}

__global__ void k_energy_final(Dev d, const double* part, int nchunk, double* out, double* out_vir) {
  const int sidx = blockIdx.x, t = threadIdx.x >> 5, lane = threadIdx.x & 31;   // a warp per quantity
  if (t >= kESum) return;
  const int nc = (d.sys[sidx].natoms + 255) / 256;
  double x = 0.0;
  for (int c = lane; c < nc; c += 32) x += part[(static_cast<size_t>(sidx) * nchunk + c) * kESum + t];
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if (lane == 0) {
    if (t < kTerms) out[sidx * kTerms + t] = x;
    else out_vir[sidx * kVir + (t - kTerms)] = x;
  }
}

}  // namespace rx
