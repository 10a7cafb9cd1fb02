// Device-side data layout of the B200 ReaxFF engine.
//
// Periodic images are never materialised as ghost atoms. Every neighbor and bond entry of an owned atom names its
// partner as (owner atom index, lattice shift), packed into one 32-bit code: the low `abits` bits hold the atom index,
// the high bits the shift index sidx = ((sx+smax)*S + (sy+smax))*S + (sz+smax), S = 2*smax+1. The reverse entry of
// (i -> j, s) is (j -> i, -s), whose shift index is S^3-1-sidx. Results equal those of the reference's ghost-native
// traversal (src/neighbor/neighbor.cpp:18-88 expands images, src/cpu/bonded.cpp runs over them) wherever its ghost
// shell is complete, which its shell rule guarantees for owned atoms.
//
// Per-atom bond slots: atom a owns slots [a*bcap, a*bcap + bcnt[a]); every slot knows the global index of its reverse
// slot (bsym). All cross-atom contributions (forces on bond partners, CdDelta of partners, torsion contributions to
// second neighbors) are written into slots owned by the writing atom and gathered by the receiving atom in a fixed
// order: no atomics, bitwise reproducible.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rx {

constexpr int kTerms = 13;   // bond, over, under, lone_pair, valence, penalty, coalition, hbond, torsion, conjugation, vdw, coulomb, polarization
constexpr int kCensus = 7;   // bonds, angle_sets, torsions, hbonds, nonbonded, sbo_region, lp_trunc
constexpr int kVir = 6;      // virial components in LAMMPS's order: xx, yy, zz, xy, xz, yz (sum of x_a f_b)
enum Term { E_BOND, E_OV, E_UN, E_LP, E_ANG, E_PEN, E_COA, E_HB, E_TOR, E_CON, E_VDW, E_ELE, E_POL };

// status bits written by kernels (read by the host after a launch sequence)
enum Status : int {
  ST_NBR_OVERFLOW = 1,
  ST_BOND_OVERFLOW = 2,
  ST_SYM_MISSING = 4,
  ST_SHIFT_RANGE = 8,
  ST_CG_BREAKDOWN = 16,
  ST_NONFINITE = 32,
  ST_NEAR_OVERFLOW = 64,
  ST_CG_NOTCONV = 128,   // a system's charge solve ended above its tolerance (iteration limit)
  ST_VERLET_OVERFLOW = 256,
  ST_NONPERIODIC_ESCAPE = 512,   // an atom left the padded extent of a non-periodic direction
  ST_ACC_OVERFLOW = 1024,
};
// status words: [0] bits, [1] max neighbor-row count, [2] max bond count, [3] max near-row count, [4] max Verlet-row
// count, [5] max acceptor-row count
constexpr int kStatusWords = 8;

struct SysInfo {
  double origin[3];
  double L[9];    // lattice vectors a, b, c as rows
  double R[9];    // rows of the inverse transform: f_d = R[d] . (r - origin)
  int begin, natoms;
  int nc[3];      // cells per lattice direction
  int cell_begin;
  int range[3];   // cell search range per direction
  int shift_base; // first entry of this system's lattice-shift table (S^3 entries)
  double h[3];    // distances between opposite faces (heights) along each lattice direction
  int ortho;      // lattice vectors mutually orthogonal
  int per[3];     // periodic directions; along the others the lattice vector is the engine's own padded extent
  double ext;     // |a| + |b| + |c|: bounds every coordinate of a wrapped position relative to origin
  double inv_nc[3], inv_h[3];
  float inv_ncf0;
  // single-precision r^2 thresholds of the Verlet, bond-candidate and acceptor rows (see layout_systems)
  float vthr[3];
};

struct DevFF {
  int nt, vdw_type, lg;
  double bo_cut, nonb_low, nonb_cut;
  const double* gp;
  const double* sb;
  const double* tb;
  const int* thb_n;
  const double* thb;
  const int* fb_on;
  const double* fb;
  const int* hb_on;
  const double* hb;
  const double* shld;    // nt x nt: (gamma_i gamma_j)^-1.5, the charge-matrix shielding
  const double* rbo2;    // nt x nt: squared bond-order reach (no bond beyond it; HUGE_VAL where it cannot be bounded)
  const float* nbf;      // nt x nt x 12: single-precision pair parameters of the non-bonded kernel
  double tap[8];   // taper coefficients on [nonb_low, nonb_cut] (include/reaxmetal/terms_host.hpp:16-29)
};

struct DevCtl {
  double bond_cut, hbond_cut, thb_cut, thb_cutsq;
  int enobonds;
};

struct AtomQ {   // atom_quantities (include/reaxmetal/terms.hpp:141-164) plus the corrected total bond order
  double total_bo, Delta, Delta_e, Delta_boc, Delta_val, vlpex, nlp, Delta_lp, dDelta_lp, Delta_lp_temp;
};

struct Dev {
  int na, nsys;
  const SysInfo* sys;
  const int* sys_of;
  double4* x;            // positions (w unused)
  const int* type;
  const long long* tag;
  double* q;             // charges
  // cells
  int* cell_key;         // global cell of every atom (sort key)
  int* cell_atoms;       // atoms sorted by cell
  float4* xs;            // positions in cell order relative to their system's origin, single precision (w = type)
  int* cell_start;       // ncell_total + 1
  int ncell_total;
  // Verlet rows: every image within nonb_cut + skin at the last rebuild of the atom's system (rebuilt when an atom of
  // the system has moved more than skin/2 since: k_nbr_check sets the system's flag)
  int vcap;
  unsigned* vrow;
  int* vcnt;
  double4* xref;         // positions at the last rebuild
  int* sys_flag;         // per system: rebuild in this evaluation
  double rv2;            // (nonb_cut + skin)^2
  double half_skin2;     // (skin / 2)^2
  // neighbor rows (full: both directions, every image within nonb_cut), filtered from the Verlet rows every step
  int ncap;
  unsigned* nbr;
  int* nbr_cnt;
  float* hhi;            // charge-matrix entry of every neighbor entry (0 beyond swb) as hi + lo single-precision
  float* hlo;            // parts: hi = (float)H, lo = (float)(H - hi), H = hi + lo to ~1e-15 relative
  int abits;
  unsigned amask;
  int smax, S;
  const double4* shifts; // per system and shift index: L.s (xyz), summed as the reference sums lattice shifts
  // near rows: the entries of the full row within max(bond_cut, hbond_cut), in the same order
  int ncap_near;         // bond-candidate rows: entries within bond_cut (k_bonds)
  unsigned* near;
  int* near_cnt;
  double rnear2;
  int ncap_acc;          // acceptor rows of the H-bond hydrogens (p_hbond = 1): p_hbond = 2 atoms within hbond_cut
  unsigned* acc;
  int* acc_cnt;
  double racc2;
  // bonds
  int bcap;
  unsigned* bcode;
  int* bsym;
  int* bcnt;
  double4* bdv;          // x_partner - x_self (xyz), distance (w)
  double4* bBO;          // BO, BO_s, BO_pi, BO_pi2 (uncorrected minus bo_cut, then corrected in place)
  double4* bdBOp;        // dBOp (xyz)
  double4* bdlnpi;       // dln_BOp_pi (xyz)
  double4* bdlnpi2;      // dln_BOp_pi2 (xyz)
  double4* bC0;          // C1dbo, C2dbo, C3dbo, C1dbopi
  double4* bC1;          // C2dbopi, C3dbopi, C4dbopi, C1dbopi2
  double4* bC2;          // C2dbopi2, C3dbopi2, C4dbopi2, -
  double4* bacc;         // Cdbo, Cdbopi, Cdbopi2, CdDelta contribution to the partner (k_bonded_atom)
  double4* bfn;          // gradient contribution to the partner (xyz) (k_bonded_atom)
  // the H-bond and torsion kernels run concurrently with k_bonded_atom, so each keeps its own per-slot and per-atom
  // contributions; the gathers add them in fixed order
  double* bcdbo_h;       // H-bond: Cdbo of the donor bond
  double4* bfn_h;        // H-bond: gradient on the donor (xyz)
  double4* bacc_t;       // torsion: Cdbo, Cdbopi, -, CdDelta to the partner
  double4* bfn_t;        // torsion: gradient on the partner (xyz)
  double4* Tl;           // torsion: per (central slot, position in the far atom's slots): gradient xyz, Cdbo (w)
  double4* Ti;           // torsion: per (central slot, position in the central atom's slots): gradient on i, Cdbo of i-j
  unsigned char* tflag;  // per slot: 1 if it is a listed central bond of the torsions (its torsion rows are written)
  int* tor_list;         // the listed central-bond slots, in arrival order, and their count
  int* tor_n;
  double4* Tsum;         // torsion: per central slot, 2 entries: central gradient + CdDelta; e_tor, e_con, count
  double* Tvir;          // torsion: per central slot, kVir virial components
  // atoms
  double* Deltap;
  double* Deltap_boc;
  double4* dDp_self;
  AtomQ* aq;
  double4* fown;         // gradient on the atom itself (xyz), own CdDelta (w) (k_bonded_atom)
  double4* fown_h;       // H-bond: gradient on the hydrogen itself
  unsigned long long* fix_h;   // scattered gradient shares (H-bond acceptors, non-bonded partners), 3 per atom, fixed point (2^32 units)
  double4* fown_t;       // torsion: gradient on the central atom (xyz), own CdDelta (w)
  double* cdtot;
  double* W;
  double4* fdb;
  double4* fnb;          // non-bonded gradient
  double4* grad;         // result
  double* eatom;         // kTerms per atom
  unsigned long long* pe_fix;   // per-atom energy tallies (fixed point, 2^32 units), written when pe_on
  int pe_on;
  double* vir;           // kVir per atom: virial of the bonded interactions this atom centres (LAMMPS order xx yy zz xy xz yz)
  double* vir_h;         // kVir per atom: H-bond triples centred on this hydrogen
  double* vir_t;         // kVir per atom: torsions centred on this atom
  double* vir_nb;        // kVir per atom: half the virial of the atom's non-bonded pairs
  int* census;           // kCensus per atom (atom-major: census[c*na + a])
  int* status;
  long long* counters;   // [0] neighbor entries, [1] counted pairs, [2] bonds (directed), [3] H-bond triples
};

// ----------------------------------------------------------------------------------------------- helpers
__host__ __device__ inline int floor_div(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

__device__ inline void decode_shift(int sidx, int S, int smax, int& sx, int& sy, int& sz) {
  sz = sidx % S - smax;
  sy = (sidx / S) % S - smax;
  sx = sidx / (S * S) - smax;
}

// Canonical separation vector of the entry (i -> j at shift s): computed from the lower-index end (for i == j from the
// positive shift) and negated for the other direction, so both directions of a pair see bitwise-negated vectors and
// identical distances; every cut-off decision is therefore symmetric. The lattice shifts come from a per-system
// table built on the host (the same double-precision sum the reference uses, src/core/system.cpp:52-57).
__device__ inline void pair_dvec_x(const Dev& d, const SysInfo& s, int i, int j, int sidx, const double4& xi, const double4& xj,
                                   double* dv) {
  // forward: (x_j + L s) - x_i; backward: -((x_i + L(-s)) - x_j). Written with selects instead of a branch, so that the
  // lanes of a warp that take different directions do not serialise; the negation is exact, the bits are the same.
  const int S3 = d.S * d.S * d.S;
  const bool fwd = (j > i) || (j == i && 2 * sidx > S3 - 1);
  const double4 sh = d.shifts[s.shift_base + (fwd ? sidx : S3 - 1 - sidx)];
  const double4 xa = fwd ? xj : xi, xb = fwd ? xi : xj;
  const double sg = fwd ? 1.0 : -1.0;
  dv[0] = sg * ((xa.x + sh.x) - xb.x);
  dv[1] = sg * ((xa.y + sh.y) - xb.y);
  dv[2] = sg * ((xa.z + sh.z) - xb.z);
}
__device__ inline void pair_dvec(const Dev& d, const SysInfo& s, int i, int j, int sidx, double* dv) {
  pair_dvec_x(d, s, i, j, sidx, d.x[i], d.x[j], dv);
}

// A list of this evaluation overflowed (the host grows it and repeats the evaluation): later kernels skip their work.
__device__ inline bool lists_failed(const Dev& d) {
  return (*reinterpret_cast<volatile const int*>(d.status) &
          (ST_NBR_OVERFLOW | ST_NEAR_OVERFLOW | ST_BOND_OVERFLOW | ST_SHIFT_RANGE | ST_VERLET_OVERFLOW | ST_ACC_OVERFLOW)) != 0;
}

// Virial of an interaction cluster, sum over its atoms of x_a f_b = -x_a g_b, taken with positions P relative to the
// cluster's own atom (every term is translation invariant, so its gradients sum to zero and the origin drops out).
// Accumulates -P (x) g into v[6] in LAMMPS's component order (virial_fdotr_compute: xx, yy, zz, xy, xz, yz).
template <class T, class U>
__device__ inline void vir_add(double* v, const T* P, const U* g, double scale = 1.0) {
  const double p0 = P[0], p1 = P[1], p2 = P[2], g0 = g[0] * scale, g1 = g[1] * scale, g2 = g[2] * scale;
  v[0] -= p0 * g0; v[1] -= p1 * g1; v[2] -= p2 * g2; v[3] -= p0 * g1; v[4] -= p0 * g2; v[5] -= p1 * g2;
}

// Fixed-point accumulation (2^32 units): integer additions commute, so contributions added with atomics in any order
// give the same bits every run (deterministic scatters to other atoms).
constexpr double kFixScale = 4294967296.0;
__device__ inline void fix_add(unsigned long long* acc, double v) {
  atomicAdd(acc, static_cast<unsigned long long>(__double2ll_rn(v * kFixScale)));
}
__device__ inline double fix_value(unsigned long long v) { return static_cast<double>(static_cast<long long>(v)) * (1.0 / kFixScale); }
// per-atom energy tally (the reference's eatom rules), when requested
__device__ inline void pe_add(const Dev& d, int a, double e) {
  if (d.pe_on && e != 0.0) fix_add(d.pe_fix + a, e);
}

__device__ inline double safe_exp(double v) { return exp(v > 700.0 ? 700.0 : v); }
__device__ inline float safe_expf(float v) { return __expf(v > 40.f ? 40.f : v); }

__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warp_sumf(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace rx
