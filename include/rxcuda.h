/* rxcuda: C ABI of the B200 ReaxFF force + charge-equilibration engine (librxcuda.so).
 *
 * This is the boundary the reference's LAMMPS adapter binds for its GPU path. Each entry point names the reference
 * interface it replaces (file:line in the reference tree):
 *   - the device context  reaxmetal::mtl::Context          include/reaxmetal/metal_backend.hpp:57-95
 *   - the force-field reader  parse_force_field           src/io/ffield_parser.cpp:91, include/reaxmetal/forcefield.hpp:134
 *   - the pair style's compute  PairReaxFFMetal::compute  plugin/adapter/pair_reaxff_metal.cpp:412-524
 *   - the charge fix  FixQEqReaxFFMetal::{compute_H, CG, sparse_matvec, calculate_Q}
 *                                                          plugin/adapter/fix_qeq_reaxff_metal.cpp:65-205
 *
 * Conventions (as the reference's Context): the caller owns every host array; the context copies inputs into
 * persistent device buffers and copies results back; one context per host thread; every call is synchronous with
 * respect to the host arrays it takes. Errors never cross the ABI as exceptions: every call returns an RX_* status
 * and rx_last_error() holds the message. Units are LAMMPS `real`: Angstrom, kcal/mol, e, fs, g/mol.
 *
 * A context holds one or more independent periodic systems ("batch"); atoms of system s occupy the index range
 * [offset_s, offset_s + natoms_s) of every per-atom array, in system order.
 */
#ifndef RXCUDA_H
#define RXCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RX_OK 0
#define RX_ERR_INVALID 1        /* invalid argument or input (SystemError / FfieldError in the reference) */
#define RX_ERR_FFIELD 2         /* force-field text rejected by the strict reader */
#define RX_ERR_CAPACITY 3       /* a per-atom list overflowed after the grow-and-retry budget (neighbor.cpp:362-374) */
#define RX_ERR_CUDA 4           /* CUDA runtime error or no device */
#define RX_ERR_NOT_CONVERGED 5  /* charge equilibration hit its iteration limit in strict mode (fix_qeq_reaxff_metal.cpp:79-80) */
#define RX_ERR_STATE 6          /* entry point called before what it needs (force field, systems) */
#define RX_ERR_TIMEOUT 7        /* a device wait exceeded its bound */

/* rx_compute flags */
#define RX_COMPUTE_QEQ 1        /* solve the charges (fix qeq/reaxff/metal resident) before the force evaluation */
#define RX_COMPUTE_CENSUS 2     /* fill the decision census (include/reaxmetal/census.hpp:12-20) */
#define RX_COMPUTE_QEQ_COLD 4     /* with RX_COMPUTE_QEQ: start the CG from s = t = 0 instead of the history extrapolation
                                     (a fresh single point; the history is then restarted from this solve) */
#define RX_COMPUTE_PERATOM 8      /* tally per-atom energies and virials (compute pe/atom, stress/atom): rx_get_peratom */

typedef struct rx_context rx_context;

/* mtl::Context construction (metal_backend.hpp:57-60). device: CUDA ordinal, or -1 for a host-only context that reads
 * and inspects force fields only (every device entry point then returns RX_ERR_STATE). NULL on failure (no device). */
rx_context* rx_create(int device);
void rx_destroy(rx_context* ctx);
/* message of the last failed call on this context ("" if none); also valid for ctx == NULL (creation errors) */
const char* rx_last_error(const rx_context* ctx);

/* parse_force_field (src/io/ffield_parser.cpp:91-451): strict reader; lgvdw = 1 for `pair_style reaxff lgvdw yes`. */
int rx_set_forcefield(rx_context* ctx, const char* ffield_text, int lgvdw);
/* canonical_table_dump (src/io/table_dump.cpp:20-84) of the parsed tables. Returns the length (without NUL) and
 * writes at most outlen bytes including the NUL; negative on error. */
long rx_forcefield_dump(rx_context* ctx, int portable, char* out, long outlen);
/* PairReaxFFMetal::extract("chi"|"eta"|"gamma") (pair_reaxff_metal.cpp:212-227): per force-field type, eta is twice the
 * file value. Arrays of ntypes entries (0-based type index). */
int rx_forcefield_params(rx_context* ctx, int* ntypes, double* chi, double* eta, double* gamma, double* mass);

/* ForceField::match_element as pair_coeff uses it (pair_reaxff_metal.cpp:121-134): the force-field type index of an
 * element symbol (case-insensitive, first three characters), or -1 when the file has no such element. */
int rx_forcefield_element(rx_context* ctx, const char* symbol);

/* ControlParams (include/reaxmetal/forcefield.hpp:73-78) and the `enobonds` pair_style keyword (bonded.hpp:25). */
int rx_set_control(rx_context* ctx, double bond_cut, double hbond_cut, double thb_cut, double thb_cutsq, int enobonds);

/* The systems of this context. natoms[nsys]; origin[3*nsys]; box[9*nsys] lattice vectors a, b, c as rows;
 * periodic[3*nsys] (NULL = all periodic) as Box::periodic (include/reaxmetal/system.hpp:29): along a non-periodic
 * direction no image is taken and atoms are never wrapped (the engine re-fits that direction's extent at every
 * rx_set_positions; an atom that drifts more than 50 A beyond it stops the evaluation); type[NA] force-field type index;
 * tag[NA] atom ids, unique within a system (the owner-computes tie-breaks of neighbor.cpp:295-310 use them).
 * The charge-equilibration histories (the warm start of the next solve) carry over for every atom whose tag existed
 * before the call in the system of the same index, atom count and lattice (the same system handed over again, e.g.
 * after re-neighbouring), wherever the atom now sits in the arrays; other atoms and systems start from zero. */
int rx_set_systems(rx_context* ctx, int nsys, const int* natoms, const double* origin, const double* box, const int* periodic,
                   const int* type, const int64_t* tag);
int rx_num_atoms(const rx_context* ctx);

/* Per-atom list capacities: neighbor-row entries, bond slots, near-row entries (in that order). The engine sizes them
 * from the densest system at rx_set_systems and grows them on overflow, repeating the evaluation (neighbor.cpp:362-374);
 * rx_set_capacities replaces the current values (nbr and near are rounded up to multiples of 32), e.g. to start a
 * serving context from capacities measured earlier. Values below 1 are rejected with RX_ERR_INVALID. */
int rx_set_capacities(rx_context* ctx, int nbr, int bonds, int near_entries);
int rx_get_capacities(const rx_context* ctx, int* out3);
/* Neighbor skin (the `neighbor <skin> bin` command; LAMMPS real units default 2.0, this engine 1.0 A): the rows hold
 * every image within nonb_cut + skin and a system's rows are rebuilt only when one of its atoms has moved more than
 * skin/2 since the last rebuild (neighbor.cpp:362-374 rebuilds every step; the cut-off decisions of every step are the
 * same either way, taken on the current positions). 0 rebuilds every evaluation. */
int rx_set_neighbor(rx_context* ctx, double skin);
/* x[3*NA], in any periodic image (each atom is moved to the image the engine's lists use; the lists are rebuilt only
 * for systems whose atoms moved more than skin/2 since their last rebuild). An array in page-locked memory (from
 * rx_host_alloc) is copied from directly; a pageable one through the context's staging buffer. */
int rx_set_positions(rx_context* ctx, const double* x);
/* Page-locked host memory for the arrays exchanged every step (positions in, gradient out): rx_set_positions and
 * rx_compute copy from and into such arrays directly, without a host-side staging copy. NULL on failure. No
 * counterpart in the reference (its adapter copies through LAMMPS's arrays). */
void* rx_host_alloc(size_t bytes);
void rx_host_free(void* p);
/* positions as held: wrapped into the primary cell at the last list rebuild of their system, unwrapped since */
int rx_get_positions(rx_context* ctx, double* x);
int rx_set_charges(rx_context* ctx, const double* q);     /* q[NA] */
int rx_get_charges(rx_context* ctx, double* q);

/* fix qeq/reaxff/metal <nevery> <swa> <swb> <tol> reaxff [maxiter imax] (fix_qeq_reaxff_metal.cpp; ENGINE_SPEC 7).
 * strict = 1: non-convergence is an error (RX_ERR_NOT_CONVERGED), 0: it is reported through iters/rel only. */
int rx_set_qeq(rx_context* ctx, double swa, double swb, double tol, int imax, int strict);
/* mtl::Context::qeq_solve (metal_backend.hpp:84-86): builds H (compute_H), solves H s = -chi and H t = -1 with the
 * Jacobi-preconditioned CG from the history-extrapolated guesses (Q-23), sets q = s - (sum s / sum t) t
 * (calculate_Q) and advances the histories. iters[2*nsys] and rel[2*nsys] (s then t per system) may be NULL. */
int rx_qeq_solve(rx_context* ctx, int* iters, double* rel);
/* Zeroes the charge-equilibration histories (the stock fix's s_hist/t_hist at initialisation): the next solve starts
 * from s = t = 0. */
int rx_qeq_reset(rx_context* ctx);
/* mtl::Context::qeq_solve (metal_backend.hpp:84-86) for the caller's right-hand sides and guesses, as the resident
 * fix hands them over (fix_qeq_reaxff_metal.cpp:69-75): builds the charge matrix of the current positions, then runs
 * the CG of both systems. b[2*NA] (the s system for every atom, then the t system), x0[2*NA] (same layout; NULL = 0),
 * x_out[2*NA]; per system, s then t: iters[2*nsys] (iterations performed + 1, as the stock loop counts),
 * rel[2*nsys] (final relative residual sqrt(r.M^-1 r)/|b|), status[2*nsys] (1 converged, 2 breakdown, 3 iteration
 * limit). The preconditioner is diag(eta)^-1 (the fix's Hdia_inv). Charges and histories are not touched. Any of
 * iters, rel, status may be NULL. */
int rx_qeq_cg(rx_context* ctx, const double* b, const double* x0, double* x_out, int* iters, double* rel, int* status);
/* mtl::Context::qeq_matvec (metal_backend.hpp:82): y = (diag(eta) + H) v over the owned atoms, v[NA], y[NA]. */
int rx_qeq_matvec(rx_context* ctx, const double* v, double* y);
/* CG iteration counts and final relative residuals (s, t per system, as rx_qeq_solve reports them) of the most recent
 * charge solve of any entry point (rx_compute with RX_COMPUTE_QEQ, rx_md_run steps, rx_qeq_solve). */
int rx_qeq_last(const rx_context* ctx, int32_t* iters, double* rel);
/* FP64 residual passes of the most recent single-system charge solve (the first residual, each refinement, and the
 * final check); -1 without one. */
int rx_qeq_refinements(rx_context* ctx);

/* PairReaxFFMetal::compute (pair_reaxff_metal.cpp:412-524) for every system: energies[13*nsys] in the reference's
 * EnergyTerm order (bond, over, under, lone_pair, valence, penalty, coalition, hbond, torsion, conjugation, vdw,
 * coulomb, polarization; kcal/mol), grad[3*NA] = dE/dx (the physical force is -grad), census[7*NA] (bonds,
 * angle_sets, torsions, hbonds, nonbonded, sbo_region, lp_trunc; only with RX_COMPUTE_CENSUS), counts[4] (bonds,
 * counted non-bonded pairs, neighbor entries, H-bond triples). Any output pointer may be NULL. */
int rx_compute(rx_context* ctx, int flags, double* energies, double* grad, int32_t* census, int64_t* counts);

/* The pair side of fix acks2/reaxff (add_acks2_terms, src/cpu/acks2.cpp:11-63; pair_reaxff_metal.cpp:482-485,492):
 * s_kin[NA] the kinetic potentials of the fix's solution (its s[N + i]), or NULL to switch the terms off. While set,
 * every force evaluation adds the polarization coupling 23.02 q s and the bond-softness Coulomb term over the pairs
 * within (bcut_acks2_i + bcut_acks2_j)/2 (softness = general parameter 34) to the Coulomb and polarization energies,
 * the forces and the virial. rx_set_systems switches them off. */
int rx_set_acks2(rx_context* ctx, const double* s_kin);

/* Per-atom tallies of the last rx_compute with RX_COMPUTE_PERATOM (the step the reference's pair style falls back to
 * cpu64 for, pair_reaxff_metal.cpp:430-433,506-510): eatom[NA] per-atom energies by the reference's rules (bond, C2,
 * torsion and pair energies half to each end, H-bonds a third to each of donor, hydrogen and acceptor, the rest to
 * the centre atom; images folded onto their owners), vatom[6*NA] per-atom virials (LAMMPS order), each interaction's
 * virial kept by the atom it is centred on (pairs and BO-chain bonds half to each end) - the atoms' sum is exactly
 * rx_get_virial, the split among atoms is not LAMMPS's v_tally fractions. Either output may be NULL. */
int rx_get_peratom(rx_context* ctx, double* eatom, double* vatom);
/* The bond table of the last force evaluation (publish_bonds, pair_reaxff_metal.cpp:330-368; BondTable,
 * include/reaxmetal/bonded.hpp:32-37), for fix reaxff/bonds and reaxff/species: start[NA+1], and per bond the
 * partner's atom index, its lattice shift shift[3*nb] (the image the bond reaches), the corrected bond order;
 * total_bo[NA] and nlp[NA] per atom. Any output but start may be NULL. Returns the number of bonds nb; with start ==
 * NULL or cap < nb nothing is written (call again with cap >= nb); -1 on error. */
long long rx_get_bonds(rx_context* ctx, int* start, int* partner, int* shift, double* bo, double* total_bo, double* nlp,
                       long long cap);

/* Gradient dE/dx[3*NA] of the most recent force evaluation (rx_compute or the last step of rx_md_run). */
int rx_get_gradient(rx_context* ctx, double* grad);

/* Virial of the most recent force evaluation (rx_compute or the last rx_md_run step) per system: virial[6*nsys] in
 * LAMMPS's order xx, yy, zz, xy, xz, yz, the sum of x_a f_b over every atom and periodic image (kcal/mol) - what
 * virial_fdotr_compute() makes of the owned + ghost forces the reference's pair style hands LAMMPS
 * (pair_reaxff_metal.cpp:500-504,523). rx_compute returns forces folded onto owned atoms, so a LAMMPS adapter sets
 * the pair's virial from this array instead of calling virial_fdotr_compute(). Computed on the device from relative
 * positions inside each interaction, in fixed order. */
int rx_get_virial(rx_context* ctx, double* virial);

/* The 14-slot energy vector LAMMPS's `pair_style reaxff` exposes (to_lammps_pvector, src/core/energy_terms.cpp:35-72;
 * pair_reaxff.cpp:501-514) from the 13 energies of one system: eb, ea (over + under), elp, emol (0), ev, epen, ecoa,
 * ehb, et, eco, ew, ep, efi (0), eqeq (polarization); and the pair's eng_vdwl (every term but Coulomb and
 * polarization) and eng_coul (Coulomb + polarization) (pair_reaxff_metal.cpp:515-519). Any output may be NULL; needs
 * no context. */
int rx_pvector(const double* energies13, double* pvector14, double* eng_vdwl, double* eng_coul);

/* Nose-Hoover chain NVT (the LAMMPS `fix nvt temp Tstart Tstop Tdamp` the reference's examples run), velocity Verlet
 * with dt [fs]. mass[ntypes] g/mol per force-field type. Charges are re-equilibrated before every force evaluation
 * unless rx_md_charges switched that off. chain = 0 runs plain NVE (`fix nve`). */
int rx_md_setup(rx_context* ctx, const double* mass, double dt, double t_start, double t_stop, double t_damp, int chain);
int rx_set_velocities(rx_context* ctx, const double* v);  /* v[3*NA] A/fs */
/* on = 0: rx_md_run keeps the charges as set (a run without a charge fix, as the reference's one-element carbon
 * example; q = 0 there); on = 1 (default): charges re-equilibrated before every force evaluation. */
int rx_md_charges(rx_context* ctx, int on);
int rx_get_velocities(rx_context* ctx, double* v);
/* nsteps steps of every system; energies (13*nsys, last step) and temperature (nsys) may be NULL */
int rx_md_run(rx_context* ctx, int nsteps, double* energies, double* temperature);

/* Charge equilibration without any device allocation (this entry point has no counterpart in the reference).
 * For callers that cannot let a library call cudaMalloc: codes that own all device memory through their own pooled
 * allocator or fixed budget, and codes running where an allocation and its implicit device synchronisation are not
 * allowed. It solves (diag(eta) + H) s = -chi and (diag(eta) + H) t = -1 with the engine's Jacobi-preconditioned CG
 * (the stopping rule of fix qeq/reaxff: sqrt(r.M^-1 r)/|b| <= tol, at most imax - 1 iterations) and writes
 * q = s - (sum s / sum t) t. Every pointer is a device pointer on the current device, owned by the caller:
 * H as CSR (row_start[n+1], col[nnz], val[nnz]; every periodic image of a pair summed into its entry), eta[n] and
 * chi[n] per atom, s[n] and t[n] the initial guesses on entry and the solutions on return, q[n] the charges,
 * iters[2] and rel[2] (s then t; may be NULL). iters[k] = -1 reports a CG breakdown of that right-hand side (a step
 * length that is not finite: a singular or indefinite matrix); s, t and q are then not a solution. Pass iters to see
 * a breakdown: without it a breakdown cannot be told from convergence. The call is asynchronous on `stream` (a
 * cudaStream_t, NULL = default). A launch failure returns RX_ERR_CUDA; the CUDA error state is peeked, not cleared, so
 * an error left pending by earlier work on the thread is reported here as well.
 * The CG work vectors live in one fixed device array of RX_QEQ_STATIC_MAX_ATOMS * 8 doubles (2 MiB) that every GPU
 * loading the library holds until the process exits; larger n is rejected with RX_ERR_INVALID. All calls share that
 * array: calls whose kernels overlap on the GPU (other streams, other threads) race, so serialise them. The array keeps
 * the last call's contents; nothing in it needs to start at zero, since every work vector is written before it is
 * read. The first call on a device does a one-time set-up with that device current: it looks up the array's device
 * address (cudaGetSymbolAddress), which under CUDA's lazy module loading also loads this library's device code and
 * its array on that device - the driver's own allocation and synchronisation. Make that first call at start-up and
 * before any stream capture; n = 0 does the set-up alone (no other argument is read, nothing is launched).
 * err/errlen (may be NULL) receive a message. */
#define RX_QEQ_STATIC_MAX_ATOMS 32768
int rx_qeq_solve_static(int n, const int* row_start, const int* col, const double* val, const double* eta, const double* chi,
                        double* s, double* t, double* q, double tol, int imax, int* iters, double* rel, void* stream,
                        char* err, int errlen);

/* Serving (continuous batching). rx_update_systems replaces the context's systems by nkeep of the current ones
 * (keep[k] = current system index, in their new order) followed by nnew new systems described as for rx_set_systems
 * (natoms[nnew], origin[3*nnew], box[9*nnew], periodic[3*nnew] or NULL, type/tag for the new atoms), with positions
 * x[3*NA_new] and velocities v[3*NA_new] (NULL = 0) of the new atoms. Kept systems carry their positions, velocities,
 * charges, charge histories and chain state on the device; every system's neighbor rows are rebuilt at the next
 * evaluation, and the next rx_md_run starts with a force evaluation. Per-system targets set by rx_md_targets are
 * cleared. No counterpart in the reference (its systems live in LAMMPS). */
int rx_update_systems(rx_context* ctx, int nkeep, const int* keep, int nnew, const int* natoms, const double* origin,
                      const double* box, const int* periodic, const int* type, const int64_t* tag, const double* x,
                      const double* v);
/* Per-system NVT settings for serving: t_target[nsys] target temperatures in K (NULL: the common ramp of
 * rx_md_setup) and active[nsys] (NULL: all; 0 freezes a system: its atoms and its chain are not advanced, its
 * forces are still evaluated). */
int rx_md_targets(rx_context* ctx, const double* t_target, const int* active);

/* Launch-shape tuning (no counterpart in the reference, whose Metal kernels use a fixed threadgroup of 64). All but
 * RX_TUNE_CG_BLOCKS_PER_SM leave every result bit unchanged. RX_TUNE_*_TPB: threads per block of a warp-per-atom kernel (64, 128, 256: atoms per
 * block x 32) or of the thread-per-atom bonded kernels (32, 64, 128); RX_TUNE_LONE_GRID_MIN: a context holding one
 * system of more atoms takes the single-system CG (all SMs on its rows, default 4096; a batch always takes the
 * segmented CG, so a system alone and in a batch give the same bits only below this size); RX_TUNE_OVERLAP: 1 (the
 * default) runs the bonded terms, which need no charge, concurrently with the charge solve, 0 after it;
 * RX_TUNE_CG_BLOCKS_PER_SM: threads per SM of the single-system CG in units of 256, as one block per SM (1-4, default
 * 2, leaving room for the concurrent bonded terms; 0: four) - unlike the other keys this changes the order of the CG's sums, so the charges' last
 * bits (a fixed setting stays bitwise reproducible), and rx_autotune does not touch it. rx_autotune times every
 * candidate shape on the current systems (reps launches each, CUDA events) and keeps the fastest; chosen[5] (may be
 * NULL) receives pairs, bonds, non-bonded, H-bond and per-atom shapes. */
#define RX_TUNE_PAIRS_TPB 1
#define RX_TUNE_BONDS_TPB 2
#define RX_TUNE_NONBONDED_TPB 3
#define RX_TUNE_HBOND_TPB 4
#define RX_TUNE_ATOM_TPB 5
#define RX_TUNE_LONE_GRID_MIN 6
#define RX_TUNE_OVERLAP 7
#define RX_TUNE_CG_BLOCKS_PER_SM 8
int rx_set_tuning(rx_context* ctx, int key, int value);
int rx_autotune(rx_context* ctx, int reps, int* chosen);

/* Number of this engine's own kernels launched on the context so far (library kernels, e.g. the radix sort of the cell
 * lists, are not counted). */
int64_t rx_kernel_launches(const rx_context* ctx);
/* The CUDA stream the context launches on (a cudaStream_t), for callers that time or order work around it. */
void* rx_stream(rx_context* ctx);
/* Per-phase device time of the last rx_compute / rx_md_run (milliseconds, summed over the call) when timing is on:
 * names is a '\n'-separated list written into names_out; returns the number of phases. */
int rx_set_timing(rx_context* ctx, int on);
int rx_phase_times(rx_context* ctx, char* names_out, long names_len, double* ms, int max_phases);

#ifdef __cplusplus
}
#endif
#endif
