/* TEST INFRASTRUCTURE ONLY: the CPU oracle of the ReaxFF force + charge-equilibration step.
 *
 * A serial FP64 restatement, in plain C, of the reference's `backend cpu64` engine and of the stock QEq solve
 * it is paired with. Only tests/, the smoke check and the CPU-baseline leg of bench.py may call it; the
 * product never links it. It is pinned against the reference itself (oracle/_ref, built from the reference
 * sources) and against golden vectors generated from it (tests/golden/).
 *
 * Parameter tables are flat double arrays; the field offsets below are this oracle's own layout (filled by
 * oracle/ffield.py from the ffield text).
 */
#ifndef RX_ORACLE_H
#define RX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* per-type ("single body") fields */
enum {
  SB_R_S, SB_VALENCY, SB_MASS, SB_R_VDW, SB_EPSILON, SB_GAMMA, SB_R_PI, SB_VALENCY_E, SB_NLP_OPT,
  SB_ALPHA, SB_GAMMA_W, SB_VALENCY_BOC, SB_P_OVUN5, SB_CHI, SB_ETA, SB_P_HBOND,
  SB_R_PI_PI, SB_P_LP2, SB_B_O_131, SB_B_O_132, SB_B_O_133,
  SB_P_OVUN2, SB_P_VAL3, SB_VALENCY_VAL, SB_P_VAL5, SB_RCORE2, SB_ECORE2, SB_ACORE2,
  SB_HEAVY, SB_C2SPECIES, SB_BCUT_ACKS2, SB_NFIELDS
};

/* per-pair ("two body") fields, symmetric n x n */
enum {
  TB_P_BO1, TB_P_BO2, TB_P_BO3, TB_P_BO4, TB_P_BO5, TB_P_BO6, TB_R_S, TB_R_P, TB_R_PP,
  TB_P_BOC3, TB_P_BOC4, TB_P_BOC5, TB_P_BE1, TB_P_BE2, TB_DE_S, TB_DE_P, TB_DE_PP, TB_P_OVUN1,
  TB_D, TB_ALPHA, TB_R_VDW, TB_GAMMA_W, TB_RCORE, TB_ECORE, TB_ACORE, TB_LGCIJ, TB_LGRE, TB_GAMMA,
  TB_V13COR, TB_OVC, TB_TRIPLE_STAB, TB_NFIELDS
};

/* three-body set fields (at most 5 sets per ordered triple), four-body and H-bond fields */
enum { TH_THETA_00, TH_P_VAL1, TH_P_VAL2, TH_P_VAL4, TH_P_VAL7, TH_P_PEN1, TH_P_COA1, TH_NFIELDS };
#define RXO_MAX_THB_SETS 5
enum { FB_V1, FB_V2, FB_V3, FB_P_TOR1, FB_P_COT1, FB_NFIELDS };
enum { HB_R0, HB_P_HB1, HB_P_HB2, HB_P_HB3, HB_NFIELDS };

typedef struct {
  int nt;                 /* number of atom types */
  int ngp;                /* number of general parameters (>= 39) */
  const double* gp;       /* ngp */
  int vdw_type;           /* 1 shielding, 2 inner wall, 3 both */
  double bo_cut, nonb_low, nonb_cut;
  const double* sbp;      /* nt * SB_NFIELDS */
  const double* tbp;      /* nt * nt * TB_NFIELDS */
  const int* thb_n;       /* nt^3: number of valence-angle sets of the ordered triple (i, centre j, k) */
  const double* thb;      /* nt^3 * RXO_MAX_THB_SETS * TH_NFIELDS */
  const int* fbp_on;      /* nt^4: torsion entry exists */
  const double* fbp;      /* nt^4 * FB_NFIELDS */
  const int* hbp_on;      /* nt^3: H-bond entry exists (donor, H, acceptor) */
  const double* hbp;      /* nt^3 * HB_NFIELDS */
  int lgvdw;              /* 1: `pair_style reaxff lgvdw yes` (the lg dispersion inside the inner-wall branch) */
} rxo_ff;

typedef struct {
  double bond_cut, hbond_cut, thb_cut, thb_cutsq;   /* control values (reference defaults 5.0, 7.5, 0.001, 0.00001) */
  int enobonds;                                     /* 1: lone pair / under-coordination for atoms without bonds */
  double shell;                                     /* ghost shell width [A] */
} rxo_ctl;

typedef struct {
  double origin[3];
  double vec[9];          /* lattice vectors a, b, c as rows */
  int periodic[3];
} rxo_box;

/* Energies in the reference's EnergyTerm order: bond, over, under, lone_pair, valence, penalty, coalition,
 * hbond, torsion, conjugation, vdw, coulomb, polarization. */
#define RXO_NTERMS 13
#define RXO_NCENSUS 7

/* One energy + gradient evaluation (bonded + non-bonded with the given charges; q == NULL skips the non-bonded
 * terms as the reference's driver does). grad: 3n, dE/dx folded onto the owned atoms. census: 7n (bonds,
 * angle_sets, torsions, hbonds, nonbonded, sbo_region, lp_trunc) or NULL. counts: [undirected bonds incl.
 * ghost rows, counted non-bonded pairs, nall, far-list entries] or NULL. virial6: NULL or the LAMMPS fdotr virial
 * (sum over owned + ghost atoms of x_a f_b, order xx yy zz xy xz yz, f = -gradient). Returns 0, or a nonzero error
 * code with a message in err. */
int rxo_single_point(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
                     const long long* tag, const double* q, double* e13, double* grad, int* census, long long* counts,
                     double* virial6, char* err, int errlen);

/* The same single point with the pair-side terms of the ACKS2 charge model added (src/cpu/acks2.cpp:11-63): s_kin[n]
 * the kinetic potentials of the owned atoms (an image takes its owner's). NULL s_kin is rxo_single_point. */
int rxo_single_point_acks2(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x,
                           const int* type, const long long* tag, const double* q, const double* s_kin, double* e13,
                           double* grad, int* census, long long* counts, double* virial6, char* err, int errlen);

/* Charge equilibration: solves H s = -chi and H t = -1 with the stock Jacobi-preconditioned CG (tolerance
 * sqrt(r.M^-1 r)/|b| <= tol, at most imax - 1 iterations) from the initial guesses s0/t0 (n each), then
 * q = s - (sum s / sum t) t. H_ij = 14.4 Tap(r) / cbrt(r^3 + (gamma_i gamma_j)^-1.5) over every periodic pair with
 * r <= swb, H_ii = eta (twice the file value). iters[2] receives the iteration counts of the s and t solves,
 * rel[2] the final relative residuals. */
int rxo_qeq(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
            const long long* tag, double swa, double swb, double tol, int imax, const double* s0, const double* t0,
            double* q, double* s, double* t, int* iters, double* rel, char* err, int errlen);

/* Matrix-vector product y = H x of the same charge matrix (n owned entries), for tests of a device matvec. */
int rxo_qeq_matvec(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
                   const long long* tag, double swa, double swb, const double* v, double* y, char* err, int errlen);

#ifdef __cplusplus
}
#endif
#endif
