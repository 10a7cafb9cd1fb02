/* TEST INFRASTRUCTURE ONLY: serial FP64 restatement of the reference's cpu64 ReaxFF engine (see rx_oracle.h).
 *
 * Every block cites the reference file:line it restates. The traversal is the reference's "ghost-native" one:
 * periodic images are materialised as ghost atoms (owner + lattice shift), a half far list with j > i is built
 * over owned and ghost atoms, the bonded terms run over that expanded set, and the gradient of every ghost is
 * folded onto its owner at the end (tools/energy_tool.cpp:131-136).
 */
#include "rx_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------------ helpers */
#define C_ELE 332.06371      /* reaxff_defs.h C_ele, as in include/reaxmetal/terms.hpp:21 */
#define KCAL_TO_EV 23.02     /* include/reaxmetal/terms.hpp:22 (really eV -> kcal/mol) */
#define EV_TO_KCAL 14.4      /* QEq matrix constant (docs/ENGINE_SPEC.md section 1) */
#define CONST_PI 3.14159265  /* src/cpu/bonded.cpp:52 */
#define HB_THRESHOLD 1e-2    /* src/cpu/bonded.cpp:54 */
#define MIN_SINE 1e-10       /* src/cpu/bonded.cpp:55 */
#define SMALL_TIE 1e-4       /* src/neighbor/neighbor.cpp:297 */

static void seterr(char* err, int errlen, const char* fmt, ...) {
  if (!err || errlen <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, (size_t)errlen, fmt, ap);
  va_end(ap);
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static void axpy3(double* y, double a, const double* x) { y[0] += a * x[0]; y[1] += a * x[1]; y[2] += a * x[2]; }

/* growable array of fixed-size records */
typedef struct { char* p; int n, cap, sz; } dyn;
static void* dyn_push(dyn* d) {
  if (d->n == d->cap) {
    d->cap = d->cap ? 2 * d->cap : 8;
    d->p = (char*)realloc(d->p, (size_t)d->cap * (size_t)d->sz);
  }
  void* r = d->p + (size_t)d->n * (size_t)d->sz;
  memset(r, 0, (size_t)d->sz);
  d->n++;
  return r;
}
#define DYN_AT(d, T, i) (((T*)(d).p)[i])

/* ------------------------------------------------------------------------------------------------ box / images */
/* src/core/system.cpp:30-41 */
static double box_volume(const rxo_box* b) {
  double c[3];
  cross3(b->vec + 3, b->vec + 6, c);
  return dot3(b->vec, c);
}
static void box_heights(const rxo_box* b, double* h) {
  const double v = fabs(box_volume(b));
  double c[3];
  cross3(b->vec + 3, b->vec + 6, c); h[0] = v / sqrt(dot3(c, c));
  cross3(b->vec + 6, b->vec + 0, c); h[1] = v / sqrt(dot3(c, c));
  cross3(b->vec + 0, b->vec + 3, c); h[2] = v / sqrt(dot3(c, c));
}
static void box_frac(const rxo_box* b, const double* r, double* f) {
  const double d[3] = {r[0] - b->origin[0], r[1] - b->origin[1], r[2] - b->origin[2]};
  const double det = box_volume(b);
  double c[3];
  cross3(b->vec + 3, b->vec + 6, c); f[0] = dot3(d, c) / det;
  cross3(b->vec + 6, b->vec + 0, c); f[1] = dot3(d, c) / det;
  cross3(b->vec + 0, b->vec + 3, c); f[2] = dot3(d, c) / det;
}

typedef struct {
  int nlocal, nall;
  double* x;      /* 3 * nall */
  int* type;
  long long* tag;
  int* owner;
} atomset;

static void atomset_free(atomset* a) { free(a->x); free(a->type); free(a->tag); free(a->owner); }

/* expand_images, src/neighbor/neighbor.cpp:18-88: owned atoms wrapped into the primary cell first, then every image
 * whose fractional coordinates lie within shell/height of [0,1] along each periodic dimension, ordered by (s0, s1, s2,
 * owner) with the zero shift omitted. */
static int expand_images(const rxo_box* box, double shell, int n, const double* x, const int* type, const long long* tag,
                         atomset* a, char* err, int errlen) {
  double h[3], w[3] = {0, 0, 0};
  int smax[3] = {0, 0, 0};
  box_heights(box, h);
  for (int d = 0; d < 3; ++d)
    if (box->periodic[d]) { w[d] = shell / h[d]; smax[d] = (int)ceil(w[d]) + 1; }
  int cap = n * 8 + 64, nall = n;
  a->x = (double*)malloc(sizeof(double) * 3 * (size_t)cap);
  a->type = (int*)malloc(sizeof(int) * (size_t)cap);
  a->tag = (long long*)malloc(sizeof(long long) * (size_t)cap);
  a->owner = (int*)malloc(sizeof(int) * (size_t)cap);
  double* frac = (double*)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) {
    double r[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]}, f[3];
    for (int c = 0; c < 3; ++c)
      if (!isfinite(r[c])) { seterr(err, errlen, "non-finite coordinate of atom %d", i); free(frac); return 1; }
    box_frac(box, r, f);
    double k[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d)
      if (box->periodic[d]) k[d] = floor(f[d]);
    for (int d = 0; d < 3; ++d)
      if (k[d] != 0.0)
        for (int c = 0; c < 3; ++c) r[c] -= k[d] * box->vec[3 * d + c];
    box_frac(box, r, f);
    for (int c = 0; c < 3; ++c) { a->x[3 * i + c] = r[c]; frac[3 * i + c] = f[c]; }
    a->type[i] = type[i]; a->tag[i] = tag[i]; a->owner[i] = i;
  }
  for (int s0 = -smax[0]; s0 <= smax[0]; ++s0)
    for (int s1 = -smax[1]; s1 <= smax[1]; ++s1)
      for (int s2 = -smax[2]; s2 <= smax[2]; ++s2) {
        if (s0 == 0 && s1 == 0 && s2 == 0) continue;
        const int s[3] = {s0, s1, s2};
        double sh[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k)
          for (int c = 0; c < 3; ++c) sh[c] += (double)s[k] * box->vec[3 * k + c];
        for (int k = 0; k < n; ++k) {
          int inside = 1;
          for (int d = 0; d < 3 && inside; ++d) {
            if (!box->periodic[d]) continue;
            const double g = frac[3 * k + d] + (double)s[d];
            inside = (g >= -w[d]) && (g <= 1.0 + w[d]);
          }
          if (!inside) continue;
          if (nall == cap) {
            cap *= 2;
            a->x = (double*)realloc(a->x, sizeof(double) * 3 * (size_t)cap);
            a->type = (int*)realloc(a->type, sizeof(int) * (size_t)cap);
            a->tag = (long long*)realloc(a->tag, sizeof(long long) * (size_t)cap);
            a->owner = (int*)realloc(a->owner, sizeof(int) * (size_t)cap);
          }
          for (int c = 0; c < 3; ++c) a->x[3 * nall + c] = a->x[3 * k + c] + sh[c];
          a->type[nall] = a->type[k]; a->tag[nall] = a->tag[k]; a->owner[nall] = k;
          ++nall;
        }
      }
  free(frac);
  a->nlocal = n;
  a->nall = nall;
  return 0;
}

/* ------------------------------------------------------------------------------------------------ far list */
typedef struct {
  long long* row_start;  /* nall + 1 */
  int* nbr;
  double* dist;
  double* dvec;          /* 3 per entry, x_j - x_i */
  long long entries;
} farlist;

static void farlist_free(farlist* f) { free(f->row_start); free(f->nbr); free(f->dist); free(f->dvec); }

static int cmp_int(const void* a, const void* b) { const int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y); }

/* build_far_list, src/neighbor/neighbor.cpp:180-212: row i holds every j > i with |x_j - x_i|^2 <= rc^2, rc = nonb for
 * owned rows and bond for ghost rows (ENGINE_SPEC Q-08), sorted by j; dvec = x_j - x_i, d = sqrt(dx^2+dy^2+dz^2). A
 * uniform cell grid over the bounding box of all atoms (cell >= max cut-off) finds the candidates. */
static int build_far_list(const atomset* a, double nonb, double bond, farlist* f) {
  const int N = a->nall;
  const double cmin = nonb > bond ? nonb : bond;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  if (N > 0)
    for (int c = 0; c < 3; ++c) lo[c] = hi[c] = a->x[c];
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) {
      if (a->x[3 * i + c] < lo[c]) lo[c] = a->x[3 * i + c];
      if (a->x[3 * i + c] > hi[c]) hi[c] = a->x[3 * i + c];
    }
  int nc[3];
  double cs[3];
  for (int c = 0; c < 3; ++c) {
    const double k = floor((hi[c] - lo[c]) / cmin);
    nc[c] = k < 1.0 ? 1 : (int)k;
    if (nc[c] > 512) nc[c] = 512;
    cs[c] = (hi[c] - lo[c]) / nc[c];
    if (cs[c] < cmin) cs[c] = cmin;
  }
  const long long ncell = (long long)nc[0] * nc[1] * nc[2];
  int* cell = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  long long* cstart = (long long*)calloc((size_t)ncell + 1, sizeof(long long));
  for (int i = 0; i < N; ++i) {
    int cc[3];
    for (int d = 0; d < 3; ++d) {
      const double t = floor((a->x[3 * i + d] - lo[d]) / cs[d]);
      cc[d] = t < 0.0 ? 0 : (t > nc[d] - 1 ? nc[d] - 1 : (int)t);
    }
    cell[i] = (cc[2] * nc[1] + cc[1]) * nc[0] + cc[0];
    cstart[cell[i] + 1]++;
  }
  for (long long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
  int* items = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  long long* fill = (long long*)malloc(sizeof(long long) * (size_t)ncell);
  memcpy(fill, cstart, sizeof(long long) * (size_t)ncell);
  for (int i = 0; i < N; ++i) items[fill[cell[i]]++] = i;
  free(fill);

  long long cap = 1024;
  f->row_start = (long long*)malloc(sizeof(long long) * ((size_t)N + 1));
  f->nbr = (int*)malloc(sizeof(int) * (size_t)cap);
  f->dist = (double*)malloc(sizeof(double) * (size_t)cap);
  f->dvec = (double*)malloc(sizeof(double) * 3 * (size_t)cap);
  long long m = 0;
  int* row = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  f->row_start[0] = 0;
  for (int i = 0; i < N; ++i) {
    const double rc = i < a->nlocal ? nonb : bond, rc2 = rc * rc;
    const int c = cell[i], cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
    int nr = 0;
    for (int z = cz - 1; z <= cz + 1; ++z) {
      if (z < 0 || z >= nc[2]) continue;
      for (int y = cy - 1; y <= cy + 1; ++y) {
        if (y < 0 || y >= nc[1]) continue;
        for (int xx = cx - 1; xx <= cx + 1; ++xx) {
          if (xx < 0 || xx >= nc[0]) continue;
          const int cc = (z * nc[1] + y) * nc[0] + xx;
          for (long long p = cstart[cc]; p < cstart[cc + 1]; ++p) {
            const int j = items[p];
            if (j <= i) continue;
            const double dv[3] = {a->x[3 * j] - a->x[3 * i], a->x[3 * j + 1] - a->x[3 * i + 1], a->x[3 * j + 2] - a->x[3 * i + 2]};
            const double d2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
            if (d2 <= rc2) row[nr++] = j;
          }
        }
      }
    }
    qsort(row, (size_t)nr, sizeof(int), cmp_int);
    if (m + nr > cap) {
      while (m + nr > cap) cap *= 2;
      f->nbr = (int*)realloc(f->nbr, sizeof(int) * (size_t)cap);
      f->dist = (double*)realloc(f->dist, sizeof(double) * (size_t)cap);
      f->dvec = (double*)realloc(f->dvec, sizeof(double) * 3 * (size_t)cap);
    }
    for (int e = 0; e < nr; ++e) {
      const int j = row[e];
      const double dv[3] = {a->x[3 * j] - a->x[3 * i], a->x[3 * j + 1] - a->x[3 * i + 1], a->x[3 * j + 2] - a->x[3 * i + 2]};
      f->nbr[m] = j;
      f->dist[m] = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
      memcpy(f->dvec + 3 * m, dv, sizeof dv);
      ++m;
    }
    f->row_start[i + 1] = m;
  }
  f->entries = m;
  free(row); free(items); free(cstart); free(cell);
  return 0;
}

/* classify_nonbonded_entry, src/neighbor/neighbor.cpp:295-310: 0 none, 1 owned-owned, 2 owned-ghost, 3 self image */
static int classify(int j, int nlocal, long long ti, long long tj, const double* dv) {
  if (j < nlocal) return 1;
  if (ti < tj) return 2;
  if (ti == tj) {
    int flag = 0;
    if (dv[2] > SMALL_TIE) flag = 1;
    else if (fabs(dv[2]) < SMALL_TIE) {
      if (dv[1] > SMALL_TIE) flag = 1;
      else if (fabs(dv[1]) < SMALL_TIE && dv[0] > SMALL_TIE) flag = 1;
    }
    return flag ? 3 : 0;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------------ term formulas */
/* safe_exp, include/reaxmetal/terms.hpp:29-33 (double cap 700) */
static double safe_exp(double x) { return exp(x > 700.0 ? 700.0 : x); }

#define SB(t, f) (ff->sbp[(size_t)(t) * SB_NFIELDS + (f)])
#define TB(a, b, f) (ff->tbp[((size_t)(a) * (size_t)ff->nt + (size_t)(b)) * TB_NFIELDS + (f)])

typedef struct {
  int nbr, sym;
  double d, dvec[3], dBOp[3], dln_s[3], dln_pi[3], dln_pi2[3];
  double BO, BO_s, BO_pi, BO_pi2;
  double C1dbo, C2dbo, C3dbo, C1dbopi, C2dbopi, C3dbopi, C4dbopi, C1dbopi2, C2dbopi2, C3dbopi2, C4dbopi2;
  double Cdbo, Cdbopi, Cdbopi2;
} bond_t;

typedef struct { int thb, pthb; double theta, dcos_di[3], dcos_dj[3], dcos_dk[3]; } thb_t;
typedef struct { int nbr; double scl, d, dvec[3]; } hbe_t;

typedef struct {   /* atom_quantities, include/reaxmetal/terms.hpp:141-164 */
  double Delta, Delta_e, Delta_boc, Delta_val, vlpex, nlp, Delta_lp, Clp, dDelta_lp, nlp_temp, Delta_lp_temp, dDelta_lp_temp;
} aq_t;

/* reaxff_valence_angles.cpp:36-70 as restated in src/cpu/bonded.cpp:58-75 */
static void calc_theta(const double* dji, double d_ji, const double* djk, double d_jk, double* theta, double* cos_theta) {
  double c = dot3(dji, djk) / (d_ji * d_jk);
  if (c > 1.0) c = 1.0;
  if (c < -1.0) c = -1.0;
  *cos_theta = c;
  *theta = acos(c);
}
static void calc_dcos(const double* dji, double d_ji, const double* djk, double d_jk, double* di, double* dj, double* dk) {
  const double sq_ji = d_ji * d_ji, sq_jk = d_jk * d_jk;
  const double inv = 1.0 / (d_ji * d_jk);
  const double inv3 = inv * inv * inv;
  const double Cdot = dot3(dji, djk) * inv3;
  for (int t = 0; t < 3; ++t) {
    di[t] = djk[t] * inv - Cdot * sq_jk * dji[t];
    dj[t] = -(djk[t] + dji[t]) * inv + Cdot * (sq_jk * dji[t] + sq_ji * djk[t]);
    dk[t] = dji[t] * inv - Cdot * sq_ji * djk[t];
  }
}

/* tag-order test used by the bond energy (src/cpu/bonded.cpp:226-232) and the torsion (:487-493): 1 = skip */
static int skip_by_tag(const atomset* a, int i, int j) {
  if (a->tag[i] > a->tag[j]) return 1;
  if (a->tag[i] == a->tag[j]) {
    const double* xi = a->x + 3 * i;
    const double* xj = a->x + 3 * j;
    if (xj[2] < xi[2]) return 1;
    if (xj[2] == xi[2] && xj[1] < xi[1]) return 1;
    if (xj[2] == xi[2] && xj[1] == xi[1] && xj[0] < xi[0]) return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------------ bonded core */
/* compute_bonded_core, src/cpu/bonded.cpp:86-800 (Real = double). e: 10 bonded terms in EnergyTerm order slots. */
static int bonded_core(const rxo_ff* ff, const rxo_ctl* ctl, const atomset* a, const farlist* far, double* e13, double* f,
                       int* census, long long* nbonds, char* err, int errlen) {
  const int N = a->nall, n = a->nlocal;
  const double* gp = ff->gp;
  const double bo_cut = ff->bo_cut;
  const double p_boc1 = gp[0], p_boc2 = gp[1], p_lp1 = gp[15], p_lp3 = gp[5];
  const double gp3 = gp[3], gp4 = gp[4], gp7 = gp[7], gp10 = gp[10];
  const double p_ovun3 = gp[32], p_ovun4 = gp[31], p_ovun6 = gp[6], p_ovun7 = gp[8], p_ovun8 = gp[9];
  const int c2_gate = p_lp3 > 0.001;
  const double thb_cut = ctl->thb_cut, thb_cutsq = ctl->thb_cutsq;

  dyn* bonds = (dyn*)calloc((size_t)N, sizeof(dyn));
  dyn* hbonds = (dyn*)calloc((size_t)N, sizeof(dyn));
  for (int i = 0; i < N; ++i) { bonds[i].sz = (int)sizeof(bond_t); hbonds[i].sz = (int)sizeof(hbe_t); }
  double* dDeltap_self = (double*)calloc(3 * (size_t)N, sizeof(double));
  double* total_bo = (double*)calloc((size_t)N, sizeof(double));
  double* Deltap = (double*)calloc((size_t)N, sizeof(double));
  double* Deltap_boc = (double*)calloc((size_t)N, sizeof(double));
  double* CdDelta = (double*)calloc((size_t)N, sizeof(double));
  aq_t* aq = (aq_t*)calloc((size_t)N, sizeof(aq_t));
  (void)err; (void)errlen;

  /* ---- bond list + BOp (src/cpu/bonded.cpp:107-162) */
  for (int i = 0; i < N; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    for (long long pj = far->row_start[i]; pj < far->row_start[i + 1]; ++pj) {
      const int j = far->nbr[pj];
      const double d = far->dist[pj];
      const double cutoff = (i < n && ctl->hbond_cut > ctl->bond_cut) ? ctl->hbond_cut : ctl->bond_cut;
      if (!(d <= cutoff)) continue;
      const int tj = a->type[j];
      if (tj < 0) continue;
      const int phi = (int)SB(ti, SB_P_HBOND), phj = (int)SB(tj, SB_P_HBOND);
      if (i < n && ctl->hbond_cut > 0 && (phi == 1 || phi == 2) && d <= ctl->hbond_cut) {
        const double* hv = far->dvec + 3 * pj;
        if (phi == 1 && phj == 2) {
          hbe_t* h = (hbe_t*)dyn_push(&hbonds[i]);
          h->nbr = j; h->scl = 1.0; h->d = d; memcpy(h->dvec, hv, sizeof h->dvec);
        } else if (j < n && phi == 2 && phj == 1) {
          hbe_t* h = (hbe_t*)dyn_push(&hbonds[j]);
          h->nbr = i; h->scl = -1.0; h->d = d; memcpy(h->dvec, hv, sizeof h->dvec);
        }
      }
      if (!(d <= ctl->bond_cut)) continue;
      /* terms::bo_prime, include/reaxmetal/terms.hpp:50-56 */
      const int s_ok = SB(ti, SB_R_S) > 0.0 && SB(tj, SB_R_S) > 0.0;
      const int pi_ok = SB(ti, SB_R_PI) > 0.0 && SB(tj, SB_R_PI) > 0.0;
      const int pp_ok = SB(ti, SB_R_PI_PI) > 0.0 && SB(tj, SB_R_PI_PI) > 0.0;
      double C12 = 0, C34 = 0, C56 = 0, BO_s = 0, BO_pi = 0, BO_pi2 = 0;
      if (s_ok) { C12 = TB(ti, tj, TB_P_BO1) * pow(d / TB(ti, tj, TB_R_S), TB(ti, tj, TB_P_BO2)); BO_s = (1.0 + bo_cut) * exp(C12); }
      if (pi_ok) { C34 = TB(ti, tj, TB_P_BO3) * pow(d / TB(ti, tj, TB_R_P), TB(ti, tj, TB_P_BO4)); BO_pi = exp(C34); }
      if (pp_ok) { C56 = TB(ti, tj, TB_P_BO5) * pow(d / TB(ti, tj, TB_R_PP), TB(ti, tj, TB_P_BO6)); BO_pi2 = exp(C56); }
      const double BOt = BO_s + BO_pi + BO_pi2;
      if (!(BOt >= bo_cut)) continue;
      bond_t* bi = (bond_t*)dyn_push(&bonds[i]);
      const int sym_i = bonds[j].n;  /* index the partner entry will get */
      bond_t* bj = (bond_t*)dyn_push(&bonds[j]);
      bi = &DYN_AT(bonds[i], bond_t, bonds[i].n - 1);  /* bonds[i] may have moved if i == j (never: j > i) */
      bi->nbr = j; bj->nbr = i;
      bi->sym = sym_i; bj->sym = bonds[i].n - 1;
      bi->d = bj->d = d;
      const double* dv = far->dvec + 3 * pj;
      for (int c = 0; c < 3; ++c) { bi->dvec[c] = dv[c]; bj->dvec[c] = -dv[c]; }
      bi->BO = bj->BO = BOt;
      bi->BO_s = bj->BO_s = BO_s; bi->BO_pi = bj->BO_pi = BO_pi; bi->BO_pi2 = bj->BO_pi2 = BO_pi2;
      const double rr2 = 1.0 / (d * d);
      const double Cln_s = TB(ti, tj, TB_P_BO2) * C12 * rr2, Cln_pi = TB(ti, tj, TB_P_BO4) * C34 * rr2, Cln_pi2 = TB(ti, tj, TB_P_BO6) * C56 * rr2;
      for (int c = 0; c < 3; ++c) {
        bi->dln_s[c] = -bi->BO_s * Cln_s * bi->dvec[c];
        bi->dln_pi[c] = -bi->BO_pi * Cln_pi * bi->dvec[c];
        bi->dln_pi2[c] = -bi->BO_pi2 * Cln_pi2 * bi->dvec[c];
        bj->dln_s[c] = -bi->dln_s[c];
        bj->dln_pi[c] = -bi->dln_pi[c];
        bj->dln_pi2[c] = -bi->dln_pi2[c];
        bi->dBOp[c] = -(bi->BO_s * Cln_s + bi->BO_pi * Cln_pi + bi->BO_pi2 * Cln_pi2) * bi->dvec[c];
        bj->dBOp[c] = -bi->dBOp[c];
        dDeltap_self[3 * i + c] += bi->dBOp[c];
        dDeltap_self[3 * j + c] += bj->dBOp[c];
      }
      bi->BO_s -= bo_cut; bi->BO -= bo_cut; bj->BO_s -= bo_cut; bj->BO -= bo_cut;
      total_bo[i] += bi->BO;
      total_bo[j] += bj->BO;
    }
  }

  /* ---- BO: corrected bond orders (src/cpu/bonded.cpp:164-196; terms::bo_correct terms.hpp:66-132). The corrected
   * values of a bond are computed from its lower-index end and copied to the other (the reference's bond_mark rule
   * only decides whether the unused coefficients of the upper end are also computed). */
  for (int i = 0; i < N; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    Deltap[i] = total_bo[i] - SB(ti, SB_VALENCY);
    Deltap_boc[i] = total_bo[i] - SB(ti, SB_VALENCY_VAL);
    total_bo[i] = 0;
  }
  for (int i = 0; i < N; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    for (int k = 0; k < bonds[i].n; ++k) {
      bond_t* b = &DYN_AT(bonds[i], bond_t, k);
      const int j = b->nbr, tj = a->type[j];
      if (tj < 0) continue;
      if (i < j) {
        const double ovc = TB(ti, tj, TB_OVC), v13cor = TB(ti, tj, TB_V13COR);
        const double val_i = SB(ti, SB_VALENCY), val_j = SB(tj, SB_VALENCY);
        const double BO = b->BO, BO_pi = b->BO_pi, BO_pi2 = b->BO_pi2;
        if (ovc < 0.001 && v13cor < 0.001) {
          b->C1dbo = 1.0; b->C2dbo = 0; b->C3dbo = 0;
          b->C1dbopi = 1.0; b->C2dbopi = b->C3dbopi = b->C4dbopi = 0;
          b->C1dbopi2 = 1.0; b->C2dbopi2 = b->C3dbopi2 = b->C4dbopi2 = 0;
        } else {
          double f1, Cf1_ij, Cf1_ji, f4, f5, f4f5, Cf45_ij, Cf45_ji;
          if (ovc >= 0.001) {
            const double exp_p1i = safe_exp(-p_boc1 * Deltap[i]), exp_p2i = safe_exp(-p_boc2 * Deltap[i]);
            const double exp_p1j = safe_exp(-p_boc1 * Deltap[j]), exp_p2j = safe_exp(-p_boc2 * Deltap[j]);
            const double f2 = exp_p1i + exp_p1j;
            const double f3 = -1.0 / p_boc2 * log(0.5 * (exp_p2i + exp_p2j));
            f1 = 0.5 * ((val_i + f2) / (val_i + f2 + f3) + (val_j + f2) / (val_j + f2 + f3));
            const double temp = f2 + f3;
            const double u1_ij = val_i + temp, u1_ji = val_j + temp;
            const double Cf1A_ij = 0.5 * f3 * (1.0 / (u1_ij * u1_ij) + 1.0 / (u1_ji * u1_ji));
            const double Cf1B_ij = -0.5 * ((u1_ij - f3) / (u1_ij * u1_ij) + (u1_ji - f3) / (u1_ji * u1_ji));
            Cf1_ij = 0.50 * (-p_boc1 * exp_p1i / u1_ij - ((val_i + f2) / (u1_ij * u1_ij)) * (-p_boc1 * exp_p1i + exp_p2i / (exp_p2i + exp_p2j)) +
                             -p_boc1 * exp_p1i / u1_ji - ((val_j + f2) / (u1_ji * u1_ji)) * (-p_boc1 * exp_p1i + exp_p2i / (exp_p2i + exp_p2j)));
            Cf1_ji = -Cf1A_ij * p_boc1 * exp_p1j + Cf1B_ij * exp_p2j / (exp_p2i + exp_p2j);
          } else {
            f1 = 1.0; Cf1_ij = Cf1_ji = 0.0;
          }
          if (v13cor >= 0.001) {
            const double p_boc3 = TB(ti, tj, TB_P_BOC3), p_boc4 = TB(ti, tj, TB_P_BOC4), p_boc5 = TB(ti, tj, TB_P_BOC5);
            const double exp_f4 = safe_exp(-(p_boc4 * (BO * BO) - Deltap_boc[i]) * p_boc3 + p_boc5);
            const double exp_f5 = safe_exp(-(p_boc4 * (BO * BO) - Deltap_boc[j]) * p_boc3 + p_boc5);
            f4 = 1.0 / (1.0 + exp_f4);
            f5 = 1.0 / (1.0 + exp_f5);
            f4f5 = f4 * f5;
            Cf45_ij = -f4 * exp_f4;
            Cf45_ji = -f5 * exp_f5;
          } else {
            f4 = f5 = f4f5 = 1.0; Cf45_ij = Cf45_ji = 0.0;
          }
          const double p_boc3 = TB(ti, tj, TB_P_BOC3), p_boc4 = TB(ti, tj, TB_P_BOC4);
          const double A0 = f1 * f4f5;
          const double A1 = -2 * p_boc3 * p_boc4 * BO * (Cf45_ij + Cf45_ji);
          const double A2_ij = Cf1_ij / f1 + p_boc3 * Cf45_ij;
          const double A2_ji = Cf1_ji / f1 + p_boc3 * Cf45_ji;
          const double A3_ij = A2_ij + Cf1_ij / f1;
          const double A3_ji = A2_ji + Cf1_ji / f1;
          b->BO = BO * A0;
          b->BO_pi = BO_pi * A0 * f1;
          b->BO_pi2 = BO_pi2 * A0 * f1;
          b->BO_s = b->BO - (b->BO_pi + b->BO_pi2);
          b->C1dbo = A0 + b->BO * A1;
          b->C2dbo = b->BO * A2_ij;
          b->C3dbo = b->BO * A2_ji;
          b->C1dbopi = f1 * f1 * f4 * f5;
          b->C2dbopi = b->BO_pi * A1;
          b->C3dbopi = b->BO_pi * A3_ij;
          b->C4dbopi = b->BO_pi * A3_ji;
          b->C1dbopi2 = f1 * f1 * f4 * f5;
          b->C2dbopi2 = b->BO_pi2 * A1;
          b->C3dbopi2 = b->BO_pi2 * A3_ij;
          b->C4dbopi2 = b->BO_pi2 * A3_ji;
        }
        if (b->BO < 1e-10) b->BO = 0;
        if (b->BO_s < 1e-10) b->BO_s = 0;
        if (b->BO_pi < 1e-10) b->BO_pi = 0;
        if (b->BO_pi2 < 1e-10) b->BO_pi2 = 0;
      } else {
        const bond_t* s = &DYN_AT(bonds[j], bond_t, b->sym);
        b->BO = s->BO; b->BO_s = s->BO_s; b->BO_pi = s->BO_pi; b->BO_pi2 = s->BO_pi2;
      }
      total_bo[i] += b->BO;
    }
  }
  /* atom quantities (src/cpu/bonded.cpp:197-204; terms.hpp:141-164) */
  for (int j = 0; j < N; ++j) {
    const int tj = a->type[j];
    if (tj < 0) continue;
    aq_t* q = &aq[j];
    const double valency = SB(tj, SB_VALENCY), valency_e = SB(tj, SB_VALENCY_E);
    q->Delta = total_bo[j] - valency;
    q->Delta_e = total_bo[j] - valency_e;
    q->Delta_boc = total_bo[j] - SB(tj, SB_VALENCY_BOC);
    q->Delta_val = total_bo[j] - SB(tj, SB_VALENCY_VAL);
    const double half_trunc = (double)(int)(q->Delta_e / 2.0);
    q->vlpex = q->Delta_e - 2.0 * half_trunc;
    const double explp1 = exp(-p_lp1 * ((2.0 + q->vlpex) * (2.0 + q->vlpex)));
    q->nlp = explp1 - half_trunc;
    q->Delta_lp = SB(tj, SB_NLP_OPT) - q->nlp;
    q->Clp = 2.0 * p_lp1 * explp1 * (2.0 + q->vlpex);
    q->dDelta_lp = q->Clp;
    if (SB(tj, SB_HEAVY) != 0.0) {
      q->nlp_temp = 0.5 * (valency_e - valency);
      q->Delta_lp_temp = SB(tj, SB_NLP_OPT) - q->nlp_temp;
      q->dDelta_lp_temp = 0.0;
    } else {
      q->nlp_temp = q->nlp;
      q->Delta_lp_temp = SB(tj, SB_NLP_OPT) - q->nlp_temp;
      q->dDelta_lp_temp = q->Clp;
    }
  }
  if (census) {
    for (int i = 0; i < n; ++i) {
      census[0 * n + i] = bonds[i].n;
      census[6 * n + i] = (int)(aq[i].Delta_e / 2.0);
    }
  }

  double e_bond = 0, e_lp = 0, e_ov = 0, e_un = 0, e_ang = 0, e_pen = 0, e_coa = 0, e_tor = 0, e_con = 0, e_hb = 0;
  /* ---- bond energy + triple-bond stabilisation (src/cpu/bonded.cpp:219-253; terms.hpp:170-195) */
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    for (int k = 0; k < bonds[i].n; ++k) {
      bond_t* b = &DYN_AT(bonds[i], bond_t, k);
      const int j = b->nbr;
      if (skip_by_tag(a, i, j)) continue;
      const int tj = a->type[j];
      if (ti < 0 || tj < 0) continue;
      const double p_be1 = TB(ti, tj, TB_P_BE1), p_be2 = TB(ti, tj, TB_P_BE2), De_s = TB(ti, tj, TB_DE_S);
      const double De_p = TB(ti, tj, TB_DE_P), De_pp = TB(ti, tj, TB_DE_PP);
      const double pow_BOs_be2 = b->BO_s == 0.0 ? 0.0 : pow(b->BO_s, p_be2);
      const double exp_be12 = exp(p_be1 * (1.0 - pow_BOs_be2));
      const double CEbo = -De_s * exp_be12 * (1.0 - p_be1 * p_be2 * pow_BOs_be2);
      e_bond += -De_s * b->BO_s * exp_be12 - De_p * b->BO_pi - De_pp * b->BO_pi2;
      b->Cdbo += CEbo;
      b->Cdbopi -= (CEbo + De_p);
      b->Cdbopi2 -= (CEbo + De_pp);
      if (b->BO >= 1.00 && TB(ti, tj, TB_TRIPLE_STAB) != 0.0) {
        const double BO = b->BO;
        const double exphu = exp(-gp7 * ((BO - 2.50) * (BO - 2.50)));
        const double exphua1 = exp(-gp3 * (total_bo[i] - BO));
        const double exphub1 = exp(-gp3 * (total_bo[j] - BO));
        const double exphuov = exp(gp4 * (aq[i].Delta + aq[j].Delta));
        const double hulpov = 1.0 / (1.0 + 25.0 * exphuov);
        e_bond += gp10 * exphu * hulpov * (exphua1 + exphub1);
        b->Cdbo += gp10 * exphu * hulpov * (exphua1 + exphub1) * (gp3 - 2.0 * gp7 * (BO - 2.50));
        CdDelta[i] += -gp10 * exphu * hulpov * (gp3 * exphua1 + 25.0 * gp4 * exphuov * hulpov * (exphua1 + exphub1));
        CdDelta[j] += -gp10 * exphu * hulpov * (gp3 * exphub1 + 25.0 * gp4 * exphuov * hulpov * (exphua1 + exphub1));
      }
    }
  }

  /* ---- lone pair + C2 correction (src/cpu/bonded.cpp:257-281; terms.hpp:201-223) */
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    const int active = bonds[i].n > 0 || ctl->enobonds;
    if (active) {
      const double p_lp2 = SB(ti, SB_P_LP2), Delta_lp = aq[i].Delta_lp;
      const double expvd2 = safe_exp(-75 * Delta_lp);
      const double inv = 1.0 / (1.0 + expvd2);
      e_lp += p_lp2 * Delta_lp * inv;
      const double dElp = p_lp2 * inv + 75 * p_lp2 * Delta_lp * expvd2 * (inv * inv);
      CdDelta[i] += dElp * aq[i].dDelta_lp;
    }
    if (c2_gate && SB(ti, SB_C2SPECIES) != 0.0) {
      for (int k = 0; k < bonds[i].n; ++k) {
        bond_t* b = &DYN_AT(bonds[i], bond_t, k);
        const int tj = a->type[b->nbr];
        if (tj < 0 || SB(tj, SB_C2SPECIES) == 0.0) continue;
        const double Di = aq[i].Delta;
        const double vov3 = b->BO - Di - 0.040 * pow(Di, 4.);
        if (vov3 > 3.) {
          const double dd = vov3 - 3.0;
          e_lp += p_lp3 * (dd * dd);
          b->Cdbo += 2. * p_lp3 * (vov3 - 3.);
          CdDelta[i] += 2. * p_lp3 * (vov3 - 3.) * (-1. - 0.16 * pow(Di, 3.));
        }
      }
    }
  }
  /* ---- over / under coordination (src/cpu/bonded.cpp:282-318; terms.hpp:231-260) */
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    const double dfvl = SB(ti, SB_HEAVY) != 0.0 ? 0.0 : 1.0;
    double sum1 = 0, sum2 = 0;
    for (int k = 0; k < bonds[i].n; ++k) {
      const bond_t* b = &DYN_AT(bonds[i], bond_t, k);
      const int j = b->nbr, tj = a->type[j];
      if (tj < 0) continue;
      sum1 += TB(ti, tj, TB_P_OVUN1) * TB(ti, tj, TB_DE_S) * b->BO;
      sum2 += (aq[j].Delta - dfvl * aq[j].Delta_lp_temp) * (b->BO_pi + b->BO_pi2);
    }
    const int under_active = bonds[i].n > 0 || ctl->enobonds;
    const double Delta = aq[i].Delta, Delta_lp_temp = aq[i].Delta_lp_temp, dDelta_lp = aq[i].dDelta_lp;
    const double valency = SB(ti, SB_VALENCY), p_ovun2 = SB(ti, SB_P_OVUN2), p_ovun5 = SB(ti, SB_P_OVUN5);
    const double exp_ovun1 = p_ovun3 * safe_exp(p_ovun4 * sum2);
    const double inv_exp_ovun1 = 1.0 / (1 + exp_ovun1);
    const double Delta_lpcorr = Delta - (dfvl * Delta_lp_temp) * inv_exp_ovun1;
    const double exp_ovun2 = safe_exp(p_ovun2 * Delta_lpcorr);
    const double inv_exp_ovun2 = 1.0 / (1.0 + exp_ovun2);
    const double DlpVi = 1.0 / (Delta_lpcorr + valency + 1e-8);
    const double CEover1 = Delta_lpcorr * DlpVi * inv_exp_ovun2;
    e_ov += sum1 * CEover1;
    const double CEover2 = sum1 * DlpVi * inv_exp_ovun2 * (1.0 - Delta_lpcorr * (DlpVi + p_ovun2 * exp_ovun2 * inv_exp_ovun2));
    const double CEover3 = CEover2 * (1.0 - dfvl * dDelta_lp * inv_exp_ovun1);
    const double CEover4 = CEover2 * (dfvl * Delta_lp_temp) * p_ovun4 * exp_ovun1 * (inv_exp_ovun1 * inv_exp_ovun1);
    const double exp_ovun2n = safe_exp(-p_ovun2 * Delta_lpcorr);
    const double exp_ovun6 = safe_exp(p_ovun6 * Delta_lpcorr);
    const double exp_ovun8 = p_ovun7 * safe_exp(p_ovun8 * sum2);
    const double inv_exp_ovun2n = 1.0 / (1.0 + exp_ovun2n);
    const double inv_exp_ovun8 = 1.0 / (1.0 + exp_ovun8);
    const double eun = under_active ? -p_ovun5 * (1.0 - exp_ovun6) * inv_exp_ovun2n * inv_exp_ovun8 : 0.0;
    const double CEunder1 = inv_exp_ovun2n * (p_ovun5 * p_ovun6 * exp_ovun6 * inv_exp_ovun8 + p_ovun2 * eun * exp_ovun2n);
    const double CEunder2 = -eun * p_ovun8 * exp_ovun8 * inv_exp_ovun8;
    const double CEunder3 = CEunder1 * (1.0 - dfvl * dDelta_lp * inv_exp_ovun1);
    const double CEunder4 = CEunder1 * (dfvl * Delta_lp_temp) * p_ovun4 * exp_ovun1 * (inv_exp_ovun1 * inv_exp_ovun1) + CEunder2;
    if (under_active) e_un += eun;
    CdDelta[i] += CEover3;
    if (under_active) CdDelta[i] += CEunder3;
    for (int k = 0; k < bonds[i].n; ++k) {
      bond_t* b = &DYN_AT(bonds[i], bond_t, k);
      const int j = b->nbr, tj = a->type[j];
      b->Cdbo += CEover1 * TB(ti, tj, TB_P_OVUN1) * TB(ti, tj, TB_DE_S);
      const double pis = b->BO_pi + b->BO_pi2;
      const double dj = aq[j].Delta - dfvl * aq[j].Delta_lp_temp;
      CdDelta[j] += CEover4 * (1.0 - dfvl * aq[j].dDelta_lp) * pis;
      b->Cdbopi += CEover4 * dj;
      b->Cdbopi2 += CEover4 * dj;
      CdDelta[j] += CEunder4 * (1.0 - dfvl * aq[j].dDelta_lp) * pis;
      b->Cdbopi += CEunder4 * dj;
      b->Cdbopi2 += CEunder4 * dj;
    }
  }

  /* ---- valence angle / penalty / coalition; three-body lists (src/cpu/bonded.cpp:321-474) */
  dyn** thb = (dyn**)calloc((size_t)N, sizeof(dyn*));
  for (int j = 0; j < N; ++j) {
    thb[j] = (dyn*)calloc((size_t)(bonds[j].n > 0 ? bonds[j].n : 1), sizeof(dyn));
    for (int k = 0; k < bonds[j].n; ++k) thb[j][k].sz = (int)sizeof(thb_t);
  }
  {
    const double p_val6 = gp[14], p_val8 = gp[33], p_val9 = gp[16], p_val10 = gp[17];
    for (int j = 0; j < N; ++j) {
      const int type_j = a->type[j];
      if (type_j < 0) continue;
      const int nb = bonds[j].n;
      bond_t* bj = (bond_t*)bonds[j].p;
      const double p_val3 = SB(type_j, SB_P_VAL3), p_val5 = SB(type_j, SB_P_VAL5);
      double SBOp = 0, prod_SBO = 1;
      for (int t = 0; t < nb; ++t) {
        SBOp += (bj[t].BO_pi + bj[t].BO_pi2);
        double temp = bj[t].BO * bj[t].BO;
        temp *= temp;
        temp *= temp;
        prod_SBO *= exp(-temp);
      }
      double vlpadj, dSBO2;
      if (aq[j].vlpex >= 0) { vlpadj = 0; dSBO2 = prod_SBO - 1; }
      else { vlpadj = aq[j].nlp; dSBO2 = (prod_SBO - 1) * (1 - p_val8 * aq[j].dDelta_lp); }
      const double Dboc = aq[j].Delta_boc;
      const double SBO = SBOp + (1 - prod_SBO) * (-Dboc - p_val8 * vlpadj);
      const double dSBO1 = -8 * prod_SBO * (Dboc + p_val8 * vlpadj);
      double SBO2, CSBO2;
      if (SBO <= 0) { SBO2 = 0; CSBO2 = 0; }
      else if (SBO > 0 && SBO <= 1) { SBO2 = pow(SBO, p_val9); CSBO2 = p_val9 * pow(SBO, p_val9 - 1); }
      else if (SBO > 1 && SBO < 2) { SBO2 = 2 - pow(2 - SBO, p_val9); CSBO2 = p_val9 * pow(2 - SBO, p_val9 - 1); }
      else { SBO2 = 2; CSBO2 = 0; }
      const double expval6 = exp(p_val6 * Dboc);
      if (census && j < n) census[5 * n + j] = SBO <= 0 ? 0 : (SBO <= 1 ? 1 : (SBO < 2 ? 2 : 3));

      for (int pi = 0; pi < nb; ++pi) {
        bond_t* bij = &bj[pi];
        const double BOA_ij = bij->BO - thb_cut;
        if (!(BOA_ij > 0.0 && (j < n || bij->nbr < n))) continue;
        const int i = bij->nbr, type_i = a->type[i];
        dyn* list_i = &thb[j][pi];
        for (int pk = 0; pk < pi; ++pk) {
          for (int u = 0; u < thb[j][pk].n; ++u) {
            const thb_t* kji = &DYN_AT(thb[j][pk], thb_t, u);
            if (kji->thb == i) {
              thb_t* t = (thb_t*)dyn_push(list_i);
              t->thb = bj[pk].nbr; t->pthb = pk; t->theta = kji->theta;
              memcpy(t->dcos_di, kji->dcos_dk, sizeof t->dcos_di);
              memcpy(t->dcos_dj, kji->dcos_dj, sizeof t->dcos_dj);
              memcpy(t->dcos_dk, kji->dcos_di, sizeof t->dcos_dk);
              break;
            }
          }
        }
        for (int pk = pi + 1; pk < nb; ++pk) {
          bond_t* bjk = &bj[pk];
          const double BOA_jk = bjk->BO - thb_cut;
          const int k = bjk->nbr, type_k = a->type[k];
          thb_t* t = (thb_t*)dyn_push(list_i);
          double theta, cos_theta;
          calc_theta(bij->dvec, bij->d, bjk->dvec, bjk->d, &theta, &cos_theta);
          calc_dcos(bij->dvec, bij->d, bjk->dvec, bjk->d, t->dcos_di, t->dcos_dj, t->dcos_dk);
          t->thb = k; t->pthb = pk; t->theta = theta;
          const thb_t tt = *t;  /* list_i may grow no further inside this iteration */
          double sin_theta = sin(theta);
          if (sin_theta < 1.0e-5) sin_theta = 1.0e-5;
          if (!((j < n) && (BOA_jk > 0.0) && (bij->BO > thb_cut) && (bjk->BO > thb_cut) && (bij->BO * bjk->BO > thb_cutsq))) continue;
          if (census) census[1 * n + j]++;
          const size_t key = ((size_t)type_i * (size_t)ff->nt + (size_t)type_j) * (size_t)ff->nt + (size_t)type_k;
          for (int sidx = 0; sidx < ff->thb_n[key]; ++sidx) {
            const double* th = ff->thb + (key * RXO_MAX_THB_SETS + (size_t)sidx) * TH_NFIELDS;
            if (!(fabs(th[TH_P_VAL1]) > 0.001)) continue;
            const double p_val1 = th[TH_P_VAL1], p_val2 = th[TH_P_VAL2], p_val4 = th[TH_P_VAL4], p_val7 = th[TH_P_VAL7];
            const double theta_00 = th[TH_THETA_00];
            const double exp3ij = exp(-p_val3 * pow(BOA_ij, p_val4));
            const double f7_ij = 1.0 - exp3ij;
            const double Cf7ij = p_val3 * p_val4 * pow(BOA_ij, p_val4 - 1.0) * exp3ij;
            const double exp3jk = exp(-p_val3 * pow(BOA_jk, p_val4));
            const double f7_jk = 1.0 - exp3jk;
            const double Cf7jk = p_val3 * p_val4 * pow(BOA_jk, p_val4 - 1.0) * exp3jk;
            const double expval7 = exp(-p_val7 * Dboc);
            const double trm8 = 1.0 + expval6 + expval7;
            const double f8_Dj = p_val5 - ((p_val5 - 1.0) * (2.0 + expval6) / trm8);
            const double Cf8j = ((1.0 - p_val5) / (trm8 * trm8)) * (p_val6 * expval6 * trm8 - (2.0 + expval6) * (p_val6 * expval6 - p_val7 * expval7));
            double theta_0 = 180.0 - theta_00 * (1.0 - exp(-p_val10 * (2.0 - SBO2)));
            theta_0 = theta_0 * CONST_PI / 180.0;
            const double expval2theta = exp(-p_val2 * ((theta_0 - theta) * (theta_0 - theta)));
            const double expval12theta = p_val1 >= 0 ? p_val1 * (1.0 - expval2theta) : p_val1 * -expval2theta;
            const double CEval1 = Cf7ij * f7_jk * f8_Dj * expval12theta;
            const double CEval2 = Cf7jk * f7_ij * f8_Dj * expval12theta;
            const double CEval3 = Cf8j * f7_ij * f7_jk * expval12theta;
            const double CEval4 = -2.0 * p_val1 * p_val2 * f7_ij * f7_jk * f8_Dj * expval2theta * (theta_0 - theta);
            const double Ctheta_0 = p_val10 * (theta_00 * CONST_PI / 180.0) * exp(-p_val10 * (2.0 - SBO2));
            const double CEval5 = -CEval4 * Ctheta_0 * CSBO2;
            const double CEval6 = CEval5 * dSBO1;
            const double CEval7 = CEval5 * dSBO2;
            const double CEval8 = -CEval4 / sin_theta;
            e_ang += f7_ij * f7_jk * f8_Dj * expval12theta;
            /* penalty */
            const double p_pen1 = th[TH_P_PEN1], p_pen2 = gp[19], p_pen3 = gp[20], p_pen4 = gp[21];
            const double exp_pen2ij = exp(-p_pen2 * ((BOA_ij - 2.0) * (BOA_ij - 2.0)));
            const double exp_pen2jk = exp(-p_pen2 * ((BOA_jk - 2.0) * (BOA_jk - 2.0)));
            const double exp_pen3 = exp(-p_pen3 * aq[j].Delta);
            const double exp_pen4 = exp(p_pen4 * aq[j].Delta);
            const double trm_pen34 = 1.0 + exp_pen3 + exp_pen4;
            const double f9_Dj = (2.0 + exp_pen3) / trm_pen34;
            const double Cf9j = (-p_pen3 * exp_pen3 * trm_pen34 - (2.0 + exp_pen3) * (-p_pen3 * exp_pen3 + p_pen4 * exp_pen4)) / (trm_pen34 * trm_pen34);
            const double e_pen_t = p_pen1 * f9_Dj * exp_pen2ij * exp_pen2jk;
            e_pen += e_pen_t;
            const double CEpen1 = e_pen_t * Cf9j / f9_Dj;
            const double tmp = -2.0 * p_pen2 * e_pen_t;
            const double CEpen2 = tmp * (BOA_ij - 2.0), CEpen3 = tmp * (BOA_jk - 2.0);
            /* coalition */
            const double p_coa1 = th[TH_P_COA1], p_coa2 = gp[2], p_coa3 = gp[38], p_coa4 = gp[30];
            const double exp_coa2 = exp(p_coa2 * aq[j].Delta_val);
            const double dti = total_bo[i] - BOA_ij, dtk = total_bo[k] - BOA_jk;
            const double e_coa_t = p_coa1 / (1. + exp_coa2) * exp(-p_coa3 * (dti * dti)) * exp(-p_coa3 * (dtk * dtk)) *
                                   exp(-p_coa4 * ((BOA_ij - 1.5) * (BOA_ij - 1.5))) * exp(-p_coa4 * ((BOA_jk - 1.5) * (BOA_jk - 1.5)));
            e_coa += e_coa_t;
            const double CEcoa1 = -2 * p_coa4 * (BOA_ij - 1.5) * e_coa_t;
            const double CEcoa2 = -2 * p_coa4 * (BOA_jk - 1.5) * e_coa_t;
            const double CEcoa3 = -p_coa2 * exp_coa2 * e_coa_t / (1 + exp_coa2);
            const double CEcoa4 = -2 * p_coa3 * dti * e_coa_t;
            const double CEcoa5 = -2 * p_coa3 * dtk * e_coa_t;
            bij->Cdbo += (CEval1 + CEpen2 + (CEcoa1 - CEcoa4));
            bjk->Cdbo += (CEval2 + CEpen3 + (CEcoa2 - CEcoa5));
            CdDelta[j] += ((CEval3 + CEval7) + CEpen1 + CEcoa3);
            CdDelta[i] += CEcoa4;
            CdDelta[k] += CEcoa5;
            for (int u = 0; u < nb; ++u) {
              const double bo = bj[u].BO;
              const double cube = bo * bo * bo;
              bj[u].Cdbo += (CEval6 * (cube * cube * bo));
              bj[u].Cdbopi += CEval5;
              bj[u].Cdbopi2 += CEval5;
            }
            axpy3(f + 3 * i, CEval8, tt.dcos_di);
            axpy3(f + 3 * j, CEval8, tt.dcos_dj);
            axpy3(f + 3 * k, CEval8, tt.dcos_dk);
          }
        }
      }
    }
  }

  /* ---- torsion + 4-body conjugation (src/cpu/bonded.cpp:476-652) */
  {
    const double p_tor2 = gp[23], p_tor3 = gp[24], p_tor4 = gp[25], p_cot2 = gp[27];
    for (int j = 0; j < n; ++j) {
      const int type_j = a->type[j];
      const double Delta_j = aq[j].Delta_boc;
      for (int pk = 0; pk < bonds[j].n; ++pk) {
        bond_t* bjk = &DYN_AT(bonds[j], bond_t, pk);
        const int k = bjk->nbr;
        const double BOA_jk = bjk->BO - thb_cut;
        if (skip_by_tag(a, j, k)) continue;
        if (!(bjk->BO > thb_cut && thb[j][pk].n > 0)) continue;
        const int pj = bjk->sym;
        if (thb[k][pj].n == 0) continue;
        const int type_k = a->type[k];
        const double Delta_k = aq[k].Delta_boc;
        const double r_jk = bjk->d;
        const double exp_tor2_jk = exp(-p_tor2 * BOA_jk);
        const double exp_cot2_jk = exp(-p_cot2 * ((BOA_jk - 1.5) * (BOA_jk - 1.5)));
        const double exp_tor3_DjDk = exp(-p_tor3 * (Delta_j + Delta_k));
        const double exp_tor4_DjDk = exp(p_tor4 * (Delta_j + Delta_k));
        const double exp_tor34_inv = 1.0 / (1.0 + exp_tor3_DjDk + exp_tor4_DjDk);
        const double f11_DjDk = (2.0 + exp_tor3_DjDk) * exp_tor34_inv;
        for (int u = 0; u < thb[j][pk].n; ++u) {
          const thb_t* p_ijk = &DYN_AT(thb[j][pk], thb_t, u);
          bond_t* bij = &DYN_AT(bonds[j], bond_t, p_ijk->pthb);
          if (!(bij->BO > thb_cut)) continue;
          const int i = p_ijk->thb, type_i = a->type[i];
          const double r_ij = bij->d;
          const double BOA_ij = bij->BO - thb_cut;
          const double theta_ijk = p_ijk->theta;
          const double sin_ijk = sin(theta_ijk), cos_ijk = cos(theta_ijk);
          double tan_ijk_i;
          if (sin_ijk >= 0 && sin_ijk <= MIN_SINE) tan_ijk_i = cos_ijk / MIN_SINE;
          else if (sin_ijk <= 0 && sin_ijk >= -MIN_SINE) tan_ijk_i = cos_ijk / -MIN_SINE;
          else tan_ijk_i = cos_ijk / sin_ijk;
          const double exp_tor2_ij = exp(-p_tor2 * BOA_ij);
          const double exp_cot2_ij = exp(-p_cot2 * ((BOA_ij - 1.5) * (BOA_ij - 1.5)));
          for (int v = 0; v < thb[k][pj].n; ++v) {
            const thb_t* p_jkl = &DYN_AT(thb[k][pj], thb_t, v);
            const int l = p_jkl->thb;
            bond_t* bkl = &DYN_AT(bonds[k], bond_t, p_jkl->pthb);
            const int type_l = a->type[l];
            const size_t key4 = (((size_t)type_i * (size_t)ff->nt + (size_t)type_j) * (size_t)ff->nt + (size_t)type_k) * (size_t)ff->nt + (size_t)type_l;
            if (!(i != l && ff->fbp_on[key4] && bkl->BO > thb_cut && bij->BO * bjk->BO * bkl->BO > thb_cut)) continue;
            const double* fb = ff->fbp + key4 * FB_NFIELDS;
            if (census) census[2 * n + j]++;
            const double r_kl = bkl->d;
            const double BOA_kl = bkl->BO - thb_cut;
            const double theta_jkl = p_jkl->theta;
            const double sin_jkl = sin(theta_jkl), cos_jkl = cos(theta_jkl);
            double tan_jkl_i;
            if (sin_jkl >= 0 && sin_jkl <= MIN_SINE) tan_jkl_i = cos_jkl / MIN_SINE;
            else if (sin_jkl <= 0 && sin_jkl >= -MIN_SINE) tan_jkl_i = cos_jkl / -MIN_SINE;
            else tan_jkl_i = cos_jkl / sin_jkl;
            const double* xi = a->x + 3 * i;
            const double* xl = a->x + 3 * l;
            const double dvec_li[3] = {xi[0] - xl[0], xi[1] - xl[1], xi[2] - xl[2]};
            const double r_li = sqrt(dot3(dvec_li, dvec_li));
            /* Calculate_Omega (src/cpu/bonded.cpp:544-586) */
            double dco_i[3], dco_j[3], dco_k[3], dco_l[3], omega;
            {
              double s_ijk = sin(p_ijk->theta), c_ijk = cos(p_ijk->theta), s_jkl = sin(p_jkl->theta), c_jkl = cos(p_jkl->theta);
              if (s_ijk >= 0 && s_ijk <= MIN_SINE) s_ijk = MIN_SINE; else if (s_ijk <= 0 && s_ijk >= -MIN_SINE) s_ijk = -MIN_SINE;
              if (s_jkl >= 0 && s_jkl <= MIN_SINE) s_jkl = MIN_SINE; else if (s_jkl <= 0 && s_jkl >= -MIN_SINE) s_jkl = -MIN_SINE;
              const double* dij = bij->dvec;
              const double* djk = bjk->dvec;
              const double* dkl = bkl->dvec;
              const double unnorm_cos_omega = -dot3(dij, djk) * dot3(djk, dkl) + (r_jk * r_jk) * dot3(dij, dkl);
              double cjkkl[3];
              cross3(djk, dkl, cjkkl);
              const double unnorm_sin_omega = -r_jk * dot3(dij, cjkkl);
              omega = atan2(unnorm_sin_omega, unnorm_cos_omega);
              const double htra = r_ij + c_ijk * (r_kl * c_jkl - r_jk);
              const double htrb = r_jk - r_ij * c_ijk - r_kl * c_jkl;
              const double htrc = r_kl + c_jkl * (r_ij * c_ijk - r_jk);
              const double hthd = r_ij * s_ijk * (r_jk - r_kl * c_jkl);
              const double hthe = r_kl * s_jkl * (r_jk - r_ij * c_ijk);
              const double hnra = r_kl * s_ijk * s_jkl;
              const double hnrc = r_ij * s_ijk * s_jkl;
              const double hnhd = r_ij * r_kl * c_ijk * s_jkl;
              const double hnhe = r_ij * r_kl * s_ijk * c_jkl;
              const double tel = (r_ij * r_ij) + (r_jk * r_jk) + (r_kl * r_kl) - (r_li * r_li) -
                                 2.0 * (r_ij * r_jk * c_ijk - r_ij * r_kl * c_ijk * c_jkl + r_jk * r_kl * c_jkl);
              const double poem = 2.0 * r_ij * r_kl * s_ijk * s_jkl;
              double arg = tel / poem;
              if (arg > 1.0) arg = 1.0;
              if (arg < -1.0) arg = -1.0;
              for (int c = 0; c < 3; ++c) {
                dco_i[c] = (htra - arg * hnra) / r_ij * dij[c] + -1. * dvec_li[c];
                dco_i[c] += -(hthd - arg * hnhd) / s_ijk * p_ijk->dcos_dk[c];
                dco_i[c] = 2.0 / poem * dco_i[c];
                dco_j[c] = -(htra - arg * hnra) / r_ij * dij[c] + -htrb / r_jk * djk[c];
                dco_j[c] += -(hthd - arg * hnhd) / s_ijk * p_ijk->dcos_dj[c];
                dco_j[c] += -(hthe - arg * hnhe) / s_jkl * p_jkl->dcos_di[c];
                dco_j[c] = 2.0 / poem * dco_j[c];
                dco_k[c] = -(htrc - arg * hnrc) / r_kl * dkl[c] + htrb / r_jk * djk[c];
                dco_k[c] += -(hthd - arg * hnhd) / s_ijk * p_ijk->dcos_di[c];
                dco_k[c] += -(hthe - arg * hnhe) / s_jkl * p_jkl->dcos_dj[c];
                dco_k[c] = 2.0 / poem * dco_k[c];
                dco_l[c] = (htrc - arg * hnrc) / r_kl * dkl[c] + 1. * dvec_li[c];
                dco_l[c] += -(hthe - arg * hnhe) / s_jkl * p_jkl->dcos_dk[c];
                dco_l[c] = 2.0 / poem * dco_l[c];
              }
            }
            const double cos_omega = cos(omega), cos2omega = cos(2. * omega), cos3omega = cos(3. * omega);
            const double V1 = fb[FB_V1], V2 = fb[FB_V2], V3 = fb[FB_V3], p_tor1 = fb[FB_P_TOR1], p_cot1 = fb[FB_P_COT1];
            const double exp_tor1 = exp(p_tor1 * ((2.0 - bjk->BO_pi - f11_DjDk) * (2.0 - bjk->BO_pi - f11_DjDk)));
            const double exp_tor2_kl = exp(-p_tor2 * BOA_kl);
            const double exp_cot2_kl = exp(-p_cot2 * ((BOA_kl - 1.5) * (BOA_kl - 1.5)));
            const double fn10 = (1.0 - exp_tor2_ij) * (1.0 - exp_tor2_jk) * (1.0 - exp_tor2_kl);
            const double CV = 0.5 * (V1 * (1.0 + cos_omega) + V2 * exp_tor1 * (1.0 - cos2omega) + V3 * (1.0 + cos3omega));
            e_tor += fn10 * sin_ijk * sin_jkl * CV;
            const double dfn11 = (-p_tor3 * exp_tor3_DjDk + (p_tor3 * exp_tor3_DjDk - p_tor4 * exp_tor4_DjDk) * (2.0 + exp_tor3_DjDk) * exp_tor34_inv) * exp_tor34_inv;
            const double CEtors1 = sin_ijk * sin_jkl * CV;
            const double CEtors2 = -fn10 * 2.0 * p_tor1 * V2 * exp_tor1 * (2.0 - bjk->BO_pi - f11_DjDk) * (1.0 - (cos_omega * cos_omega)) * sin_ijk * sin_jkl;
            const double CEtors3 = CEtors2 * dfn11;
            const double CEtors4 = CEtors1 * p_tor2 * exp_tor2_ij * (1.0 - exp_tor2_jk) * (1.0 - exp_tor2_kl);
            const double CEtors5 = CEtors1 * p_tor2 * (1.0 - exp_tor2_ij) * exp_tor2_jk * (1.0 - exp_tor2_kl);
            const double CEtors6 = CEtors1 * p_tor2 * (1.0 - exp_tor2_ij) * (1.0 - exp_tor2_jk) * exp_tor2_kl;
            const double cmn = -fn10 * CV;
            const double CEtors7 = cmn * sin_jkl * tan_ijk_i;
            const double CEtors8 = cmn * sin_ijk * tan_jkl_i;
            const double CEtors9 = fn10 * sin_ijk * sin_jkl * (0.5 * V1 - 2.0 * V2 * exp_tor1 * cos_omega + 1.5 * V3 * (cos2omega + 2.0 * (cos_omega * cos_omega)));
            const double fn12 = exp_cot2_ij * exp_cot2_jk * exp_cot2_kl;
            e_con += p_cot1 * fn12 * (1.0 + ((cos_omega * cos_omega) - 1.0) * sin_ijk * sin_jkl);
            const double Cconj = -2.0 * fn12 * p_cot1 * p_cot2 * (1.0 + ((cos_omega * cos_omega) - 1.0) * sin_ijk * sin_jkl);
            const double CEconj1 = Cconj * (BOA_ij - 1.5e0), CEconj2 = Cconj * (BOA_jk - 1.5e0), CEconj3 = Cconj * (BOA_kl - 1.5e0);
            const double CEconj4 = -p_cot1 * fn12 * ((cos_omega * cos_omega) - 1.0) * sin_jkl * tan_ijk_i;
            const double CEconj5 = -p_cot1 * fn12 * ((cos_omega * cos_omega) - 1.0) * sin_ijk * tan_jkl_i;
            const double CEconj6 = 2.0 * p_cot1 * fn12 * cos_omega * sin_ijk * sin_jkl;
            bjk->Cdbopi += CEtors2;
            CdDelta[j] += CEtors3;
            CdDelta[k] += CEtors3;
            bij->Cdbo += (CEtors4 + CEconj1);
            bjk->Cdbo += (CEtors5 + CEconj2);
            bkl->Cdbo += (CEtors6 + CEconj3);
            axpy3(f + 3 * i, CEtors7 + CEconj4, p_ijk->dcos_dk);
            axpy3(f + 3 * j, CEtors7 + CEconj4, p_ijk->dcos_dj);
            axpy3(f + 3 * k, CEtors7 + CEconj4, p_ijk->dcos_di);
            axpy3(f + 3 * j, CEtors8 + CEconj5, p_jkl->dcos_di);
            axpy3(f + 3 * k, CEtors8 + CEconj5, p_jkl->dcos_dj);
            axpy3(f + 3 * l, CEtors8 + CEconj5, p_jkl->dcos_dk);
            axpy3(f + 3 * i, CEtors9 + CEconj6, dco_i);
            axpy3(f + 3 * j, CEtors9 + CEconj6, dco_j);
            axpy3(f + 3 * k, CEtors9 + CEconj6, dco_k);
            axpy3(f + 3 * l, CEtors9 + CEconj6, dco_l);
          }
        }
      }
    }
  }

  /* ---- hydrogen bonds (src/cpu/bonded.cpp:654-715) */
  if (ctl->hbond_cut > 0) {
    int* hblist = (int*)malloc(sizeof(int) * 256);
    int hbcap = 256;
    for (int j = 0; j < n; ++j) {
      const int type_j = a->type[j];
      if (type_j < 0 || (int)SB(type_j, SB_P_HBOND) != 1) continue;
      int nh = 0;
      for (int pi = 0; pi < bonds[j].n; ++pi) {
        const bond_t* b = &DYN_AT(bonds[j], bond_t, pi);
        const int type_i = a->type[b->nbr];
        if (type_i < 0) continue;
        if ((int)SB(type_i, SB_P_HBOND) == 2 && b->BO >= HB_THRESHOLD) {
          if (nh == hbcap) { hbcap *= 2; hblist = (int*)realloc(hblist, sizeof(int) * (size_t)hbcap); }
          hblist[nh++] = pi;
        }
      }
      for (int u = 0; u < hbonds[j].n; ++u) {
        const hbe_t* hk = &DYN_AT(hbonds[j], hbe_t, u);
        const int k = hk->nbr, type_k = a->type[k];
        if (type_k < 0) continue;
        const double r_jk = hk->d;
        const double dvec_jk[3] = {hk->scl * hk->dvec[0], hk->scl * hk->dvec[1], hk->scl * hk->dvec[2]};
        for (int w = 0; w < nh; ++w) {
          bond_t* bij = &DYN_AT(bonds[j], bond_t, hblist[w]);
          const int i = bij->nbr;
          if (a->tag[i] == a->tag[k]) continue;
          const int type_i = a->type[i];
          if (type_i < 0) continue;
          const size_t key = ((size_t)type_i * (size_t)ff->nt + (size_t)type_j) * (size_t)ff->nt + (size_t)type_k;
          if (!ff->hbp_on[key]) continue;
          const double* hb = ff->hbp + key * HB_NFIELDS;
          if (hb[HB_R0] <= 0.0) continue;
          if (census) census[3 * n + j]++;
          double theta, cos_theta, dti[3], dtj[3], dtk[3];
          calc_theta(bij->dvec, bij->d, dvec_jk, r_jk, &theta, &cos_theta);
          calc_dcos(bij->dvec, bij->d, dvec_jk, r_jk, dti, dtj, dtk);
          const double sin_theta2 = sin(theta / 2.0);
          double sin_xhz4 = sin_theta2 * sin_theta2;
          sin_xhz4 *= sin_xhz4;
          const double cos_xhz1 = (1.0 - cos_theta);
          const double exp_hb2 = exp(-hb[HB_P_HB2] * bij->BO);
          const double exp_hb3 = exp(-hb[HB_P_HB3] * (hb[HB_R0] / r_jk + r_jk / hb[HB_R0] - 2.0));
          const double e_hb_t = hb[HB_P_HB1] * (1.0 - exp_hb2) * exp_hb3 * sin_xhz4;
          e_hb += e_hb_t;
          const double CEhb1 = hb[HB_P_HB1] * hb[HB_P_HB2] * exp_hb2 * exp_hb3 * sin_xhz4;
          const double CEhb2 = -hb[HB_P_HB1] / 2.0 * (1.0 - exp_hb2) * exp_hb3 * cos_xhz1;
          const double CEhb3 = -hb[HB_P_HB3] * (-hb[HB_R0] / (r_jk * r_jk) + 1.0 / hb[HB_R0]) * e_hb_t;
          bij->Cdbo += CEhb1;
          axpy3(f + 3 * i, +CEhb2, dti);
          axpy3(f + 3 * j, +CEhb2, dtj);
          axpy3(f + 3 * k, +CEhb2, dtk);
          axpy3(f + 3 * j, -CEhb3 / r_jk, dvec_jk);
          axpy3(f + 3 * k, +CEhb3 / r_jk, dvec_jk);
        }
      }
    }
    free(hblist);
  }

  /* ---- Add_dBond_to_Forces (src/cpu/bonded.cpp:717-766) */
  for (int i = 0; i < N; ++i) {
    for (int u = 0; u < bonds[i].n; ++u) {
      const bond_t* bij = &DYN_AT(bonds[i], bond_t, u);
      const int j = bij->nbr;
      if (!(i < j)) continue;
      const bond_t* bji = &DYN_AT(bonds[j], bond_t, bij->sym);
      double c = bij->Cdbo + bji->Cdbo;
      const double C1dbo = bij->C1dbo * c, C2dbo = bij->C2dbo * c, C3dbo = bij->C3dbo * c;
      c = bij->Cdbopi + bji->Cdbopi;
      const double C1dbopi = bij->C1dbopi * c, C2dbopi = bij->C2dbopi * c, C3dbopi = bij->C3dbopi * c, C4dbopi = bij->C4dbopi * c;
      c = bij->Cdbopi2 + bji->Cdbopi2;
      const double C1dbopi2 = bij->C1dbopi2 * c, C2dbopi2 = bij->C2dbopi2 * c, C3dbopi2 = bij->C3dbopi2 * c, C4dbopi2 = bij->C4dbopi2 * c;
      c = CdDelta[i] + CdDelta[j];
      const double C1dDelta = bij->C1dbo * c, C2dDelta = bij->C2dbo * c, C3dDelta = bij->C3dbo * c;
      double t[3];
      for (int cc = 0; cc < 3; ++cc) {
        t[cc] = (C1dbo + C1dDelta + C2dbopi + C2dbopi2) * bij->dBOp[cc];
        t[cc] += (C2dbo + C2dDelta + C3dbopi + C3dbopi2) * dDeltap_self[3 * i + cc];
        t[cc] += C1dbopi * bij->dln_pi[cc];
        t[cc] += C1dbopi2 * bij->dln_pi2[cc];
        f[3 * i + cc] += t[cc];
      }
      for (int cc = 0; cc < 3; ++cc) {
        t[cc] = -(C1dbo + C1dDelta + C2dbopi + C2dbopi2) * bij->dBOp[cc];
        t[cc] += (C3dbo + C3dDelta + C4dbopi + C4dbopi2) * dDeltap_self[3 * j + cc];
        t[cc] += -C1dbopi * bij->dln_pi[cc];
        t[cc] += -C1dbopi2 * bij->dln_pi2[cc];
        f[3 * j + cc] += t[cc];
      }
      for (int w = 0; w < bonds[i].n; ++w) {
        const bond_t* bk = &DYN_AT(bonds[i], bond_t, w);
        axpy3(f + 3 * bk->nbr, -(C2dbo + C2dDelta + C3dbopi + C3dbopi2), bk->dBOp);
      }
      for (int w = 0; w < bonds[j].n; ++w) {
        const bond_t* bk = &DYN_AT(bonds[j], bond_t, w);
        axpy3(f + 3 * bk->nbr, -(C3dbo + C3dDelta + C4dbopi + C4dbopi2), bk->dBOp);
      }
    }
  }

  e13[0] = e_bond; e13[1] = e_ov; e13[2] = e_un; e13[3] = e_lp; e13[4] = e_ang; e13[5] = e_pen; e13[6] = e_coa;
  e13[7] = e_hb; e13[8] = e_tor; e13[9] = e_con;
  long long nb_total = 0;
  for (int i = 0; i < N; ++i) nb_total += bonds[i].n;
  *nbonds = nb_total / 2;

  for (int j = 0; j < N; ++j) {
    for (int k = 0; k < bonds[j].n; ++k) free(thb[j][k].p);
    free(thb[j]);
    free(bonds[j].p);
    free(hbonds[j].p);
  }
  free(thb); free(bonds); free(hbonds); free(dDeltap_self); free(total_bo); free(Deltap); free(Deltap_boc); free(CdDelta); free(aq);
  return 0;
}

/* ------------------------------------------------------------------------------------------------ non-bonded core */
/* taper_coeffs + taper_horner, include/reaxmetal/terms_host.hpp:16-39 */
static void taper_coeffs(double swa, double swb, double* c) {
  const double d1 = swb - swa, d7 = pow(d1, 7.0);
  const double swa2 = swa * swa, swa3 = swa * swa * swa, swb2 = swb * swb, swb3 = swb * swb * swb;
  c[7] = 20.0 / d7;
  c[6] = -70.0 * (swa + swb) / d7;
  c[5] = 84.0 * (swa2 + 3.0 * swa * swb + swb2) / d7;
  c[4] = -35.0 * (swa3 + 9.0 * swa2 * swb + 9.0 * swa * swb2 + swb3) / d7;
  c[3] = 140.0 * (swa3 * swb + 3.0 * swa2 * swb2 + swa * swb3) / d7;
  c[2] = -210.0 * (swa3 * swb2 + swa2 * swb3) / d7;
  c[1] = 140.0 * swa3 * swb3 / d7;
  c[0] = (-35.0 * swa3 * swb2 * swb2 + 21.0 * swa2 * swb3 * swb2 - 7.0 * swa * swb3 * swb3 + swb3 * swb3 * swb) / d7;
}
static void taper_horner(const double* c, double r, double* Tap, double* dTap) {
  double t = c[7] * r + c[6];
  t = t * r + c[5]; t = t * r + c[4]; t = t * r + c[3]; t = t * r + c[2]; t = t * r + c[1]; t = t * r + c[0];
  double d = 7 * c[7] * r + 6 * c[6];
  d = d * r + 5 * c[5]; d = d * r + 4 * c[4]; d = d * r + 3 * c[3]; d = d * r + 2 * c[2];
  d += c[1] / r;
  *Tap = t;
  *dTap = d;
}

/* compute_nonbonded_core, src/cpu/nonbonded.cpp:18-82 with terms::nonbonded_pair / polarization (terms.hpp:282-326) */
static void nonbonded_core(const rxo_ff* ff, const atomset* a, const farlist* far, const double* q, double* e13, double* f,
                           int* census, long long* npairs) {
  const int n = a->nlocal;
  const double p_vdW1 = ff->gp[28];
  const int vdw_type = ff->vdw_type;
  double tap[8];
  taper_coeffs(ff->nonb_low, ff->nonb_cut, tap);
  double e_vdw = 0, e_ele = 0, e_pol = 0;
  long long pairs = 0;
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    for (long long pj = far->row_start[i]; pj < far->row_start[i + 1]; ++pj) {
      const int j = far->nbr[pj];
      const int tj = a->type[j];
      if (tj < 0) continue;
      const double r = far->dist[pj];
      if (!(r <= ff->nonb_cut)) continue;
      const double* dv = far->dvec + 3 * pj;
      if (classify(j, n, a->tag[i], a->tag[j], dv) == 0) continue;
      double Tap, dTap;
      taper_horner(tap, r, &Tap, &dTap);
      const double qi = q[i], qj = q[a->owner[j]];
      const double p_vdW1i = 1.0 / p_vdW1;
      const double alpha = TB(ti, tj, TB_ALPHA), D = TB(ti, tj, TB_D), r_vdW = TB(ti, tj, TB_R_VDW);
      double e_vdW = 0, CEvd, ev;
      if (vdw_type == 1 || vdw_type == 3) {
        const double powr_vdW1 = pow(r, p_vdW1);
        const double powgi_vdW1 = pow(1.0 / TB(ti, tj, TB_GAMMA_W), p_vdW1);
        const double fn13 = pow(powr_vdW1 + powgi_vdW1, p_vdW1i);
        const double exp1 = exp(alpha * (1.0 - fn13 / r_vdW));
        const double exp2 = exp(0.5 * alpha * (1.0 - fn13 / r_vdW));
        ev = D * (exp1 - 2.0 * exp2);
        e_vdW += Tap * ev;
        const double dfn13 = pow(powr_vdW1 + powgi_vdW1, p_vdW1i - 1.0) * pow(r, p_vdW1 - 2.0);
        CEvd = dTap * ev - Tap * D * (alpha / r_vdW) * (exp1 - exp2) * dfn13;
      } else {
        const double exp1 = exp(alpha * (1.0 - r / r_vdW));
        const double exp2 = exp(0.5 * alpha * (1.0 - r / r_vdW));
        ev = D * (exp1 - 2.0 * exp2);
        e_vdW += Tap * ev;
        CEvd = dTap * ev - Tap * D * (alpha / r_vdW) * (exp1 - exp2) / r;
      }
      if (vdw_type == 2 || vdw_type == 3) {
        const double ecore = TB(ti, tj, TB_ECORE), acore = TB(ti, tj, TB_ACORE), rcore = TB(ti, tj, TB_RCORE);
        const double e_core = ecore * exp(acore * (1.0 - (r / rcore)));
        e_vdW += Tap * e_core;
        const double de_core = -(acore / rcore) * e_core;
        CEvd += dTap * e_core + Tap * de_core / r;
        if (ff->lgvdw) {   /* include/reaxmetal/terms.hpp:308-314: nested in the inner-wall branch (Q-06) */
          const double r_ij5 = pow(r, 5.0), r_ij6 = pow(r, 6.0), re6 = pow(TB(ti, tj, TB_LGRE), 6.0);
          const double e_lg = -(TB(ti, tj, TB_LGCIJ) / (r_ij6 + re6));
          e_vdW += Tap * e_lg;
          const double de_lg = -6.0 * e_lg * r_ij5 / (r_ij6 + re6);
          CEvd += dTap * e_lg + Tap * de_lg / r;
        }
      }
      const double dr3gamij_1 = (r * r * r + TB(ti, tj, TB_GAMMA));
      const double dr3gamij_3 = pow(dr3gamij_1, 0.33333333333333);
      const double tmp = Tap / dr3gamij_3;
      const double e_ele_t = C_ELE * qi * qj * tmp;
      const double CEclmb = C_ELE * qi * qj * (dTap - Tap * r / dr3gamij_1) / dr3gamij_3;
      const double CE = CEvd + CEclmb;
      e_vdw += e_vdW;
      e_ele += e_ele_t;
      for (int c = 0; c < 3; ++c) {
        f[3 * i + c] += -CE * dv[c];
        f[3 * j + c] += +CE * dv[c];
      }
      ++pairs;
      if (census) census[4 * n + i]++;
    }
  }
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    e_pol += KCAL_TO_EV * (SB(ti, SB_CHI) * q[i] + (SB(ti, SB_ETA) / 2.) * (q[i] * q[i]));
  }
  e13[10] = e_vdw; e13[11] = e_ele; e13[12] = e_pol;
  *npairs = pairs;
}

/* ------------------------------------------------------------------------------------------------ public entry points */
static int setup(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
                 const long long* tag, atomset* a, farlist* far, char* err, int errlen) {
  memset(a, 0, sizeof *a);
  memset(far, 0, sizeof *far);
  if (ff->ngp < 39) { seterr(err, errlen, "need at least 39 general parameters"); return 2; }
  for (int i = 0; i < n; ++i)
    if (type[i] >= ff->nt) { seterr(err, errlen, "atom %d has type %d outside the force field", i, type[i]); return 2; }
  const double nonb = ff->nonb_cut;
  double shell = ctl->shell;
  const double req = nonb > ctl->hbond_cut ? nonb : ctl->hbond_cut;
  if (shell <= 0) shell = req > 2 * ctl->bond_cut ? req : 2 * ctl->bond_cut;
  if (expand_images(box, shell, n, x, type, tag, a, err, errlen)) return 3;
  build_far_list(a, nonb, ctl->bond_cut, far);
  return 0;
}

/* The pair-side ACKS2 terms (src/cpu/acks2.cpp:11-63): the polarization coupling 23.02 q_i s_i per owned atom, and
 * the bond-softness Coulomb over the counted far-list pairs within xcut = (bcut_i + bcut_j)/2,
 * E = -23.02/2 bs (s_i - s_j)^2, bs = softness d^3 (1 - d)^6, d = r / xcut, softness = gp[34]. */
static void acks2_terms(const rxo_ff* ff, const atomset* a, const farlist* far, const double* q, const double* s_kin,
                        double* e13, double* f) {
  const int n = a->nlocal;
  const double softness = ff->ngp > 34 ? ff->gp[34] : 0.0;
  double e_ele = 0.0, e_pol = 0.0;
  for (int i = 0; i < n; ++i) {
    if (a->type[i] < 0) continue;
    e_pol += KCAL_TO_EV * q[i] * s_kin[i];
  }
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    if (ti < 0) continue;
    for (long long pj = far->row_start[i]; pj < far->row_start[i + 1]; ++pj) {
      const int j = far->nbr[pj];
      const int tj = a->type[j];
      if (tj < 0) continue;
      const double xcut = 0.5 * (SB(ti, SB_BCUT_ACKS2) + SB(tj, SB_BCUT_ACKS2));
      const double dist = far->dist[pj];
      if (!(dist <= xcut)) continue;
      const double* dv = far->dvec + 3 * pj;
      if (classify(j, n, a->tag[i], a->tag[j], dv) == 0) continue;
      const double d = dist / xcut;
      const double bs = softness * pow(d, 3.0) * pow(1.0 - d, 6.0);
      if (!(bs > 0.0)) continue;
      const double effpot = s_kin[i] - s_kin[a->owner[j]];
      e_ele += -0.5 * KCAL_TO_EV * bs * effpot * effpot;
      double dbs = softness * 3.0 / xcut * pow(d, 2.0) * pow(1.0 - d, 5.0) * (1.0 - 3.0 * d);
      dbs = -0.5 * dbs * effpot * effpot;
      dbs = KCAL_TO_EV * dbs / dist;
      for (int c = 0; c < 3; ++c) {
        f[3 * i + c] += -dbs * dv[c];
        f[3 * j + c] += +dbs * dv[c];
      }
    }
  }
  e13[11] += e_ele;
  e13[12] += e_pol;
}

int rxo_single_point(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
                     const long long* tag, const double* q, double* e13, double* grad, int* census, long long* counts,
                     double* virial6, char* err, int errlen) {
  return rxo_single_point_acks2(ff, ctl, box, n, x, type, tag, q, NULL, e13, grad, census, counts, virial6, err, errlen);
}

int rxo_single_point_acks2(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x,
                           const int* type, const long long* tag, const double* q, const double* s_kin, double* e13,
                           double* grad, int* census, long long* counts, double* virial6, char* err, int errlen) {
  atomset a;
  farlist far;
  int rc = setup(ff, ctl, box, n, x, type, tag, &a, &far, err, errlen);
  if (rc) { atomset_free(&a); farlist_free(&far); return rc; }
  const int N = a.nall;
  double* f = (double*)calloc(3 * (size_t)N, sizeof(double));
  for (int t = 0; t < RXO_NTERMS; ++t) e13[t] = 0.0;
  if (census) memset(census, 0, sizeof(int) * RXO_NCENSUS * (size_t)n);
  long long nbonds = 0, npairs = 0;
  rc = bonded_core(ff, ctl, &a, &far, e13, f, census, &nbonds, err, errlen);
  if (!rc && q) nonbonded_core(ff, &a, &far, q, e13, f, census, &npairs);
  if (!rc && q && s_kin) acks2_terms(ff, &a, &far, q, s_kin, e13, f);
  if (!rc) {
    memset(grad, 0, sizeof(double) * 3 * (size_t)n);
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c) grad[3 * a.owner[i] + c] += f[3 * i + c];
    if (virial6) {   /* LAMMPS virial_fdotr_compute over owned + ghost atoms, force = -gradient */
      for (int c = 0; c < 6; ++c) virial6[c] = 0.0;
      for (int i = 0; i < N; ++i) {
        const double* xi = a.x + 3 * (size_t)i;
        const double* gi = f + 3 * (size_t)i;
        virial6[0] -= gi[0] * xi[0]; virial6[1] -= gi[1] * xi[1]; virial6[2] -= gi[2] * xi[2];
        virial6[3] -= gi[1] * xi[0]; virial6[4] -= gi[2] * xi[0]; virial6[5] -= gi[2] * xi[1];
      }
    }
    if (counts) { counts[0] = nbonds; counts[1] = npairs; counts[2] = N; counts[3] = far.entries; }
  }
  free(f);
  atomset_free(&a);
  farlist_free(&far);
  return rc;
}

/* The charge matrix of fix qeq/reaxff (docs/ENGINE_SPEC.md section 7) over the owned rows of the far list, with the
 * owner-computes rule of the stock fix (the same tie-break as the non-bonded rule, EPSILON = 1e-4). Each counted entry
 * contributes to both of its ends; ghost ends are folded onto their owners (the reverse communication of the stock
 * fix). */
typedef struct { int n; long long m; int* row_i; int* col_o; double* h; double* eta; } qmat;

static void qmat_build(const rxo_ff* ff, const atomset* a, const farlist* far, double swa, double swb, qmat* Q) {
  const int n = a->nlocal;
  double tap[8];
  taper_coeffs(swa, swb, tap);
  Q->n = n;
  Q->m = 0;
  Q->row_i = (int*)malloc(sizeof(int) * (size_t)(far->entries + 1));
  Q->col_o = (int*)malloc(sizeof(int) * (size_t)(far->entries + 1));
  Q->h = (double*)malloc(sizeof(double) * (size_t)(far->entries + 1));
  Q->eta = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) {
    const int ti = a->type[i];
    Q->eta[i] = SB(ti, SB_ETA);
    for (long long p = far->row_start[i]; p < far->row_start[i + 1]; ++p) {
      const int j = far->nbr[p];
      const double r = far->dist[p];
      if (!(r <= swb)) continue;
      if (classify(j, n, a->tag[i], a->tag[j], far->dvec + 3 * p) == 0) continue;
      const int tj = a->type[j];
      double Tap, dTap;
      taper_horner(tap, r, &Tap, &dTap);
      const double shld = pow(SB(ti, SB_GAMMA) * SB(tj, SB_GAMMA), -1.5);
      const double denom = pow(r * r * r + shld, 1.0 / 3.0);
      Q->row_i[Q->m] = i;
      Q->col_o[Q->m] = a->owner[j];
      Q->h[Q->m] = Tap * EV_TO_KCAL / denom;
      Q->m++;
    }
  }
}
static void qmat_free(qmat* Q) { free(Q->row_i); free(Q->col_o); free(Q->h); free(Q->eta); }
static void qmat_mv(const qmat* Q, const double* x, double* y) {
  for (int i = 0; i < Q->n; ++i) y[i] = Q->eta[i] * x[i];
  for (long long e = 0; e < Q->m; ++e) {
    y[Q->row_i[e]] += Q->h[e] * x[Q->col_o[e]];
    y[Q->col_o[e]] += Q->h[e] * x[Q->row_i[e]];
  }
}
static double vdot(int n, const double* a, const double* b) { double s = 0; for (int i = 0; i < n; ++i) s += a[i] * b[i]; return s; }

/* The stock CG loop as reproduced line for line in plugin/adapter/fix_qeq_reaxff_metal.cpp:89-123 */
static int qeq_cg(const qmat* Q, const double* b, double* x, double tol, int imax, double* rel) {
  const int n = Q->n;
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* d = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* q = (double*)malloc(sizeof(double) * (size_t)n);
  qmat_mv(Q, x, q);
  for (int j = 0; j < n; ++j) { r[j] = b[j] - q[j]; d[j] = r[j] / Q->eta[j]; }
  const double b_norm = sqrt(vdot(n, b, b));
  double sig_new = vdot(n, r, d), sig_old;
  int i;
  for (i = 1; i < imax && sqrt(sig_new) / b_norm > tol; ++i) {
    qmat_mv(Q, d, q);
    const double tmp = vdot(n, d, q);
    const double alpha = sig_new / tmp;
    for (int j = 0; j < n; ++j) { x[j] += alpha * d[j]; r[j] -= alpha * q[j]; p[j] = r[j] / Q->eta[j]; }
    sig_old = sig_new;
    sig_new = vdot(n, r, p);
    const double beta = sig_new / sig_old;
    for (int j = 0; j < n; ++j) d[j] = p[j] + beta * d[j];
  }
  *rel = sqrt(sig_new) / b_norm;
  free(r); free(d); free(p); free(q);
  return i;
}

int rxo_qeq(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
            const long long* tag, double swa, double swb, double tol, int imax, const double* s0, const double* t0,
            double* q, double* s, double* t, int* iters, double* rel, char* err, int errlen) {
  atomset a;
  farlist far;
  int rc = setup(ff, ctl, box, n, x, type, tag, &a, &far, err, errlen);
  if (rc) { atomset_free(&a); farlist_free(&far); return rc; }
  if (swb > ff->nonb_cut) { seterr(err, errlen, "taper radius exceeds nonb_cut"); atomset_free(&a); farlist_free(&far); return 2; }
  qmat Q;
  qmat_build(ff, &a, &far, swa, swb, &Q);
  double* b = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) { b[i] = -SB(type[i], SB_CHI); s[i] = s0[i]; }
  iters[0] = qeq_cg(&Q, b, s, tol, imax, &rel[0]);
  for (int i = 0; i < n; ++i) { b[i] = -1.0; t[i] = t0[i]; }
  iters[1] = qeq_cg(&Q, b, t, tol, imax, &rel[1]);
  /* calculate_Q (docs/ENGINE_SPEC.md section 7): q = s - (sum s / sum t) t */
  double ss = 0, st = 0;
  for (int i = 0; i < n; ++i) { ss += s[i]; st += t[i]; }
  const double u = ss / st;
  for (int i = 0; i < n; ++i) q[i] = s[i] - u * t[i];
  free(b);
  qmat_free(&Q);
  atomset_free(&a);
  farlist_free(&far);
  return 0;
}

int rxo_qeq_matvec(const rxo_ff* ff, const rxo_ctl* ctl, const rxo_box* box, int n, const double* x, const int* type,
                   const long long* tag, double swa, double swb, const double* v, double* y, char* err, int errlen) {
  atomset a;
  farlist far;
  int rc = setup(ff, ctl, box, n, x, type, tag, &a, &far, err, errlen);
  if (rc) { atomset_free(&a); farlist_free(&far); return rc; }
  qmat Q;
  qmat_build(ff, &a, &far, swa, swb, &Q);
  qmat_mv(&Q, v, y);
  qmat_free(&Q);
  atomset_free(&a);
  farlist_free(&far);
  return 0;
}
