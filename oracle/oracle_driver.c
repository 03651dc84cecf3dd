/*
 * oracle_driver.c -- CPU restatement of the reference's integral driver.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Follows, loop for loop:
 *   lattice      src/imago/lattice.f90:182-444 (recip vectors, cutoff
 *                sphere), 469-782 (cell list, border check, sort by |R|^2)
 *   k-points     src/imago/kpoints.f90:543-609 (to xyz, phase factors)
 *   basis        src/imago/basis.f90:55-243 (renormalizeBasis), 257-383
 *   screening    src/imago/gaussRelations.f90:64-278
 *   OL/KE/NP/EP  src/imago/integrals.F90:151-652, 656-1090, 1531-1942,
 *                1946-2531 with nuclearPE 2533-2698, electronicPE 2700-2858
 *   saving       src/imago/intgSaving.F90:56-89 (multWithBasisFn1),
 *                132-189 (applyPhaseFactors), 241-292 (origin shift),
 *                346-702 (saveCurrentPair and the block savers)
 *   ortho        src/imago/integrals.F90:3608-3911 with intgOrtho.F90:23-213
 *                (zherk/zher2k semantics as plain loops, packing, 1e-10)
 *
 * One deliberate difference: findLatticeVector (lattice.f90:784-888) finds
 * the lattice vector nearest an arbitrary vector through a precomputed
 * Wigner-Seitz/octant table (lattice.f90:892-1764).  Here the nearest
 * vector is found by rounding fractional coordinates and checking the 26
 * neighbouring lattice points.  Both return a nearest lattice vector; when
 * several are equally near they may pick different ones, which changes the
 * order of the lattice sums but not which terms pass the screens.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

static const double PI = 3.141592653589793; /* constants.f90:36 */
static const double SMALL_THRESH = 1.0e-8;  /* constants.f90:49 */

/* basis.f90:91-106: real-harmonic normalisations folded into the basis. */
static const double ANG_NORM[16] = {
    0.2820947917738782, 0.4886025119029199, 0.4886025119029199,
    0.4886025119029199, 1.0925484305920790, 1.0925484305920790,
    1.0925484305920790, 0.5462742152960396, 0.3153915652525200,
    2.8906114426405543, 1.4453057213202771, 0.5900435899266435,
    0.5900435899266435, 0.3731763325901154, 0.4570457994644657,
    0.4570457994644657};

typedef struct {
  int element;
  int nalpha;       /* numOrbAlphas(1) */
  int norb[4];      /* numOrbAlphas(1..4) */
  double *alphas;
  int ncore, nvale, nstates; /* states (m-resolved) */
  int *lm;          /* lmIndex (1-based lm) per state */
  int *lmalpha;     /* lmAlphaIndex per alpha: 1, 4, 9, 16 */
  double *basis;    /* [a * nstates + m] renormalised coefficients */
} otype;

typedef struct {
  int element;
  double Z, nucalpha;
  int nalpha, multiplicity, cumul;
  double *alphas;
} optype;

struct orc_ctx {
  int nt, ns, npt, nps, nk, nel;
  otype *types;
  int *site_type;     /* 0-based */
  double *site_pos;
  optype *ptypes;
  int *psite_type;    /* 0-based */
  double *psite_pos;
  int *psite_first;
  double rv[9], recip[9], inv[9];
  double T;           /* logBasisFnThresh */
  int ncell;
  double *cell;       /* [n*3] */
  double *csize;
  double *kxyz;       /* [nk*3] */
  double *phase;      /* [k*ncell + cell] (re, im) pairs: [(k*ncell+c)*2] */
  int vale_dim, core_dim, pot_dim, max_alpha, max_states, max_palpha;
  int *cum_vale, *cum_core;
  /* screening tables, indexed with 0-based elements/alphas */
  double *alpha_dist, *alpha_center, *alpha_nuc, *alpha_pot;
  /* overlap coreVale kept for the orthogonalisation of other matrices */
  double *s_cv;       /* [k][v][c] complex: ((k*V + v)*C + c)*2 */
  int have_ol;
  int stride, nthreads;
  int skip_ortho; /* timing samples: pair loops only */
  double t_loops, t_ortho;
  long long n_pair_images, n_shell_pairs, n_triples;
};

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ---------- screening table accessors (gaussRelations.f90) ---------- */
#define ADIST(c, e1, e2, a, b) \
  (c)->alpha_dist[((((e1) * (c)->nel + (e2)) * (c)->max_alpha + (a)) * (c)->max_alpha) + (b)]
#define ACENT(c, e1, e2, a, b) \
  (c)->alpha_center[((((e1) * (c)->nel + (e2)) * (c)->max_alpha + (a)) * (c)->max_alpha) + (b)]
#define ANUC(c, e1, e2, ep, a, b)                                            \
  (c)->alpha_nuc[(((((e1) * (c)->nel + (e2)) * (c)->nel + (ep)) * (c)->max_alpha + (a)) * \
                  (c)->max_alpha) + (b)]
#define APOT(c, e1, e2, ep, a, b, j)                                          \
  (c)->alpha_pot[((((((e1) * (c)->nel + (e2)) * (c)->nel + (ep)) * (c)->max_alpha + (a)) * \
                   (c)->max_alpha + (b)) * (c)->max_palpha) + (j)]

/* ---------- lattice (lattice.f90) ---------- */

/* getRecipCellVectors, lattice.f90:182-233. */
static void recip_vectors(orc_ctx *c) {
  double vol = 0.0;
  for (int i = 0; i < 3; ++i) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    vol = 0.0;
    for (int j = 0; j < 3; ++j) {
      int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      c->recip[3 * i + j] = c->rv[3 * i1 + j1] * c->rv[3 * i2 + j2] -
                            c->rv[3 * i1 + j2] * c->rv[3 * i2 + j1];
      vol += c->recip[3 * i + j] * c->rv[3 * i + j];
    }
    for (int j = 0; j < 3; ++j)
      c->recip[3 * i + j] = 2.0 * PI * c->recip[3 * i + j] / vol;
  }
  for (int i = 0; i < 9; ++i) c->inv[i] = c->recip[i] / (2.0 * PI);
}

/* cellBorderCheck, lattice.f90:698-782: walk the seven other corners of
 * the cell spanned at lattice point t. */
static int border_check(const double *rv, const double *t, double lim) {
  double sh[3] = {0, 0, 0}, cur[3];
  for (int i = 0; i < 3; ++i)
    for (int x = 0; x < 3; ++x) sh[x] += rv[3 * i + x];
  memcpy(cur, t, sizeof cur);
  static const int step[7][2] = {{0, 1}, {1, 1}, {0, -1}, {2, 1},
                                 {0, 1}, {1, -1}, {0, -1}};
  for (int s = 0; s < 7; ++s) {
    cur[step[s][0]] += step[s][1] * sh[step[s][0]];
    double r2 = cur[0] * cur[0] + cur[1] * cur[1] + cur[2] * cur[2];
    if (r2 < lim) return 1;
  }
  return 0;
}

typedef struct {
  double size;
  int idx;
} cellkey;

/* mergeSort / mergeLists (sortSubs.f90:18-200): bottom-up merges of
 * neighbouring runs, starting from runs of one; when the two heads are
 * equal the head of the second run goes first (the comparison is a strict
 * "<" on the first run), so equal sizes are not kept in input order. */
static void reference_merge_sort(cellkey *k, int n) {
  if (n < 2) return;
  cellkey *tmp = malloc(sizeof(cellkey) * n);
  int *bord = malloc(sizeof(int) * (n + 1));
  for (int i = 0; i <= n; ++i) bord[i] = i;
  cellkey *from = k, *to = tmp;
  int nseg = n;
  while (nseg > 1) {
    int t = 0;
    for (int s = 0; s < nseg / 2; ++s) {
      int p1 = bord[2 * s], e1 = bord[2 * s + 1], p2 = e1, e2 = bord[2 * s + 2];
      while (p1 < e1 && p2 < e2) to[t++] = (from[p1].size < from[p2].size) ? from[p1++] : from[p2++];
      while (p1 < e1) to[t++] = from[p1++];
      while (p2 < e2) to[t++] = from[p2++];
      bord[s + 1] = e2;
    }
    if (nseg % 2) {
      for (int i = t; i < bord[nseg]; ++i) to[i] = from[i];
      bord[nseg / 2 + 1] = bord[nseg];
    }
    nseg = nseg / 2 + nseg % 2;
    cellkey *sw = from;
    from = to;
    to = sw;
  }
  if (from != k) memcpy(k, from, sizeof(cellkey) * n);
  free(tmp);
  free(bord);
}

/* initializeLattice + makeLattice, lattice.f90:310-444, 571-690. */
static int make_lattice(orc_ctx *c, double min_atom_alpha,
                        double min_pot_alpha) {
  double lim = c->T * fmax(2.0 / min_atom_alpha,
                           1.0 / min_pot_alpha + 0.5 / min_atom_alpha);
  double maxsq = 0.0;
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int x = 0; x < 3; ++x) s += c->rv[3 * i + x] * c->rv[3 * i + x];
    maxsq = fmax(s, maxsq);
  }
  lim = lim + 0.75 * maxsq + sqrt(3.0 * maxsq * lim);
  lim = fmax(lim, 2.0 * c->T / min_atom_alpha);
  int reps[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int x = 0; x < 3; ++x) s += c->rv[3 * i + x] * c->rv[3 * i + x];
    reps[i] = 2 * (int)ceil(sqrt(lim) / sqrt(s)) + 1;
  }
  long cap = (long)reps[0] * reps[1] * reps[2];
  double *dims = malloc(sizeof(double) * 3 * cap);
  cellkey *keys = malloc(sizeof(cellkey) * cap);
  if (!dims || !keys) return IMAGO_ERR_NOMEM;
  int n = 0;
  for (int i = 1; i <= reps[0]; ++i)
    for (int j = 1; j <= reps[1]; ++j)
      for (int k = 1; k <= reps[2]; ++k) {
        int rep[3] = {i - (1 + reps[0]) / 2, j - (1 + reps[1]) / 2,
                      k - (1 + reps[2]) / 2};
        double t[3] = {0, 0, 0};
        for (int l = 0; l < 3; ++l)
          for (int m = 0; m < 3; ++m) t[m] = t[m] + c->rv[3 * l + m] * rep[l];
        double s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (s > lim && !border_check(c->rv, t, lim)) continue;
        memcpy(dims + 3 * n, t, sizeof t);
        keys[n].size = s;
        keys[n].idx = n;
        ++n;
      }
  reference_merge_sort(keys, n);
  c->ncell = n;
  c->cell = malloc(sizeof(double) * 3 * n);
  c->csize = malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    memcpy(c->cell + 3 * i, dims + 3 * keys[i].idx, 3 * sizeof(double));
    c->csize[i] = keys[i].size;
  }
  free(dims);
  free(keys);
  return IMAGO_OK;
}

/* Nearest lattice vector to v (the role of findLatticeVector,
 * lattice.f90:784-888). */
static void nearest_lattice(const orc_ctx *c, const double *v, double *out) {
  double base[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    double f = v[0] * c->inv[3 * i] + v[1] * c->inv[3 * i + 1] +
               v[2] * c->inv[3 * i + 2];
    double r = (double)(long)(fabs(f) + 0.5);
    if (f < 0.0) r = -r;
    for (int x = 0; x < 3; ++x) base[x] += c->rv[3 * i + x] * r;
  }
  double best[3] = {base[0], base[1], base[2]};
  double bd = (v[0] - base[0]) * (v[0] - base[0]) +
              (v[1] - base[1]) * (v[1] - base[1]) +
              (v[2] - base[2]) * (v[2] - base[2]);
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        if (!i && !j && !k) continue;
        double cand[3], d = 0.0;
        for (int x = 0; x < 3; ++x) {
          cand[x] = base[x] + i * c->rv[x] + j * c->rv[3 + x] + k * c->rv[6 + x];
          d += (v[x] - cand[x]) * (v[x] - cand[x]);
        }
        if (d < bd * (1.0 - 1e-12)) {
          bd = d;
          memcpy(best, cand, sizeof best);
        }
      }
  memcpy(out, best, sizeof best);
}

void orc_find_lattice_vector(const orc_ctx *c, const double *v, double *out) {
  nearest_lattice(c, v, out);
}

/* ---------- setup ---------- */

static int nsh_of_lmalpha(int lmalpha) {
  return lmalpha == 1 ? 0 : lmalpha == 4 ? 1 : lmalpha == 9 ? 2 : 3;
}

int orc_create(const imago_system *s, orc_ctx **out) {
  *out = NULL;
  if (!s || s->num_atom_types <= 0 || s->num_atom_sites <= 0 ||
      s->num_pot_types <= 0 || s->num_pot_sites <= 0 || s->num_kpoints <= 0)
    return IMAGO_ERR_INVALID;
  if (!(s->basis_fn_convg > 0.0 && s->basis_fn_convg <= 1.0))
    return IMAGO_ERR_INVALID;
  orc_ctx *c = calloc(1, sizeof(orc_ctx));
  if (!c) return IMAGO_ERR_NOMEM;
  c->stride = 1;
  c->nthreads = 1;
  c->nt = s->num_atom_types;
  c->ns = s->num_atom_sites;
  c->npt = s->num_pot_types;
  c->nps = s->num_pot_sites;
  c->nk = s->num_kpoints;
  memcpy(c->rv, s->real_vectors, sizeof c->rv);
  c->T = -log(s->basis_fn_convg); /* setCutoffThresh, lattice.f90:293 */
  recip_vectors(c);

  /* atom types + renormalizeBasis (basis.f90:55-243) */
  c->types = calloc(c->nt, sizeof(otype));
  int aoff = 0, foff = 0, coff = 0;
  double min_atom_alpha = 100.0; /* atomicTypes.f90: initial 100 */
  c->nel = 0;
  for (int t = 0; t < c->nt; ++t) {
    otype *ty = &c->types[t];
    ty->element = s->type_element[t] - 1;
    if (ty->element < 0) goto bad;
    if (ty->element + 1 > c->nel) c->nel = ty->element + 1;
    for (int l = 0; l < 4; ++l) ty->norb[l] = s->type_num_orb_alphas[4 * t + l];
    for (int l = 0; l < 3; ++l)
      if (ty->norb[l] < ty->norb[l + 1]) goto bad;
    ty->nalpha = ty->norb[0];
    if (ty->nalpha <= 0) goto bad;
    ty->alphas = malloc(sizeof(double) * ty->nalpha);
    memcpy(ty->alphas, s->type_alphas + aoff, sizeof(double) * ty->nalpha);
    aoff += ty->nalpha;
    min_atom_alpha = fmin(min_atom_alpha, ty->alphas[0]);
    if (ty->nalpha > c->max_alpha) c->max_alpha = ty->nalpha;
    int ncf = s->type_num_core_fns[t], nvf = s->type_num_vale_fns[t];
    const int *fl = s->fn_l + foff;
    ty->ncore = ty->nvale = 0;
    for (int f = 0; f < ncf; ++f) ty->ncore += 2 * fl[f] + 1;
    for (int f = 0; f < nvf; ++f) ty->nvale += 2 * fl[ncf + f] + 1;
    ty->nstates = ty->ncore + ty->nvale;
    if (ty->nstates > c->max_states) c->max_states = ty->nstates;
    ty->lm = malloc(sizeof(int) * ty->nstates);
    ty->lmalpha = malloc(sizeof(int) * ty->nalpha);
    ty->basis = calloc((size_t)ty->nalpha * ty->nstates, sizeof(double));
    for (int j = 0; j < ty->nalpha; ++j) {
      if (j < ty->norb[3]) ty->lmalpha[j] = 16;
      else if (j < ty->norb[2]) ty->lmalpha[j] = 9;
      else if (j < ty->norb[1]) ty->lmalpha[j] = 4;
      else ty->lmalpha[j] = 1;
    }
    /* coefficient offsets per fn */
    int *fco = malloc(sizeof(int) * (ncf + nvf + 1));
    int o = coff;
    for (int f = 0; f < ncf + nvf; ++f) {
      if (fl[f] < 0 || fl[f] > 3) { free(fco); goto bad; }
      fco[f] = o;
      o += ty->norb[fl[f]];
    }
    coff = o;
    int m = 0;
    /* valence first, then core (basis.f90:171-241) */
    for (int pass = 0; pass < 2; ++pass) {
      int f0 = pass == 0 ? ncf : 0, f1 = pass == 0 ? ncf + nvf : ncf;
      for (int f = f0; f < f1; ++f) {
        int l = fl[f], na = ty->norb[l];
        for (int k = 1; k <= 2 * l + 1; ++k) {
          ty->lm[m] = l * l + k;
          for (int a = 0; a < na; ++a)
            ty->basis[a * ty->nstates + m] =
                s->fn_coeffs[fco[f] + a] * ANG_NORM[ty->lm[m] - 1];
          ++m;
        }
      }
    }
    free(fco);
    foff += ncf + nvf;
  }
  /* atom sites (atomicSites.f90:160-186) */
  c->site_type = malloc(sizeof(int) * c->ns);
  c->site_pos = malloc(sizeof(double) * 3 * c->ns);
  c->cum_vale = malloc(sizeof(int) * c->ns);
  c->cum_core = malloc(sizeof(int) * c->ns);
  for (int i = 0; i < c->ns; ++i) {
    int t = s->site_type[i] - 1;
    if (t < 0 || t >= c->nt) goto bad;
    c->site_type[i] = t;
    memcpy(c->site_pos + 3 * i, s->site_pos + 3 * i, 3 * sizeof(double));
    c->cum_vale[i] = c->vale_dim;
    c->cum_core[i] = c->core_dim;
    c->vale_dim += c->types[t].nvale;
    c->core_dim += c->types[t].ncore;
  }
  /* pot types (potTypes.f90:86-241) */
  c->ptypes = calloc(c->npt, sizeof(optype));
  double min_pot_alpha = 10000.0; /* potTypes.f90: initial 10000 */
  int poff = 0;
  for (int t = 0; t < c->npt; ++t) {
    optype *p = &c->ptypes[t];
    p->element = s->pot_type_element[t] - 1;
    if (p->element < 0) goto bad;
    if (p->element + 1 > c->nel) c->nel = p->element + 1;
    p->Z = s->pot_type_nuc_charge[t];
    p->nucalpha = s->pot_type_nuc_alpha[t];
    p->nalpha = s->pot_type_num_alphas[t];
    if (p->nalpha <= 0) goto bad;
    p->alphas = malloc(sizeof(double) * p->nalpha);
    memcpy(p->alphas, s->pot_type_alphas + poff, sizeof(double) * p->nalpha);
    poff += p->nalpha;
    p->cumul = c->pot_dim;
    c->pot_dim += p->nalpha;
    if (p->nalpha > c->max_palpha) c->max_palpha = p->nalpha;
    min_pot_alpha = fmin(min_pot_alpha, p->alphas[0]);
  }
  c->psite_type = malloc(sizeof(int) * c->nps);
  c->psite_pos = malloc(sizeof(double) * 3 * c->nps);
  c->psite_first = malloc(sizeof(int) * c->nps);
  {
    int cur = 0;
    for (int i = 0; i < c->nps; ++i) {
      int t = s->pot_site_type[i] - 1;
      if (t < 0 || t >= c->npt) goto bad;
      c->psite_type[i] = t;
      memcpy(c->psite_pos + 3 * i, s->pot_site_pos + 3 * i, 3 * sizeof(double));
      c->ptypes[t].multiplicity += 1;
      /* getPotSiteImplicitInfo, potSites.f90:62-80 */
      if (i == 0) { c->psite_first[i] = 1; cur = t; }
      else if (t > cur) { c->psite_first[i] = 1; cur = t; }
      else c->psite_first[i] = 0;
    }
  }
  if (make_lattice(c, min_atom_alpha, min_pot_alpha) != IMAGO_OK) goto nomem;

  /* k-points to xyz (kpoints.f90:543-576) and phase factors (578-609) */
  c->kxyz = malloc(sizeof(double) * 3 * c->nk);
  for (int k = 0; k < c->nk; ++k) {
    const double *f = s->kpoints_abc + 3 * k;
    for (int x = 0; x < 3; ++x)
      c->kxyz[3 * k + x] = f[0] * c->recip[0 + x] + f[1] * c->recip[3 + x] +
                           f[2] * c->recip[6 + x];
  }
  c->phase = malloc(sizeof(double) * 2 * (size_t)c->nk * c->ncell);
  if (!c->phase) goto nomem;
  for (int i = 0; i < c->ncell; ++i)
    for (int k = 0; k < c->nk; ++k) {
      double d = c->kxyz[3 * k] * c->cell[3 * i] +
                 c->kxyz[3 * k + 1] * c->cell[3 * i + 1] +
                 c->kxyz[3 * k + 2] * c->cell[3 * i + 2];
      c->phase[2 * ((size_t)k * c->ncell + i)] = cos(d);
      c->phase[2 * ((size_t)k * c->ncell + i) + 1] = sin(d);
    }

  /* screening tables (gaussRelations.f90:64-278), per element from the
   * first type / pot type of that element */
  {
    int ne = c->nel, ma = c->max_alpha, mp = c->max_palpha;
    int *el_type = malloc(sizeof(int) * ne), *el_ptype = malloc(sizeof(int) * ne);
    for (int e = 0; e < ne; ++e) el_type[e] = el_ptype[e] = -1;
    for (int t = 0; t < c->nt; ++t)
      if (el_type[c->types[t].element] < 0) el_type[c->types[t].element] = t;
    for (int t = 0; t < c->npt; ++t)
      if (el_ptype[c->ptypes[t].element] < 0) el_ptype[c->ptypes[t].element] = t;
    size_t n2 = (size_t)ne * ne * ma * ma;
    c->alpha_dist = calloc(n2, sizeof(double));
    c->alpha_center = calloc(n2, sizeof(double));
    c->alpha_nuc = calloc(n2 * ne, sizeof(double));
    c->alpha_pot = calloc(n2 * ne * mp, sizeof(double));
    if (!c->alpha_dist || !c->alpha_center || !c->alpha_nuc || !c->alpha_pot) {
      free(el_type); free(el_ptype); goto nomem;
    }
    for (int e1 = 0; e1 < ne; ++e1)
      for (int e2 = 0; e2 < ne; ++e2) {
        if (el_type[e1] < 0 || el_type[e2] < 0) continue;
        const otype *t1 = &c->types[el_type[e1]], *t2 = &c->types[el_type[e2]];
        for (int a = 0; a < t1->nalpha; ++a)
          for (int b = 0; b < t2->nalpha; ++b) {
            double x1 = t1->alphas[a], x2 = t2->alphas[b];
            double cen = x1 / (x1 + x2);
            ACENT(c, e1, e2, a, b) = cen;
            ADIST(c, e1, e2, a, b) = c->T / x2 / cen;
            for (int ep = 0; ep < ne; ++ep) {
              if (el_ptype[ep] < 0) continue;
              const optype *pt = &c->ptypes[el_ptype[ep]];
              double nuc = pt->nucalpha;
              ANUC(c, e1, e2, ep, a, b) = c->T * (x1 + x2 + nuc) / (x1 + x2) / nuc;
              for (int j = 0; j < pt->nalpha; ++j) {
                double pa = pt->alphas[j];
                APOT(c, e1, e2, ep, a, b, j) = c->T * (x1 + x2 + pa) / (x1 + x2) / pa;
              }
            }
          }
      }
    free(el_type);
    free(el_ptype);
  }
  c->s_cv = calloc((size_t)2 * c->nk * c->vale_dim * (c->core_dim ? c->core_dim : 1),
                   sizeof(double));
  if (!c->s_cv) goto nomem;
  *out = c;
  return IMAGO_OK;
bad:
  orc_destroy(c);
  return IMAGO_ERR_INVALID;
nomem:
  orc_destroy(c);
  return IMAGO_ERR_NOMEM;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  if (c->types)
    for (int t = 0; t < c->nt; ++t) {
      free(c->types[t].alphas);
      free(c->types[t].lm);
      free(c->types[t].lmalpha);
      free(c->types[t].basis);
    }
  if (c->ptypes)
    for (int t = 0; t < c->npt; ++t) free(c->ptypes[t].alphas);
  free(c->types); free(c->ptypes); free(c->site_type); free(c->site_pos);
  free(c->psite_type); free(c->psite_pos); free(c->psite_first);
  free(c->cell); free(c->csize); free(c->kxyz); free(c->phase);
  free(c->cum_vale); free(c->cum_core);
  free(c->alpha_dist); free(c->alpha_center); free(c->alpha_nuc);
  free(c->alpha_pot); free(c->s_cv);
  free(c);
}

int orc_dims(const orc_ctx *c, imago_dims *d) {
  memset(d, 0, sizeof *d);
  d->vale_dim = c->vale_dim;
  d->core_dim = c->core_dim;
  d->num_kpoints = c->nk;
  d->pot_dim = c->pot_dim;
  d->num_cells = c->ncell;
  d->packed = (long long)c->vale_dim * (c->vale_dim + 1) / 2;
  d->num_pair_images = c->n_pair_images;
  d->num_shell_pairs = c->n_shell_pairs;
  return IMAGO_OK;
}

/* Timing samples only: with skip != 0 the builds run their pair loops but
 * not the orthogonalisation and packing, so their outputs stay unwritten. */
void orc_set_skip_ortho(orc_ctx *c, int skip) { c->skip_ortho = skip; }

void orc_set_sampling(orc_ctx *c, int stride, int nthreads) {
  c->stride = stride > 0 ? stride : 1;
  c->nthreads = nthreads;
}

int orc_num_cells(const orc_ctx *c) { return c->ncell; }
void orc_cells(const orc_ctx *c, double *dims, double *sizes) {
  memcpy(dims, c->cell, sizeof(double) * 3 * c->ncell);
  memcpy(sizes, c->csize, sizeof(double) * c->ncell);
}
void orc_kpoints_xyz(const orc_ctx *c, double *k) {
  memcpy(k, c->kxyz, sizeof(double) * 3 * c->nk);
}
void orc_last_times(const orc_ctx *c, double *loops_s, double *ortho_s) {
  *loops_s = c->t_loops;
  *ortho_s = c->t_ortho;
}
void orc_last_counts(const orc_ctx *c, long long *pi, long long *sp,
                     long long *tr) {
  *pi = c->n_pair_images;
  *sp = c->n_shell_pairs;
  *tr = c->n_triples;
}

/* ---------- the integral builds ---------- */

enum { K_OL = 0, K_KE = 1, K_NP = 2, K_EP = 3, K_MV = 4, K_HAM = 5, K_MM = 6, K_DM = 7,
       K_KOV = 8 };

typedef struct {
  /* global matrices for one build (complex, column-major like Fortran) */
  double *vv;  /* [k][v(col)][v(row)] -> ((k*V + col)*V + row)*2 */
  double *cv;  /* [k][v(col)][c(row)] */
  double *cc;  /* [k][c(col)][c(row)] */
} gmats;

#define VV(g, c, k, row, col) ((g)->vv + 2 * (((size_t)(k) * (c)->vale_dim + (col)) * (c)->vale_dim + (row)))
#define CV(g, c, k, row, col) ((g)->cv + 2 * (((size_t)(k) * (c)->vale_dim + (col)) * (c)->core_dim + (row)))
#define CC(g, c, k, row, col) ((g)->cc + 2 * (((size_t)(k) * (c)->core_dim + (col)) * (c)->core_dim + (row)))

typedef struct {
  int kind;
  int ptype;    /* EP: pot type */
  int pterm;    /* EP: alpha index within the type */
  unsigned char *anyint; /* EP: [i][j][cell] interaction bits */
  const double *coeffs;  /* HAM: potCoeffs(potDim, spin), column-major */
  int spin, q, rel;      /* HAM: spins, the spin built, mass velocity;
                          * MM, DM: q is the Cartesian component built */
  const double *center;  /* DM: dipoleCenter; KOV: the wave vector dK */
} buildspec;

/* saveCurrentPair, intgSaving.F90:346-459 with valeValeSaving 463-510,
 * coreValeSaving 555-608, coreCoreSaving 611-650.  cp is
 * [k][m1][m2] complex, ni x nj used of ms x ms. */
static void save_pair(const orc_ctx *c, gmats *g, int i, int j,
                      const double *cp, int ms) {
  const otype *t1 = &c->types[c->site_type[i]], *t2 = &c->types[c->site_type[j]];
  int v1 = t1->nvale, v2 = t2->nvale, c1 = t1->ncore, c2 = t2->ncore;
  int vi = c->cum_vale[i], vj = c->cum_vale[j];
  int ci = c->cum_core[i], cj = c->cum_core[j];
#define CP(k, a, b) (cp + 2 * (((size_t)(k) * ms + (a)) * ms + (b)))
  for (int k = 0; k < c->nk; ++k) {
    for (int a = 0; a < v1; ++a)
      for (int b = 0; b < v2; ++b) {
        double *d = VV(g, c, k, vi + a, vj + b);
        d[0] = CP(k, a, b)[0];
        d[1] = CP(k, a, b)[1];
      }
    if (i == j)
      for (int col = vi; col < vi + v1; ++col)
        for (int row = col + 1; row < vj + v2; ++row) {
          double *d = VV(g, c, k, row, col);
          d[0] = 0.0;
          d[1] = 0.0;
        }
  }
  if (c->core_dim == 0) return;
  if (c1 != 0)
    for (int k = 0; k < c->nk; ++k)
      for (int a = 0; a < c1; ++a)
        for (int b = 0; b < v2; ++b) {
          double *d = CV(g, c, k, ci + a, vj + b);
          d[0] = CP(k, v1 + a, b)[0];
          d[1] = CP(k, v1 + a, b)[1];
        }
  if (c2 != 0)
    for (int k = 0; k < c->nk; ++k)
      for (int a = 0; a < c2; ++a)
        for (int b = 0; b < v1; ++b) {
          /* currentPairDagger(v2+a, b) = conjg(currentPair(b, v2+a)) */
          double *d = CV(g, c, k, cj + a, vi + b);
          d[0] = CP(k, b, v2 + a)[0];
          d[1] = -CP(k, b, v2 + a)[1];
        }
  if (c1 == 0 || c2 == 0) return;
  for (int k = 0; k < c->nk; ++k) {
    for (int a = 0; a < c1; ++a)
      for (int b = 0; b < c2; ++b) {
        double *d = CC(g, c, k, ci + a, cj + b);
        d[0] = CP(k, v1 + a, v2 + b)[0];
        d[1] = CP(k, v1 + a, v2 + b)[1];
      }
    if (i != j)
      for (int a = 0; a < c2; ++a)
        for (int b = 0; b < c1; ++b) {
          double *d = CC(g, c, k, cj + a, ci + b);
          d[0] = CP(k, v1 + b, v2 + a)[0];
          d[1] = -CP(k, v1 + b, v2 + a)[1];
        }
  }
#undef CP
}

/* saveCurrentPair with saveFull = 1 (intgSaving.F90:346-459, 513-551,
 * 555-608, 654-690): block (i, j) takes the pair, block (j, i) its dagger;
 * for i == j the dagger, written second, replaces the block. */
static void save_pair_full(const orc_ctx *c, gmats *g, int i, int j,
                           const double *cp, int ms) {
  const otype *t1 = &c->types[c->site_type[i]], *t2 = &c->types[c->site_type[j]];
  int v1 = t1->nvale, v2 = t2->nvale, c1 = t1->ncore, c2 = t2->ncore;
  int vi = c->cum_vale[i], vj = c->cum_vale[j];
  int ci = c->cum_core[i], cj = c->cum_core[j];
#define CP(k, a, b) (cp + 2 * (((size_t)(k) * ms + (a)) * ms + (b)))
  for (int k = 0; k < c->nk; ++k) {
    for (int a = 0; a < v1; ++a)
      for (int b = 0; b < v2; ++b) {
        double *d = VV(g, c, k, vi + a, vj + b);
        d[0] = CP(k, a, b)[0];
        d[1] = CP(k, a, b)[1];
      }
    for (int a = 0; a < v2; ++a)
      for (int b = 0; b < v1; ++b) {
        double *d = VV(g, c, k, vj + a, vi + b);
        d[0] = CP(k, b, a)[0];
        d[1] = -CP(k, b, a)[1];
      }
  }
  if (c->core_dim == 0) return;
  if (c1 != 0)
    for (int k = 0; k < c->nk; ++k)
      for (int a = 0; a < c1; ++a)
        for (int b = 0; b < v2; ++b) {
          double *d = CV(g, c, k, ci + a, vj + b);
          d[0] = CP(k, v1 + a, b)[0];
          d[1] = CP(k, v1 + a, b)[1];
        }
  if (c2 != 0)
    for (int k = 0; k < c->nk; ++k)
      for (int a = 0; a < c2; ++a)
        for (int b = 0; b < v1; ++b) {
          double *d = CV(g, c, k, cj + a, vi + b);
          d[0] = CP(k, b, v2 + a)[0];
          d[1] = -CP(k, b, v2 + a)[1];
        }
  if (c1 == 0 || c2 == 0) return;
  for (int k = 0; k < c->nk; ++k) {
    for (int a = 0; a < c1; ++a)
      for (int b = 0; b < c2; ++b) {
        double *d = CC(g, c, k, ci + a, cj + b);
        d[0] = CP(k, v1 + a, v2 + b)[0];
        d[1] = CP(k, v1 + a, v2 + b)[1];
      }
    for (int a = 0; a < c2; ++a)
      for (int b = 0; b < c1; ++b) {
        double *d = CC(g, c, k, cj + a, ci + b);
        d[0] = CP(k, v1 + b, v2 + a)[0];
        d[1] = -CP(k, v1 + b, v2 + a)[1];
      }
  }
#undef CP
}

/* nuclearPE (integrals.F90:2533-2698) / electronicPE (2700-2858): the
 * three-centre sum over potential sites and their lattice images for one
 * alpha pair.  Returns 1 when some site passed the closest-image screen. */
static int three_centre(const orc_ctx *c, const buildspec *bs, int e1, int e2,
                        int a, int b, double alpha1, double alpha2,
                        double r2, const double *A, const double *Bp, int la,
                        int lb, double *acc, long long *ntrip) {
  double cen = ACENT(c, e1, e2, a, b);
  double P[3];
  for (int x = 0; x < 3; ++x) P[x] = cen * (A[x] - Bp[x]) + Bp[x];
  double sh[256];
  memset(acc, 0, sizeof(double) * 256);
  int contrib = 0;
  int s0, s1;
  if (bs->kind == K_NP) { s0 = 0; s1 = c->nps; }
  else {
    s0 = -1;
    for (int s = 0; s < c->nps; ++s)
      if (c->psite_type[s] == bs->ptype) { s0 = s; break; }
    s1 = s0 + c->ptypes[bs->ptype].multiplicity;
  }
  double t_ep = 0.0;
  if (bs->kind == K_EP) {
    int ep = c->ptypes[bs->ptype].element;
    t_ep = (1 - r2 / ADIST(c, e1, e2, a, b)) * APOT(c, e1, e2, ep, a, b, bs->pterm);
  }
  for (int s = s0; s < s1; ++s) {
    const optype *pt = &c->ptypes[c->psite_type[s]];
    double t, alpha3, w;
    if (bs->kind == K_NP) {
      if (pt->Z < SMALL_THRESH) continue;
      t = (1 - r2 / ADIST(c, e1, e2, a, b)) * ANUC(c, e1, e2, pt->element, a, b);
      alpha3 = pt->nucalpha;
      w = -pt->Z;
    } else {
      t = t_ep;
      alpha3 = pt->alphas[bs->pterm];
      w = 1.0;
    }
    const double *Cp = c->psite_pos + 3 * s;
    double d[3], L2[3], v[3];
    for (int x = 0; x < 3; ++x) d[x] = P[x] - Cp[x];
    nearest_lattice(c, d, L2);
    double c0 = 0.0;
    for (int x = 0; x < 3; ++x) {
      v[x] = P[x] - Cp[x] - L2[x];
      c0 += v[x] * v[x];
    }
    if (c0 > t) continue;
    contrib = 1;
    double maxr = c0 + t + 2.0 * sqrt(c0 * t);
    for (int n = 0; n < c->ncell; ++n) {
      if (c->csize[n] > maxr) break;
      const double *R = c->cell + 3 * n;
      double sc = (v[0] - R[0]) * (v[0] - R[0]) + (v[1] - R[1]) * (v[1] - R[1]) +
                  (v[2] - R[2]) * (v[2] - R[2]);
      if (sc > t) continue;
      double Cs[3];
      for (int x = 0; x < 3; ++x) Cs[x] = Cp[x] + L2[x] + R[x];
      if (bs->kind == K_NP)
        orc_nuclear3c(alpha1, alpha2, alpha3, A, Bp, Cs, la, lb, sh);
      else
        orc_electron3c(alpha1, alpha2, alpha3, A, Bp, Cs, la, lb, sh);
      ++*ntrip;
      int n1 = (la + 1) * (la + 1), n2 = (lb + 1) * (lb + 1);
      for (int p = 0; p < n1; ++p)
        for (int q = 0; q < n2; ++q) {
          if (w == 1.0) acc[p * 16 + q] = acc[p * 16 + q] + sh[p * 16 + q];
          else acc[p * 16 + q] = acc[p * 16 + q] - sh[p * 16 + q] * pt->Z;
        }
    }
  }
  return contrib;
}

/* The PSCF Hamiltonian of one alpha pair for spin q, gaussOverlapHamPSCF
 * (integrals.F90:3240-3442): for the first site of each potential type
 * (potSites%firstPotType), each of the type's alphas weighted by its
 * potCoeffs entry and then the nuclear term weighted by -Z (skipped when
 * Z < smallThresh), over the type's sites and their lattice images within
 * the inline radius logBasisFnThresh (1 - r2/alphaDist) (a1+a2+a3)/(a1+a2)/a3
 * (3297-3306, evaluated left to right); then + kinetic and, when rel,
 * - mass velocity (3444-3490).  potCoeffIndex runs over the types' alphas
 * in that order, which is the EP term order. */
static void ham_pscf_pair(const orc_ctx *c, const buildspec *bs, int e1, int e2,
                          int a, int b, double alpha1, double alpha2, double r2,
                          const double *A, const double *Bp, int la, int lb,
                          double *acc, long long *ntrip) {
  double cen = ACENT(c, e1, e2, a, b);
  double P[3];
  for (int x = 0; x < 3; ++x) P[x] = cen * (A[x] - Bp[x]) + Bp[x];
  const int n1 = (la + 1) * (la + 1), n2 = (lb + 1) * (lb + 1);
  double sh[256];
  memset(acc, 0, sizeof(double) * 256);
  int coeff_index = 0;
  for (int m = 0; m < c->nps; ++m) {
    if (!c->psite_first[m]) continue;
    const optype *pt = &c->ptypes[c->psite_type[m]];
    for (int n = 0; n <= pt->nalpha; ++n) {
      double coeff = 0.0, alpha3;
      if (n < pt->nalpha) {
        coeff = bs->coeffs[(size_t)bs->q * c->pot_dim + coeff_index];
        ++coeff_index;
        alpha3 = pt->alphas[n];
      } else {
        if (pt->Z < SMALL_THRESH) continue;
        alpha3 = pt->nucalpha;
      }
      double t = c->T * (1 - r2 / ADIST(c, e1, e2, a, b)) * (alpha1 + alpha2 + alpha3) /
                 (alpha1 + alpha2) / alpha3;
      for (int o = 0; o < pt->multiplicity; ++o) {
        const double *Cp = c->psite_pos + 3 * (m + o);
        double d[3], L2[3], v[3];
        for (int x = 0; x < 3; ++x) d[x] = P[x] - Cp[x];
        nearest_lattice(c, d, L2);
        double c0 = 0.0;
        for (int x = 0; x < 3; ++x) {
          v[x] = P[x] - Cp[x] - L2[x];
          c0 += v[x] * v[x];
        }
        if (c0 > t) continue;
        double maxr = c0 + t + 2.0 * sqrt(c0 * t);
        for (int p = 0; p < c->ncell; ++p) {
          if (c->csize[p] > maxr) break;
          const double *R = c->cell + 3 * p;
          double sc = (v[0] - R[0]) * (v[0] - R[0]) + (v[1] - R[1]) * (v[1] - R[1]) +
                      (v[2] - R[2]) * (v[2] - R[2]);
          if (sc > t) continue;
          double Cs[3];
          for (int x = 0; x < 3; ++x) Cs[x] = Cp[x] + L2[x] + R[x];
          ++*ntrip;
          if (n < pt->nalpha) {
            orc_electron3c(alpha1, alpha2, alpha3, A, Bp, Cs, la, lb, sh);
            for (int i = 0; i < n1; ++i)
              for (int j = 0; j < n2; ++j)
                acc[i * 16 + j] = acc[i * 16 + j] + sh[i * 16 + j] * coeff;
          } else {
            orc_nuclear3c(alpha1, alpha2, alpha3, A, Bp, Cs, la, lb, sh);
            for (int i = 0; i < n1; ++i)
              for (int j = 0; j < n2; ++j)
                acc[i * 16 + j] = acc[i * 16 + j] - sh[i * 16 + j] * pt->Z;
          }
        }
      }
    }
  }
  orc_kinetic2c(alpha1, alpha2, A, Bp, la, lb, sh);
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j) acc[i * 16 + j] = acc[i * 16 + j] + sh[i * 16 + j];
  if (bs->rel) {
    orc_massvel2c(alpha1, alpha2, A, Bp, la, lb, sh);
    for (int i = 0; i < n1; ++i)
      for (int j = 0; j < n2; ++j) acc[i * 16 + j] = acc[i * 16 + j] - sh[i * 16 + j];
  }
}

/* The atom-pair x lattice x alpha-pair loop nest shared by gaussOverlapOL
 * (integrals.F90:151-652), gaussOverlapKE (656-1090), gaussOverlapNP
 * (1531-1942) and gaussOverlapEP (1946-2356). */
static int pair_loops(orc_ctx *c, const buildspec *bs, gmats *g) {
  const int nk = c->nk, ms = c->max_states, ma = c->max_alpha;
  int npairs = c->ns * (c->ns + 1) / 2;
  int err = IMAGO_OK;
  long long npi = 0, nsp = 0, ntr = 0;
#ifdef _OPENMP
  int nth = c->nthreads > 0 ? c->nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nth) reduction(+ : npi, nsp, ntr)
#endif
  {
    double *cp = malloc(sizeof(double) * 2 * (size_t)nk * ms * ms);
    double *X = malloc(sizeof(double) * 16 * (size_t)ma * ms);
    double *M = malloc(sizeof(double) * (size_t)ms * ms);
    /* KOV: imaginary parts of X and M */
    double *X2 = bs->kind == K_KOV ? malloc(sizeof(double) * 16 * (size_t)ma * ms) : NULL;
    double *M2 = bs->kind == K_KOV ? malloc(sizeof(double) * (size_t)ms * ms) : NULL;
    double sh[256], sh2[512];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
    for (int p = 0; p < npairs; ++p) {
      if (p % c->stride) continue;
      /* invert the i-major upper-triangle pair index */
      int i = 0, rem = p;
      while (rem >= c->ns - i) { rem -= c->ns - i; ++i; }
      int j = i + rem;
      const otype *t1 = &c->types[c->site_type[i]], *t2 = &c->types[c->site_type[j]];
      int e1 = t1->element, e2 = t2->element;
      const double *A = c->site_pos + 3 * i, *B = c->site_pos + 3 * j;
      double dv[3], L0[3];
      for (int x = 0; x < 3; ++x) dv[x] = A[x] - B[x];
      nearest_lattice(c, dv, L0);
      double r02 = 0.0;
      for (int x = 0; x < 3; ++x) r02 += (A[x] - B[x] - L0[x]) * (A[x] - B[x] - L0[x]);
      double lim = ADIST(c, e1, e2, 0, 0);
      if (r02 > lim) continue;
      double maxr = r02 + lim + 2.0 * sqrt(r02 * lim);
      if (maxr > c->csize[c->ncell - 1]) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
        err = IMAGO_ERR_CELL_LIST;
        continue;
      }
      int n1 = t1->nstates, n2 = t2->nstates;
      memset(cp, 0, sizeof(double) * 2 * (size_t)nk * ms * ms);
      for (int k = 0; k < c->ncell; ++k) {
        if (c->csize[k] > maxr) break;
        unsigned char *bit = NULL;
        if (bs->kind == K_EP) {
          bit = bs->anyint + ((size_t)i * c->ns + j) * c->ncell + k;
          if (!*bit) continue; /* checkElecPotInteraction */
        }
        int elec_int = 0;
        double Bp[3];
        for (int x = 0; x < 3; ++x) Bp[x] = B[x] + L0[x] + c->cell[3 * k + x];
        double r2 = 0.0;
        for (int x = 0; x < 3; ++x) r2 += (A[x] - Bp[x]) * (A[x] - Bp[x]);
        if (r2 > lim) continue;
        ++npi;
        memset(X, 0, sizeof(double) * 16 * (size_t)ma * ms);
        if (X2) memset(X2, 0, sizeof(double) * 16 * (size_t)ma * ms);
        int max_a1 = 0;
        int nmin = t1->nalpha < t2->nalpha ? t1->nalpha : t2->nalpha;
        for (int l = 0; l < nmin; ++l) {
          int mode = 0, ai[2] = {l, l};
          if (ADIST(c, e1, e2, l, l) < r2) break;
          for (;;) {
            if (mode == 1) {
              ai[0] += 1;
              if (ai[0] >= t1->nalpha) { mode = 2; ai[0] = l; continue; }
            } else if (mode == 2) {
              ai[1] += 1;
              if (ai[1] >= t2->nalpha) break;
            }
            if (ADIST(c, e1, e2, ai[0], ai[1]) < r2) {
              if (mode == 1) { mode = 2; ai[0] = l; continue; }
              break;
            }
            if (mode == 0) mode = 1;
            int a = ai[0], b = ai[1];
            int la = nsh_of_lmalpha(t1->lmalpha[a]);
            int lb = nsh_of_lmalpha(t2->lmalpha[b]);
            ++nsp;
            int contrib = 1;
            if (bs->kind == K_OL)
              orc_overlap2c(t1->alphas[a], t2->alphas[b], A, Bp, la, lb, sh);
            else if (bs->kind == K_KE)
              orc_kinetic2c(t1->alphas[a], t2->alphas[b], A, Bp, la, lb, sh);
            else if (bs->kind == K_HAM)
              ham_pscf_pair(c, bs, e1, e2, a, b, t1->alphas[a], t2->alphas[b], r2, A,
                            Bp, la, lb, sh, &ntr);
            else if (bs->kind == K_KOV) {
              /* KOverlap2CIntg, complex (integrals3Terms.F90:1293-1297) */
              orc_koverlap2c(t1->alphas[a], t2->alphas[b], A, Bp, bs->center, la, lb, sh2);
              for (int q = 0; q < 256; ++q) sh[q] = sh2[2 * q];
            } else if (bs->kind == K_MM || bs->kind == K_DM) {
              /* one component of momentum2CIntg / dipole3CIntg
               * (integrals3Terms.F90:398-401, 849-852) */
              double sh3[768];
              if (bs->kind == K_MM)
                orc_momentum2c(t1->alphas[a], t2->alphas[b], A, Bp, la, lb, sh3);
              else
                orc_dipole2c(t1->alphas[a], t2->alphas[b], A, Bp, bs->center, la, lb, sh3);
              memcpy(sh, sh3 + 256 * bs->q, sizeof(double) * 256);
            } else if (bs->kind == K_MV) {
              /* accumulated with a minus sign (integrals.F90:1440-1447):
               * a + (-x) c is a - x c exactly */
              orc_massvel2c(t1->alphas[a], t2->alphas[b], A, Bp, la, lb, sh);
              for (int q = 0; q < 256; ++q) sh[q] = -sh[q];
            } else {
              contrib = three_centre(c, bs, e1, e2, a, b, t1->alphas[a],
                                     t2->alphas[b], r2, A, Bp, la, lb, sh,
                                     &ntr);
              if (contrib && bs->kind == K_EP) elec_int = 1;
            }
            if (contrib) {
              int nl = t1->lmalpha[a];
              for (int m = 0; m < n2; ++m) {
                double cb = t2->basis[b * n2 + m];
                int lm2 = t2->lm[m] - 1;
                for (int lm1 = 0; lm1 < nl; ++lm1)
                  X[((size_t)lm1 * ma + a) * ms + m] =
                      X[((size_t)lm1 * ma + a) * ms + m] + sh[lm1 * 16 + lm2] * cb;
                if (X2)
                  for (int lm1 = 0; lm1 < nl; ++lm1)
                    X2[((size_t)lm1 * ma + a) * ms + m] =
                        X2[((size_t)lm1 * ma + a) * ms + m] +
                        sh2[2 * (lm1 * 16 + lm2) + 1] * cb;
              }
              if (a + 1 > max_a1) max_a1 = a + 1;
            }
          }
        }
        /* multWithBasisFn1, intgSaving.F90:56-89 */
        for (int m2 = 0; m2 < n2; ++m2)
          for (int m1 = 0; m1 < n1; ++m1) {
            double s = 0.0;
            int lm1 = t1->lm[m1] - 1;
            for (int a = 0; a < max_a1; ++a)
              s = s + t1->basis[a * n1 + m1] * X[((size_t)lm1 * ma + a) * ms + m2];
            M[m1 * ms + m2] = s;
            if (M2) {
              /* cmplxMultWithBasisFn1 */
              double s2 = 0.0;
              for (int a = 0; a < max_a1; ++a)
                s2 = s2 + t1->basis[a * n1 + m1] * X2[((size_t)lm1 * ma + a) * ms + m2];
              M2[m1 * ms + m2] = s2;
            }
          }
        /* applyPhaseFactors, intgSaving.F90:132-189 */
        /* gaussOverlapMV phases only pairs that used an alpha
         * (integrals.F90:1458-1480), and gaussOverlapHamPSCF likewise
         * (3519-3553), as gaussOverlapOL does */
        if (max_a1 > 0 || (bs->kind != K_OL && bs->kind != K_MV && bs->kind != K_HAM))
          for (int kp = 0; kp < nk; ++kp) {
            double pr = c->phase[2 * ((size_t)kp * c->ncell + k)];
            double pi = c->phase[2 * ((size_t)kp * c->ncell + k) + 1];
            for (int m1 = 0; m1 < n1; ++m1)
              for (int m2 = 0; m2 < n2; ++m2) {
                double *d = cp + 2 * (((size_t)kp * ms + m1) * ms + m2);
                double x = M[m1 * ms + m2];
                if (bs->kind == K_KOV) {
                  /* cmplxApplyPhaseFactors: phase * (x + i x2),
                   * intgSaving.F90:218-230 */
                  const double x2 = M2[m1 * ms + m2];
                  d[0] = d[0] + (pr * x - pi * x2);
                  d[1] = d[1] + (pr * x2 + pi * x);
                } else if (bs->kind == K_MM) {
                  /* applyPhaseFactors runCode 1: (0,-1) * phase * x,
                   * intgSaving.F90:178-186 */
                  d[0] = d[0] + pi * x;
                  d[1] = d[1] + (-pr) * x;
                } else {
                  d[0] = d[0] + pr * x;
                  d[1] = d[1] + pi * x;
                }
              }
          }
        if (bs->kind == K_EP && !elec_int) *bit = 0;
      }
      /* kPointLatticeOriginShift, intgSaving.F90:241-292 */
      for (int kp = 0; kp < nk; ++kp) {
        const double *kv = c->kxyz + 3 * kp;
        double dot = kv[0] * L0[0] + kv[1] * L0[1] + kv[2] * L0[2];
        if (fabs(dot) >= SMALL_THRESH) {
          double cr = cos(dot), ci = sin(dot);
          for (int m2 = 0; m2 < n2; ++m2)
            for (int m1 = 0; m1 < n1; ++m1) {
              double *d = cp + 2 * (((size_t)kp * ms + m1) * ms + m2);
              double re = cr * d[0] - ci * d[1], im = cr * d[1] + ci * d[0];
              d[0] = re;
              d[1] = im;
            }
        }
      }
      if (bs->kind == K_KOV)
        save_pair_full(c, g, i, j, cp, ms);
      else
        save_pair(c, g, i, j, cp, ms);
    }
    free(cp);
    free(X2);
    free(M2);
    free(X);
    free(M);
  }
  c->n_pair_images += npi;
  c->n_shell_pairs += nsp;
  c->n_triples += ntr;
  return err;
}

/* Core orthogonalisation and packing, integrals.F90:3608-3911 with
 * intgOrtho.F90:23-213.  is_ol selects zherk (OL) or zher2k (others);
 * x_cv is the matrix's own coreVale, s_cv the overlap's. */
static void ortho_pack(orc_ctx *c, gmats *g, int is_ol, double *packed) {
  const int V = c->vale_dim, C = c->core_dim;
  const size_t np = (size_t)V * (V + 1) / 2;
#ifdef _OPENMP
  int nth = c->nthreads > 0 ? c->nthreads : omp_get_max_threads();
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1)
#endif
  for (int k = 0; k < c->nk; ++k) {
    double *out = packed + 2 * np * (size_t)k;
    if (C == 0) {
      size_t idx = 0;
      for (int col = 0; col < V; ++col)
        for (int row = 0; row <= col; ++row, ++idx) {
          out[2 * idx] = VV(g, c, k, row, col)[0];
          out[2 * idx + 1] = VV(g, c, k, row, col)[1];
        }
      continue;
    }
    const double *S = c->s_cv + 2 * (size_t)k * V * C; /* [v][c] */
#define SCV(row, col) (S + 2 * ((size_t)(col) * C + (row)))
    if (is_ol) {
      /* zherk('U','C',V,C,-2,coreValeOL,C,1,valeVale,V) */
      for (int j = 0; j < V; ++j) {
        for (int i = 0; i < j; ++i) {
          double tr = 0.0, ti = 0.0;
          for (int l = 0; l < C; ++l) {
            const double *a = SCV(l, i), *b = SCV(l, j);
            tr += a[0] * b[0] + a[1] * b[1];
            ti += a[0] * b[1] - a[1] * b[0];
          }
          double *d = VV(g, c, k, i, j);
          d[0] = -2.0 * tr + d[0];
          d[1] = -2.0 * ti + d[1];
        }
        double rt = 0.0;
        for (int l = 0; l < C; ++l) {
          const double *a = SCV(l, j);
          rt += a[0] * a[0] + a[1] * a[1];
        }
        double *d = VV(g, c, k, j, j);
        d[0] = -2.0 * rt + d[0];
        d[1] = 0.0;
      }
    } else {
      /* zher2k('U','C',V,C,(-1,0),coreValeOL,C,coreVale,C,1,valeVale,V) */
      for (int j = 0; j < V; ++j)
        for (int i = 0; i <= j; ++i) {
          double t1r = 0, t1i = 0, t2r = 0, t2i = 0;
          for (int l = 0; l < C; ++l) {
            const double *a_i = SCV(l, i), *a_j = SCV(l, j);
            const double *b_i = CV(g, c, k, l, i), *b_j = CV(g, c, k, l, j);
            t1r += a_i[0] * b_j[0] + a_i[1] * b_j[1];
            t1i += a_i[0] * b_j[1] - a_i[1] * b_j[0];
            t2r += b_i[0] * a_j[0] + b_i[1] * a_j[1];
            t2i += b_i[0] * a_j[1] - b_i[1] * a_j[0];
          }
          double *d = VV(g, c, k, i, j);
          /* alpha = -1: alpha*temp1 + conjg(alpha)*temp2 = -(t1 + t2) */
          if (i == j) {
            d[0] = d[0] + (-(t1r + t2r));
            d[1] = 0.0;
          } else {
            d[0] = d[0] + (-t1r - t2r);
            d[1] = d[1] + (-t1i - t2i);
          }
        }
    }
    /* coreValeCoreCore: valeCore(ci, v) = sum_c conj(S(c, v)) * CC(c, ci) */
    double *vc = malloc(sizeof(double) * 2 * (size_t)C * V);
    for (int ci = 0; ci < C; ++ci)
      for (int v = 0; v < V; ++v) {
        double sr = 0, si = 0;
        for (int l = 0; l < C; ++l) {
          const double *a = SCV(l, v), *b = CC(g, c, k, l, ci);
          sr += a[0] * b[0] + a[1] * b[1];
          si += a[0] * b[1] - a[1] * b[0];
        }
        vc[2 * ((size_t)v * C + ci)] = sr;
        vc[2 * ((size_t)v * C + ci) + 1] = si;
      }
    /* makeValeVale: VV(j,i) += sum_c valeCore(c,j) * S(c,i), pack, 1e-10 */
    size_t idx = 0;
    for (int i = 0; i < V; ++i)
      for (int j = 0; j <= i; ++j, ++idx) {
        double sr = 0, si = 0;
        for (int l = 0; l < C; ++l) {
          const double *a = vc + 2 * ((size_t)j * C + l), *b = SCV(l, i);
          sr += a[0] * b[0] - a[1] * b[1];
          si += a[0] * b[1] + a[1] * b[0];
        }
        double *d = VV(g, c, k, j, i);
        d[0] = d[0] + sr;
        d[1] = d[1] + si;
        double re = d[0], im = d[1];
        if (fabs(re) < 1.0e-10) re = 0.0;
        if (fabs(im) < 1.0e-10) im = 0.0;
        out[2 * idx] = re;
        out[2 * idx + 1] = im;
      }
    free(vc);
#undef SCV
  }
}

static int alloc_gmats(const orc_ctx *c, gmats *g) {
  size_t V = c->vale_dim, C = c->core_dim, nk = c->nk;
  g->vv = calloc(2 * nk * V * V, sizeof(double));
  g->cv = calloc(2 * nk * V * (C ? C : 1), sizeof(double));
  g->cc = calloc(2 * nk * (C ? C * C : 1), sizeof(double));
  if (!g->vv || !g->cv || !g->cc) {
    free(g->vv); free(g->cv); free(g->cc);
    return IMAGO_ERR_NOMEM;
  }
  return IMAGO_OK;
}

static void free_gmats(gmats *g) {
  free(g->vv);
  free(g->cv);
  free(g->cc);
}

static int build_one(orc_ctx *c, const buildspec *bs, double *packed,
                     double *cv_re, double *cv_im) {
  if (bs->kind != K_OL && c->core_dim > 0 && !c->have_ol)
    return IMAGO_ERR_NEED_OVERLAP;
  gmats g;
  int st = alloc_gmats(c, &g);
  if (st) return st;
  double t0 = now_s();
  st = pair_loops(c, bs, &g);
  double t1 = now_s();
  c->t_loops += t1 - t0;
  if (st) { free_gmats(&g); return st; }
  if (bs->kind == K_OL) {
    /* coreValeOL is kept for the other matrices (integrals.F90:3686) */
    size_t n = 2 * (size_t)c->nk * c->vale_dim * c->core_dim;
    if (n) memcpy(c->s_cv, g.cv, n * sizeof(double));
    c->have_ol = 1;
    if (cv_re && cv_im)
      for (size_t q = 0; q < n / 2; ++q) {
        cv_re[q] = g.cv[2 * q];
        cv_im[q] = g.cv[2 * q + 1];
      }
  }
  if (!c->skip_ortho) ortho_pack(c, &g, bs->kind == K_OL, packed);
  c->t_ortho += now_s() - t1;
  free_gmats(&g);
  return IMAGO_OK;
}

static void reset_stats(orc_ctx *c) {
  c->t_loops = c->t_ortho = 0.0;
  c->n_pair_images = c->n_shell_pairs = c->n_triples = 0;
}

/* ortho3Terms(8) (integrals3Terms.F90:1388-1608 with intgOrtho.F90
 * valeCoreCoreVale / makeValeVale, fullFlag 1): on the full matrix,
 *   W = VV - S^H X_cv - X_cv^H S + S^H X_cc S,
 * no Hermitian form, no diagonal rule, no zeroing; written as the real and
 * imaginary valeVale planes, column-major per k: re[(k*V + col)*V + row]. */
static void ortho_full(orc_ctx *c, gmats *g, double *re, double *im) {
  const int V = c->vale_dim, C = c->core_dim;
  for (int k = 0; k < c->nk; ++k) {
    double *orr = re + (size_t)k * V * V, *oi = im + (size_t)k * V * V;
    if (C == 0) {
      for (int col = 0; col < V; ++col)
        for (int row = 0; row < V; ++row) {
          orr[(size_t)col * V + row] = VV(g, c, k, row, col)[0];
          oi[(size_t)col * V + row] = VV(g, c, k, row, col)[1];
        }
      continue;
    }
    const double *S = c->s_cv + 2 * (size_t)k * V * C;
#define SCV(row, col) (S + 2 * ((size_t)(col) * C + (row)))
    double *vc = malloc(sizeof(double) * 2 * (size_t)C * V);
    for (int ci = 0; ci < C; ++ci)
      for (int v = 0; v < V; ++v) {
        double sr = 0, si = 0;
        for (int l = 0; l < C; ++l) {
          const double *a = SCV(l, v), *b = CC(g, c, k, l, ci);
          sr += a[0] * b[0] + a[1] * b[1];
          si += a[0] * b[1] - a[1] * b[0];
        }
        vc[2 * ((size_t)v * C + ci)] = sr;
        vc[2 * ((size_t)v * C + ci) + 1] = si;
      }
    for (int i = 0; i < V; ++i)
      for (int j = 0; j < V; ++j) {
        double ar = 0, ai = 0, br = 0, bi = 0, cr = 0, cim = 0;
        for (int l = 0; l < C; ++l) {
          const double *sj = SCV(l, j), *xi_ = CV(g, c, k, l, i);
          const double *xj = CV(g, c, k, l, j), *si_ = SCV(l, i);
          ar += sj[0] * xi_[0] + sj[1] * xi_[1];
          ai += sj[0] * xi_[1] - sj[1] * xi_[0];
          br += xj[0] * si_[0] + xj[1] * si_[1];
          bi += xj[0] * si_[1] - xj[1] * si_[0];
          const double *w = vc + 2 * ((size_t)j * C + l);
          cr += w[0] * si_[0] - w[1] * si_[1];
          cim += w[0] * si_[1] + w[1] * si_[0];
        }
        const double *d = VV(g, c, k, j, i);
        orr[(size_t)i * V + j] = (d[0] - ar - br) + cr;
        oi[(size_t)i * V + j] = (d[1] - ai - bi) + cim;
      }
#undef SCV
    free(vc);
  }
}

/* gaussKOverlap + ortho3Terms(8) (integrals3Terms.F90:956-1384): three
 * complex matrices, one per wave vector dK[axis] (the reference's
 * recipVectors(:, axis) / numAxialKPoints(axis)), as real and imaginary
 * full planes [3][nk][V][V]. */
int orc_gauss_koverlap(orc_ctx *c, const double *dk, double *re, double *im) {
  if (c->core_dim > 0 && !c->have_ol) return IMAGO_ERR_NEED_OVERLAP;
  reset_stats(c);
  const size_t vv = (size_t)c->nk * c->vale_dim * c->vale_dim;
  for (int q = 0; q < 3; ++q) {
    gmats g;
    int st = alloc_gmats(c, &g);
    if (st) return st;
    buildspec bs = {K_KOV, 0, 0, NULL, NULL, 0, q, 0, dk + 3 * q};
    st = pair_loops(c, &bs, &g);
    if (!st) ortho_full(c, &g, re + q * vv, im + q * vv);
    free_gmats(&g);
    if (st) return st;
  }
  return IMAGO_OK;
}


int orc_gauss_overlap_ol(orc_ctx *c, double *packed, double *cv_re,
                         double *cv_im) {
  reset_stats(c);
  buildspec bs = {K_OL, 0, 0, NULL, NULL, 0, 0, 0, NULL};
  return build_one(c, &bs, packed, cv_re, cv_im);
}

int orc_gauss_overlap_ke(orc_ctx *c, double *packed) {
  reset_stats(c);
  buildspec bs = {K_KE, 0, 0, NULL, NULL, 0, 0, 0, NULL};
  return build_one(c, &bs, packed, NULL, NULL);
}

/* gaussOverlapMV, integrals.F90:1091-1527: the kinetic build's loops with
 * massVel2CIntg, accumulated negatively, orthogonalised like KE (ortho
 * opcode 5). */
int orc_gauss_overlap_mv(orc_ctx *c, double *packed) {
  reset_stats(c);
  buildspec bs = {K_MV, 0, 0, NULL, NULL, 0, 0, 0, NULL};
  return build_one(c, &bs, packed, NULL, NULL);
}

/* gaussOverlapHamPSCF + orthoHamPSCF, integrals.F90:2860-3606 and
 * 3913-4043: one matrix per spin, each orthogonalised like KE. */
int orc_ham_pscf(orc_ctx *c, int spin, const double *coeffs, int rel,
                 double *packed) {
  if (spin < 1 || spin > 2 || !coeffs) return IMAGO_ERR_INVALID;
  reset_stats(c);
  const size_t np = (size_t)c->vale_dim * (c->vale_dim + 1) / 2;
  for (int q = 0; q < spin; ++q) {
    buildspec bs = {K_HAM, 0, 0, NULL, coeffs, spin, q, rel, NULL};
    int st = build_one(c, &bs, packed + (size_t)q * 2 * np * c->nk, NULL, NULL);
    if (st) return st;
  }
  return IMAGO_OK;
}

/* gaussOverlapMM / gaussOverlapDM + ortho3Terms, integrals3Terms.F90:
 * 64-507, 511-951, 1388-1608: three matrices (x, y, z), each built with the
 * kinetic build's loops and orthogonalised like KE; the momentum matrix
 * takes the -i of applyPhaseFactors runCode 1, so it is Hermitian. */
static int build_vec(orc_ctx *c, int kind, const double *center, double *packed) {
  reset_stats(c);
  const size_t np = (size_t)c->vale_dim * (c->vale_dim + 1) / 2;
  for (int q = 0; q < 3; ++q) {
    buildspec bs = {kind, 0, 0, NULL, NULL, 0, q, 0, center};
    int st = build_one(c, &bs, packed + (size_t)q * 2 * np * c->nk, NULL, NULL);
    if (st) return st;
  }
  return IMAGO_OK;
}

int orc_gauss_overlap_mm(orc_ctx *c, double *packed) {
  return build_vec(c, K_MM, NULL, packed);
}

int orc_gauss_overlap_dm(orc_ctx *c, const double center[3], double *packed) {
  if (!center) return IMAGO_ERR_INVALID;
  return build_vec(c, K_DM, center, packed);
}

int orc_gauss_overlap_np(orc_ctx *c, double *packed) {
  reset_stats(c);
  buildspec bs = {K_NP, 0, 0, NULL, NULL, 0, 0, 0, NULL};
  return build_one(c, &bs, packed, NULL, NULL);
}

/* elecPotGaussOverlap, integrals.F90:2357-2486: per potential type (its
 * first site), the interaction bits start all set, then one build per
 * alpha of the type. */
int orc_elec_pot_gauss_overlap(orc_ctx *c, int term_lo, int term_hi,
                               double *packed) {
  reset_stats(c);
  if (term_lo < 0 || term_hi > c->pot_dim || term_lo > term_hi)
    return IMAGO_ERR_RANGE;
  size_t nb = (size_t)c->ns * c->ns * c->ncell;
  unsigned char *bits = malloc(nb);
  if (!bits) return IMAGO_ERR_NOMEM;
  size_t np = (size_t)c->vale_dim * (c->vale_dim + 1) / 2;
  int st = IMAGO_OK;
  for (int t = 0; t < c->npt && st == IMAGO_OK; ++t) {
    const optype *pt = &c->ptypes[t];
    if (pt->cumul + pt->nalpha <= term_lo || pt->cumul >= term_hi) continue;
    memset(bits, 1, nb);
    for (int j = 0; j < pt->nalpha; ++j) {
      int term = pt->cumul + j;
      if (term >= term_hi) break;
      /* Terms before the sample are not run: their only effect on later
       * terms is the exact skip bits, which leave the values unchanged. */
      if (term < term_lo) continue;
      buildspec bs = {K_EP, t, j, bits, NULL, 0, 0, 0, NULL};
      double l0 = c->t_loops, o0 = c->t_ortho;
      long long a0 = c->n_pair_images, b0 = c->n_shell_pairs, t0 = c->n_triples;
      st = build_one(c, &bs, packed + 2 * np * c->nk * (size_t)(term - term_lo),
                     NULL, NULL);
      (void)l0; (void)o0; (void)a0; (void)b0; (void)t0;
      if (st) break;
    }
  }
  free(bits);
  return st;
}
