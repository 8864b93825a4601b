/* TEST INFRASTRUCTURE (oracle) -- CPU restatement of the BIT treecode hot path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline / reference arm) use
 * this file, and only as the checker or the timed CPU baseline; the shipped library
 * never links it.  Compiled by oracle/Makefile with -O2 -ffp-contract=off.
 *
 * Structure is this project's own (flat node arrays, per-node slot program, recurrences
 * evaluated degree by degree).  Where parity needs it, the floating-point expression of
 * each quantity is the reference's, operation for operation, so the results pin to the
 * reference bit for bit:
 *   tree fields        src/tree3d.cpp:1045-1073 (treeinit), 1099-1127 (treeshrink)
 *   split rule         src/tree3d.cpp:1163-1304 (treedivide), 1345-1551 (treemake)
 *   moments            src/tree3d.cpp:2631-2711 (treemoments)
 *   Coulomb far field  src/tree3d.cpp:4468-4640 (treetaylorpotential), summed to degree
 *                      nterms-1 (the reference's loop also reads moment[nterms], out of
 *                      bounds at :4635; those terms are zero by :2675-2681)
 *   Coulomb traversal  src/tree3d.cpp:4679-4778 (treepotential)
 *   screened far field src/tree3d.cpp:3004-3227 (shielded_treetaylorpot)
 *   screened traversal src/tree3d.cpp:3448-3627 (shielded_treepot)
 *   force              src/tree3d.cpp:456-612,794-808 (treetaylorforce), 851-971
 *                      (treeforce), 73-97 (eval_grad_kernel_reg)
 *   direct sums        src/tree3d.cpp:298-330, 1966-2016
 *   dense GMRES        src/solver.h:157-310
 */
#include "bit_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MT 12          /* coefficient table edge: degrees up to nterms+1 <= 11 */
#define NTERMS_MAX 10  /* nterms <= 10 keeps every index of the force path < MT */
#define EPS_NEAR 1e-14 /* src/constants.h:35 */

int orc_nterms_max(void) { return NTERMS_MAX; }
int orc_num_terms(int n) { return n * (n + 1) * (n + 2) / 6; }

int orc_moment_index(int n, int i, int j, int k) {
  int idx = 0;
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n - a; b++)
      for (int c = 0; c < n - a - b; c++) {
        if (a == i && b == j && c == k) return idx;
        idx++;
      }
  return -1;
}

/* 1/sqrt(2) evaluated as src/tree3d.cpp:1371 does (not sqrt(0.5): one ulp apart). */
double orc_aspect_limit(void) { return 1.0 / sqrt(2.0); }

/* ------------------------------------------------------------------------------------
 * Tree build
 * ----------------------------------------------------------------------------------*/

/* Box-derived fields exactly as treeinit computes them (src/tree3d.cpp:1045-1073). */
static void box_fields(double* f, double x0, double x1, double y0, double y1, double z0,
                       double z1) {
  double x = 0.5 * (x1 + x0), y = 0.5 * (y1 + y0), z = 0.5 * (z1 + z0);
  f[0] = x0; f[1] = x1; f[2] = y0; f[3] = y1; f[4] = z0; f[5] = z1;
  f[6] = x; f[7] = y; f[8] = z;
  f[9] = fabs((x1 - x0) / (y1 - y0));
  f[10] = fabs((x1 - x0) / (z1 - z0));
  f[11] = fabs((y1 - y0) / (z1 - z0));
  x = x1 - x; y = y1 - y; z = z1 - z;
  f[12] = x * x + y * y + z * z;
}

typedef struct {
  int n;         /* members in this slot (0 = slot not created) */
  double f[13];  /* fields after shrinking to the members       */
} slot_t;

typedef struct {
  const double* c[3];
  const int* mem;   /* node's members, ascending original index */
  int nm;
  signed char* lab; /* current slot per member; -1 = still in the parent */
  int maxmemb;
  double lim;
  slot_t s[8];
  const double* pf; /* parent's fields */
} node_ctx;

/* Bisect the members currently labelled `src` at its midpoint along `dir`, like
 * treedivide (src/tree3d.cpp:1163-1304): members with coord <= mid go first; the first
 * non-empty half goes to slot c1, the second (if any) to c2, each shrunk to its bbox.
 * Returns the number of non-empty halves. */
static int bisect(node_ctx* nc, int dir, int src, int c1, int c2) {
  const double* f = src < 0 ? nc->pf : nc->s[src].f;
  const double mid = f[6 + dir];
  const double *X = nc->c[0], *Y = nc->c[1], *Z = nc->c[2], *C = nc->c[dir];
  int cnt[2] = {0, 0};
  double bb[2][6];
  for (int e = 0; e < nc->nm; e++) {
    if (nc->lab[e] != src) continue;
    int j = nc->mem[e];
    int h = (C[j] <= mid) ? 0 : 1;
    double px = X[j], py = Y[j], pz = Z[j];
    if (cnt[h] == 0) {
      bb[h][0] = bb[h][1] = px; bb[h][2] = bb[h][3] = py; bb[h][4] = bb[h][5] = pz;
    } else {
      if (px > bb[h][1]) bb[h][1] = px;
      if (px < bb[h][0]) bb[h][0] = px;
      if (py > bb[h][3]) bb[h][3] = py;
      if (py < bb[h][2]) bb[h][2] = py;
      if (pz > bb[h][5]) bb[h][5] = pz;
      if (pz < bb[h][4]) bb[h][4] = pz;
    }
    cnt[h]++;
  }
  int dst[2], made = 0;
  dst[0] = c1;
  dst[1] = cnt[0] > 0 ? c2 : c1;
  for (int h = 0; h < 2; h++) {
    if (!cnt[h]) continue;
    slot_t* s = &nc->s[dst[h]];
    s->n = cnt[h];
    box_fields(s->f, bb[h][0], bb[h][1], bb[h][2], bb[h][3], bb[h][4], bb[h][5]);
    made++;
  }
  for (int e = 0; e < nc->nm; e++) {
    if (nc->lab[e] != src) continue;
    int j = nc->mem[e];
    nc->lab[e] = (signed char)dst[(C[j] <= mid) ? 0 : 1];
  }
  return made;
}

#define ZSPLIT_OK(S) ((S).f[10] < lim && (S).f[11] < lim && (S).n > nc->maxmemb)

/* The per-node split program of treemake (src/tree3d.cpp:1412-1545), on slots relative
 * to the first free node index.  Fills order[] with the slots in the order the reference
 * records them as children, and returns their number. */
static int split_program(node_ctx* nc, int* order) {
  const double lim = nc->lim;
  const double* P = nc->pf;
  int nchild = 0, nchild2 = 0, ind2;
  for (int s = 0; s < 8; s++) nc->s[s].n = 0;
  if (P[9] > lim && P[10] > lim) {
    int xc = bisect(nc, 0, -1, 0, 1);
    ind2 = xc;
    for (int j = 0; j < xc; j++) {
      order[nchild++] = j;
      slot_t S = nc->s[j];
      if (S.f[9] < lim && S.f[11] > lim && S.n > nc->maxmemb) {
        int yc = bisect(nc, 1, j, j, ind2);
        if (yc == 2) { order[nchild++] = ind2; ind2++; }
        for (int k = 0; k < yc; k++) {
          /* The reference indexes the k-th y-half as numtree+j+k*(nchild2+1)
           * (src/tree3d.cpp:1460); nchild2 counts z-splits made so far in this node, so
           * this can name a sibling.  Reproduced as written. */
          int t = j + k * (nchild2 + 1);
          if (t >= 8 || t >= ind2) continue; /* never-created slot: nummemb == 0 */
          if (ZSPLIT_OK(nc->s[t])) {
            int zc = bisect(nc, 2, t, t, ind2);
            if (zc == 2) { order[nchild++] = ind2; nchild2++; ind2++; }
          }
        }
      } else if (ZSPLIT_OK(nc->s[j])) {
        int zc = bisect(nc, 2, j, j, ind2);
        if (zc == 2) { order[nchild++] = ind2; ind2++; }
      }
    }
  } else if (P[9] < lim && P[11] > lim) {
    int yc = bisect(nc, 1, -1, 0, 1);
    ind2 = yc;
    for (int j = 0; j < yc; j++) {
      order[nchild++] = j;
      if (ZSPLIT_OK(nc->s[j])) {
        int zc = bisect(nc, 2, j, j, ind2);
        if (zc == 2) { order[nchild++] = ind2; ind2++; }
      }
    }
  } else {
    int zc = bisect(nc, 2, -1, 0, 1);
    for (int j = 0; j < zc; j++) order[nchild++] = j;
  }
  return nchild;
}

int orc_tree_build(int n, const double* x, const double* y, const double* z, int maxmemb,
                   int cap, int* nummemb, int* start, int* children, int* level,
                   int* parent, double* fields, int* perm) {
  if (n <= 0 || cap < 1 || maxmemb < 1) return ORC_ERR_INVALID;
  for (int i = 0; i < n; i++)
    if (isnan(x[i]) || isnan(y[i]) || isnan(z[i])) return ORC_ERR_INVALID;
  double mnx = x[0], mxx = x[0], mny = y[0], mxy = y[0], mnz = z[0], mxz = z[0];
  for (int i = 0; i < n; i++) {
    perm[i] = i;
    if (mnx > x[i]) mnx = x[i];
    if (mxx < x[i]) mxx = x[i];
    if (mny > y[i]) mny = y[i];
    if (mxy < y[i]) mxy = y[i];
    if (mnz > z[i]) mnz = z[i];
    if (mxz < z[i]) mxz = z[i];
  }
  box_fields(fields, mnx, mxx, mny, mxy, mnz, mxz);
  nummemb[0] = n; start[0] = 0; level[0] = 0; parent[0] = -1;
  for (int c = 0; c < 8; c++) children[c] = -1;

  signed char* lab = (signed char*)malloc((size_t)n);
  int* tmp = (int*)malloc(sizeof(int) * (size_t)n);
  int* snap = (int*)malloc(sizeof(int) * (size_t)n);
  node_ctx nc;
  nc.c[0] = x; nc.c[1] = y; nc.c[2] = z;
  nc.maxmemb = maxmemb;
  nc.lim = orc_aspect_limit();
  nc.lab = lab;
  int numtree = 1, rc = 0;
  for (int i = 0; i < numtree; i++) {
    if (nummemb[i] <= maxmemb) continue;
    memcpy(snap, perm + start[i], sizeof(int) * (size_t)nummemb[i]);
    nc.mem = snap; /* the children are written back over the parent's range */
    nc.nm = nummemb[i];
    nc.pf = fields + 13 * (long)i;
    memset(lab, -1, (size_t)nc.nm);
    int order[8];
    int nchild = split_program(&nc, order);
    if (nchild == 1) { rc = ORC_ERR_DEGENERATE; break; } /* the reference never ends */
    if (numtree + nchild > cap) { rc = ORC_ERR_CAPACITY; break; }
    /* lay the children out in slot order; members keep ascending order */
    int off = start[i];
    for (int s = 0; s < nchild; s++) {
      int node = numtree + s;
      nummemb[node] = nc.s[s].n;
      start[node] = off;
      level[node] = level[i] + 1;
      parent[node] = i;
      memcpy(fields + 13 * (long)node, nc.s[s].f, sizeof(double) * 13);
      for (int c = 0; c < 8; c++) children[8 * (long)node + c] = -1;
      int w = 0;
      for (int e = 0; e < nc.nm; e++)
        if (lab[e] == s) tmp[w++] = nc.mem[e];
      off += w;
      memcpy(perm + start[node], tmp, sizeof(int) * (size_t)w);
    }
    for (int c = 0; c < 8; c++) children[8 * (long)i + c] = c < nchild ? numtree + order[c] : -1;
    numtree += nchild;
  }
  free(lab);
  free(tmp);
  free(snap);
  return rc ? rc : numtree;
}

/* ------------------------------------------------------------------------------------
 * Moments (src/tree3d.cpp:2631-2711): M_ijk = sum q dx^i dy^j dz^k, i+j+k < nterms,
 * about the box midpoint, accumulated member by member in ascending member order with
 * the reference's running products.
 * ----------------------------------------------------------------------------------*/
static int cmp_int(const void* a, const void* b) {
  int u = *(const int*)a, v = *(const int*)b;
  return (u > v) - (u < v);
}

void orc_moments(const orc_tree_view* t, double* mom) {
  const int nt = t->nterms, T = orc_num_terms(nt);
#pragma omp parallel for schedule(dynamic, 1)
  for (int ind = 0; ind < t->numtree; ind++) {
    double* M = mom + (long)T * ind;
    for (int a = 0; a < T; a++) M[a] = 0.0;
    int nm = t->nummemb[ind];
    int* mem = (int*)malloc(sizeof(int) * (size_t)nm);
    memcpy(mem, t->perm + t->start[ind], sizeof(int) * (size_t)nm);
    qsort(mem, (size_t)nm, sizeof(int), cmp_int);
    const double* f = t->fields + 13 * (long)ind;
    for (int e = 0; e < nm; e++) {
      int j = mem[e];
      double dx = t->x[j] - f[6], dy = t->y[j] - f[7], dz = t->z[j] - f[8];
      double mult = t->q[j], ymul = mult, xmul = mult;
      int idx = 0;
      for (int i = 0; i < nt; i++) {
        for (int jj = 0; jj < nt - i; jj++) {
          for (int k = 0; k < nt - i - jj; k++) {
            M[idx++] += mult;
            mult *= dz;
          }
          ymul *= dy;
          mult = ymul;
        }
        xmul *= dx;
        ymul = xmul;
        mult = xmul;
      }
    }
    free(mem);
  }
}

/* ------------------------------------------------------------------------------------
 * Far-field coefficient recurrences, evaluated degree by degree.  Each coefficient is
 * computed by the expression the reference uses for its index pattern; every operand
 * has lower total degree, so the order of evaluation does not change any value.
 * ----------------------------------------------------------------------------------*/
typedef double tab_t[MT][MT][MT];

static inline double shift(tab_t T, const int* v, int axis, int by) {
  int w[3] = {v[0], v[1], v[2]};
  w[axis] -= by;
  return T[w[0]][w[1]][w[2]];
}

/* treetaylorpotential coefficient for index v (src/tree3d.cpp:4484-4629). */
static double coul_entry(tab_t b, const int* v, const double* d, double fac, double sqfac) {
  int nz = 0, n1 = 0, ax[3], na = 0;
  for (int a = 0; a < 3; a++) {
    if (v[a] == 0) nz++;
    else ax[na++] = a;
    if (v[a] == 1) n1++;
  }
  if (nz == 3) return sqfac;
  if (nz == 2) {
    int u = ax[0], k = v[u];
    if (k == 1) return fac * d[u] * sqfac;
    double ik = 1.0 / k;
    return fac * (2.0 - ik) * shift(b, v, u, 1) * d[u] - fac * (1 - ik) * shift(b, v, u, 2);
  }
  if (nz == 1 && n1 == 2) { /* (1,1,0) family: :4510-4517 */
    int u = ax[0], w = ax[1];
    return fac * d[u] * shift(b, v, u, 1) + fac * 2.0 * d[w] * shift(b, v, w, 1);
  }
  if (nz == 1 && n1 == 0) { /* (i,j,0) family, i,j >= 2: :4547-4565 */
    int u = ax[0], w = ax[1];
    double ii = 1.0 / v[u];
    return fac * (d[u] * (2.0 - ii) * shift(b, v, u, 1) + 2.0 * d[w] * shift(b, v, w, 1) -
                  (1 - ii) * shift(b, v, u, 2) - shift(b, v, w, 2));
  }
  if (n1 >= 1) { /* one index 1 with others nonzero-or-zero: :4519-4543, 4572-4614 */
    int f = -1;
    for (int a = 0; a < 3; a++)
      if (v[a] == 1) { f = a; break; }
    double s = d[f] * shift(b, v, f, 1);
    for (int a = 0; a < 3; a++)
      if (a != f && v[a] > 0) s = s + 2.0 * d[a] * shift(b, v, a, 1);
    for (int a = 0; a < 3; a++)
      if (a != f && v[a] >= 2) s = s - shift(b, v, a, 2);
    return fac * s;
  }
  /* all indices >= 2: :4617-4629 */
  double ii = 1.0 / v[0];
  return fac * (2.0 * d[0] * (1 - 0.5 * ii) * shift(b, v, 0, 1) + 2.0 * d[1] * shift(b, v, 1, 1) +
                2.0 * d[2] * shift(b, v, 2, 1) - (1.0 - ii) * shift(b, v, 0, 2) -
                shift(b, v, 1, 2) - shift(b, v, 2, 2));
}

static void coul_far(int nterms, double dx, double dy, double dz, double rs, const double* M,
                     double* pot) {
  tab_t b;
  const double d[3] = {dx, dy, dz};
  double fac = 1.0 / rs, sqfac = sqrt(fac);
  for (int deg = 0; deg < nterms; deg++)
    for (int i = deg; i >= 0; i--)
      for (int j = deg - i; j >= 0; j--) {
        int v[3] = {i, j, deg - i - j};
        b[i][j][deg - i - j] = coul_entry(b, v, d, fac, sqfac);
      }
  /* sum order of src/tree3d.cpp:4632-4638 (z outer, then y, then x) */
  for (int m = 0; m < nterms; m++)
    for (int k = 0; k < nterms - m; k++)
      for (int i = 0; i < nterms - m - k; i++)
        *pot += M[orc_moment_index(nterms, i, k, m)] * b[i][k][m];
}

/* shielded_treetaylorpot coefficients (src/tree3d.cpp:3042-3214). */
typedef struct {
  double fac, kappa, cf1[MT], cf2[MT], cf3[MT];
  double d[3], dd[3], kd[3];
} scr_ctx;

static void scr_entry(tab_t A, tab_t B, const int* v, const scr_ctx* c) {
  int nz = 0, n1 = 0, ax[3], na = 0;
  for (int a = 0; a < 3; a++) {
    if (v[a] == 0) nz++;
    else ax[na++] = a;
    if (v[a] == 1) n1++;
  }
  double a_, b_;
  if (nz == 3) return; /* set by the caller */
  if (n1 == 0) {
    /* only indices 0 or >= 2: :3075-3086, 3131-3147, 3203-3214 */
    int u = ax[0], i = v[u];
    b_ = c->cf1[i] * c->kappa * (c->d[u] * shift(A, v, u, 1) - shift(A, v, u, 2));
    double s = c->dd[u] * c->cf2[i] * shift(A, v, u, 1);
    for (int q = 1; q < na; q++) s = s + c->dd[ax[q]] * shift(A, v, ax[q], 1);
    s = s - c->cf3[i] * shift(A, v, u, 2);
    for (int q = 1; q < na; q++) s = s - shift(A, v, ax[q], 2);
    a_ = c->fac * (s + c->cf1[i] * c->kappa * (c->d[u] * shift(B, v, u, 1) - shift(B, v, u, 2)));
  } else if (nz == 2) {
    /* single index 1: :3066-3072 */
    int u = ax[0];
    b_ = c->kd[u] * A[0][0][0];
    a_ = c->fac * c->d[u] * (A[0][0][0] + c->kappa * B[0][0][0]);
  } else {
    /* at least one 1 and two nonzero indices: :3094-3122, 3156-3193 */
    int f = -1;
    for (int a = 0; a < 3; a++)
      if (v[a] == 1) { f = a; break; }
    b_ = c->kd[f] * shift(A, v, f, 1);
    double s = c->d[f] * shift(A, v, f, 1);
    for (int a = 0; a < 3; a++)
      if (a != f && v[a] > 0) s = s + c->dd[a] * shift(A, v, a, 1);
    for (int a = 0; a < 3; a++)
      if (a != f && v[a] >= 2) s = s - shift(A, v, a, 2);
    a_ = c->fac * (s + c->kd[f] * shift(B, v, f, 1));
  }
  A[v[0]][v[1]][v[2]] = a_;
  B[v[0]][v[1]][v[2]] = b_;
}

/* ------------------------------------------------------------------------------------
 * Traversal (treepotential / shielded_treepot)
 * ----------------------------------------------------------------------------------*/
typedef struct {
  const orc_tree_view* t;
  const orc_params* prm;
  int p;
  double x, y, z;
  double pot;
  long long nfar, nnear, nleaf;
  int* lnode; int* lkind; int lcap, ln; /* optional list capture */
  int count_only;
} walk_t;

static void record(walk_t* w, int node, int kind) {
  if (w->lnode && w->ln < w->lcap) { w->lnode[w->ln] = node; w->lkind[w->ln] = kind; }
  w->ln++;
}

static void near_leaf(walk_t* w, int ind) {
  const orc_tree_view* t = w->t;
  const orc_params* P = w->prm;
  const int reference = P->mode == ORC_MODE_REFERENCE;
  const int* mem = t->perm + t->start[ind];
  const int nm = t->nummemb[ind];
  w->nleaf++;
  record(w, ind, 1);
  for (int e = 0; e < nm; e++) {
    int j = mem[e];
    if (w->p != -1 && j == w->p) {
      if (P->kernel == ORC_SCREENED && reference && !w->count_only)
        w->pot += t->q[j] * P->intg / (t->w ? t->w[j] : 1.0); /* :3575-3596 */
      continue;
    }
    w->nnear++;
    if (w->count_only) continue;
    double dx = w->x - t->x[j], dy = w->y - t->y[j], dz = w->z - t->z[j];
    if (P->kernel == ORC_COULOMB) {
      /* :4744-4772 -- particle targets drop DEL in reference mode (:4765) */
      double temp = (w->p == -1 || !reference) ? dx * dx + dy * dy + dz * dz + P->del
                                               : dx * dx + dy * dy + dz * dz;
      double r = sqrt(temp);
      if (temp > EPS_NEAR) w->pot += t->q[j] / (r);
    } else if (P->kernel == ORC_SCREENED) {
      double rs = dx * dx + dy * dy + dz * dz;
      double r = sqrt(rs);
      if (w->p == -1) {
        if (rs > EPS_NEAR) {
          if (reference) w->pot += t->q[j] * exp(-P->kappa * r) / r; /* :3558 */
          else w->pot -= t->q[j] * exp(-P->kappa * r) / r;
        }
      } else {
        w->pot -= t->q[j] * exp(-P->kappa * r) / r; /* :3619 */
      }
    } else {
      double rs = dx * dx + dy * dy + dz * dz + P->del;
      double r = sqrt(rs);
      if (rs > EPS_NEAR) w->pot += t->q[j] * exp(-P->kappa * r) / r;
    }
  }
}

static void far_cluster(walk_t* w, int ind, double dx, double dy, double dz, double rs) {
  const orc_tree_view* t = w->t;
  const orc_params* P = w->prm;
  w->nfar++;
  record(w, ind, 0);
  if (w->count_only) return;
  const int nt = t->nterms;
  const double* M = t->mom + (long)orc_num_terms(nt) * ind;
  if (P->kernel == ORC_COULOMB) {
    coul_far(nt, dx, dy, dz, rs, M, &w->pot);
  } else {
    tab_t A, B;
    /* recompute into local tables (scr_far_sum keeps them on its frame) */
    scr_ctx c;
    double dist = rs;
    c.d[0] = dx; c.d[1] = dy; c.d[2] = dz;
    c.dd[0] = 2 * dx; c.dd[1] = 2 * dy; c.dd[2] = 2 * dz;
    c.kd[0] = P->kappa * dx; c.kd[1] = P->kappa * dy; c.kd[2] = P->kappa * dz;
    c.kappa = P->kappa;
    c.fac = 1.0 / dist;
    dist = sqrt(dist);
    for (int i = 1; i < MT; i++) {
      c.cf1[i] = 1.0 / i;
      c.cf2[i] = 1.0 - c.cf1[i] / 2.0;
      c.cf3[i] = 1.0 - c.cf1[i];
    }
    B[0][0][0] = exp(-P->kappa * dist);
    A[0][0][0] = B[0][0][0] / dist;
    for (int deg = 1; deg < nt; deg++)
      for (int i = deg; i >= 0; i--)
        for (int j = deg - i; j >= 0; j--) {
          int v[3] = {i, j, deg - i - j};
          scr_entry(A, B, v, &c);
        }
    /* :3219-3225 -- the screened potential is accumulated with a minus sign; the
     * regularised-screened kernel (not in the reference) with a plus sign. */
    for (int m = 0; m < nt; m++)
      for (int k = 0; k < nt - m; k++)
        for (int i = 0; i < nt - m - k; i++) {
          double term = M[orc_moment_index(nt, i, k, m)] * A[i][k][m];
          if (P->kernel == ORC_SCREENED) w->pot -= term;
          else w->pot += term;
        }
  }
}

static void walk(walk_t* w, int ind) {
  const orc_tree_view* t = w->t;
  const orc_params* P = w->prm;
  const double* f = t->fields + 13 * (long)ind;
  double dx = w->x - f[6], dy = w->y - f[7], dz = w->z - f[8];
  double add = (P->kernel == ORC_SCREENED) ? 0.0 : P->del;
  double sub = (P->kernel == ORC_SCREENED) ? P->mac_del : P->del;
  double rs = P->kernel == ORC_SCREENED ? dx * dx + dy * dy + dz * dz
                                        : dx * dx + dy * dy + dz * dz + add;
  if (f[12] < P->acc * (rs - sub)) { /* :4691 / :3473 */
    far_cluster(w, ind, dx, dy, dz, rs);
    return;
  }
  int go = 1;
  for (int c = 0; c < 8; c++) {
    int ch = t->children[8 * (long)ind + c];
    if (ch != -1) { go = 0; walk(w, ch); }
  }
  if (go) near_leaf(w, ind);
}

static void target_xyz(const orc_tree_view* t, int pi, const double* tx, const double* ty,
                       const double* tz, int i, double* x, double* y, double* z) {
  if (pi >= 0) { *x = t->x[pi]; *y = t->y[pi]; *z = t->z[pi]; }
  else { *x = tx[i]; *y = ty[i]; *z = tz[i]; }
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

void orc_eval(const orc_tree_view* t, const orc_params* prm, int nt, const int* p,
              const double* tx, const double* ty, const double* tz, double* pot,
              int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    walk_t w;
    memset(&w, 0, sizeof w);
    w.t = t; w.prm = prm; w.p = p ? p[i] : -1;
    target_xyz(t, w.p, tx, ty, tz, i, &w.x, &w.y, &w.z);
    walk(&w, 0);
    pot[i] = w.pot;
  }
}

void orc_count(const orc_tree_view* t, const orc_params* prm, int nt, const int* p,
               const double* tx, const double* ty, const double* tz, long long* nfar,
               long long* nnear_pairs, long long* nnear_leaves, int nthreads) {
  long long a = 0, b = 0, c = 0;
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : a, b, c)
  for (int i = 0; i < nt; i++) {
    walk_t w;
    memset(&w, 0, sizeof w);
    w.t = t; w.prm = prm; w.p = p ? p[i] : -1; w.count_only = 1;
    target_xyz(t, w.p, tx, ty, tz, i, &w.x, &w.y, &w.z);
    walk(&w, 0);
    a += w.nfar; b += w.nnear; c += w.nleaf;
  }
  *nfar = a; *nnear_pairs = b; *nnear_leaves = c;
}

int orc_target_lists(const orc_tree_view* t, const orc_params* prm, int p, double x,
                     double y, double z, int* node, int* kind, int cap) {
  walk_t w;
  memset(&w, 0, sizeof w);
  w.t = t; w.prm = prm; w.p = p; w.x = x; w.y = y; w.z = z;
  w.count_only = 1; w.lnode = node; w.lkind = kind; w.lcap = cap;
  walk(&w, 0);
  return w.ln;
}

/* ------------------------------------------------------------------------------------
 * Force path (treeforce / treetaylorforce / eval_grad_kernel_reg), KERNEL_ORDER = 0
 * far field; near field with the KERNEL_ORDER family of src/tree3d.cpp:88-91.
 * ----------------------------------------------------------------------------------*/
static double force_entry(tab_t b, const int* v, const double* d, double fac, double sqfac) {
  int nz = 0, n1 = 0, ax[3], na = 0;
  for (int a = 0; a < 3; a++) {
    if (v[a] == 0) nz++;
    else ax[na++] = a;
    if (v[a] == 1) n1++;
  }
  int deg = v[0] + v[1] + v[2];
  if (nz == 3) return sqfac;
  if (nz == 2) { /* :475-488 */
    int u = ax[0], k = v[u];
    if (k == 1) return -fac * d[u] * sqfac;
    double ik = 1.0 / k;
    return fac * ((ik - 2.0) * shift(b, v, u, 1) * d[u] + (ik - 1.0) * shift(b, v, u, 2));
  }
  if (nz == 1 && n1 == 2) { /* :491-496 */
    int u = ax[0], w = ax[1];
    return -1.5 * fac * (d[u] * shift(b, v, u, 1) + d[w] * shift(b, v, w, 1));
  }
  if (nz == 1 && n1 == 1) { /* :498-522 */
    int k = deg - 1, u = ax[0], w = ax[1];
    return fac / (k + 1) * ((-2 * k - 1.0) * (d[u] * shift(b, v, u, 1) + d[w] * shift(b, v, w, 1)) +
                            -k * shift(b, v, v[u] >= 2 ? u : w, 2));
  }
  if (nz == 1) { /* :526-543 */
    int u = ax[0], w = ax[1], s = v[u] + v[w];
    return fac / s * ((1 - 2 * s) * (d[u] * shift(b, v, u, 1) + d[w] * shift(b, v, w, 1)) +
                      (1 - s) * (shift(b, v, u, 2) + shift(b, v, w, 2)));
  }
  double s3 = d[0] * shift(b, v, 0, 1) + d[1] * shift(b, v, 1, 1) + d[2] * shift(b, v, 2, 1);
  if (n1 == 3) return -5.0 * fac / 3 * s3; /* :549-551 */
  if (n1 == 2) {                           /* :553-571 */
    int w = v[0] >= 2 ? 0 : (v[1] >= 2 ? 1 : 2), i = v[w];
    return fac / (2.0 + i) * ((-3.0 - 2 * i) * s3 + (-1.0 - i) * (shift(b, v, w, 2)));
  }
  if (n1 == 1) { /* :574-597 */
    int f = v[0] == 1 ? 0 : (v[1] == 1 ? 1 : 2);
    int u = f == 0 ? 1 : 0, w = f == 2 ? 1 : 2;
    int s = v[u] + v[w];
    return (fac / (1 + s)) * ((-1.0 - 2 * s) * s3 + (-s) * (shift(b, v, u, 2) + shift(b, v, w, 2)));
  }
  { /* :600-612 */
    int s = deg;
    return (fac / s) * ((1 - 2 * s) * s3 +
                        (1 - s) * (shift(b, v, 0, 2) + shift(b, v, 1, 2) + shift(b, v, 2, 2)));
  }
}

static void force_far(int nterms, double dx, double dy, double dz, double rs, const double* M,
                      double* fx, double* fy, double* fz) {
  tab_t b;
  const double d[3] = {dx, dy, dz};
  double fac = 1.0 / rs, sqfac = sqrt(fac);
  for (int deg = 0; deg <= nterms; deg++)
    for (int i = deg; i >= 0; i--)
      for (int j = deg - i; j >= 0; j--) {
        int v[3] = {i, j, deg - i - j};
        b[i][j][deg - i - j] = force_entry(b, v, d, fac, sqfac);
      }
  for (int m = 0; m < nterms; m++)
    for (int k = 0; k < nterms - m; k++)
      for (int i = 0; i < nterms - m - k; i++) {
        double Mv = M[orc_moment_index(nterms, i, k, m)];
        if ((i + m + k + 1) % 2 == 0) {
          *fx += Mv * b[i + 1][k][m] * (i + 1);
          *fy += Mv * b[i][k + 1][m] * (k + 1);
          *fz += Mv * b[i][k][m + 1] * (m + 1);
        } else {
          *fx -= Mv * b[i + 1][k][m] * (i + 1);
          *fy -= Mv * b[i][k + 1][m] * (k + 1);
          *fz -= Mv * b[i][k][m + 1] * (m + 1);
        }
      }
}

static void grad_reg(double dx, double dy, double dz, double rs, double del, int korder,
                     double* gx, double* gy, double* gz) {
  double r = sqrt(rs);
  double temp = 1.0 / (r * rs);
  double factor = temp;
  for (int ell = 1; ell <= korder; ell++) {
    factor = factor * (ell + 0.5) / ell * del / rs;
    temp += factor;
  }
  *gx = -dx * temp; *gy = -dy * temp; *gz = -dz * temp;
}

typedef struct {
  const orc_tree_view* t;
  double del, acc;
  int korder, p;
  double x, y, z, fx, fy, fz;
} fwalk_t;

static void fwalk(fwalk_t* w, int ind) {
  const orc_tree_view* t = w->t;
  const double* f = t->fields + 13 * (long)ind;
  double dx = w->x - f[6], dy = w->y - f[7], dz = w->z - f[8];
  double rs = dx * dx + dy * dy + dz * dz + w->del;
  if (f[12] < w->acc * (rs - w->del)) { /* :866 */
    force_far(t->nterms, dx, dy, dz, rs, t->mom + (long)orc_num_terms(t->nterms) * ind,
              &w->fx, &w->fy, &w->fz);
    return;
  }
  int go = 1;
  for (int c = 0; c < 8; c++) {
    int ch = t->children[8 * (long)ind + c];
    if (ch != -1) { go = 0; fwalk(w, ch); }
  }
  if (!go) return;
  const int* mem = t->perm + t->start[ind];
  for (int e = 0; e < t->nummemb[ind]; e++) { /* :932-966 */
    int j = mem[e];
    if (w->p != -1 && j == w->p) continue;
    double ex = t->x[j] - w->x, ey = t->y[j] - w->y, ez = t->z[j] - w->z;
    double r2 = ex * ex + ey * ey + ez * ez + w->del;
    double gx, gy, gz;
    grad_reg(ex, ey, ez, r2, w->del, w->korder, &gx, &gy, &gz);
    w->fx += t->q[j] * gx;
    w->fy += t->q[j] * gy;
    w->fz += t->q[j] * gz;
  }
}

void orc_eval_force(const orc_tree_view* t, double del, double acc, int kernel_order, int nt,
                    const int* p, const double* tx, const double* ty, const double* tz,
                    double* fx, double* fy, double* fz, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    fwalk_t w;
    memset(&w, 0, sizeof w);
    w.t = t; w.del = del; w.acc = acc; w.korder = kernel_order; w.p = p ? p[i] : -1;
    target_xyz(t, w.p, tx, ty, tz, i, &w.x, &w.y, &w.z);
    fwalk(&w, 0);
    fx[i] = w.fx; fy[i] = w.fy; fz[i] = w.fz;
  }
}

/* ------------------------------------------------------------------------------------
 * Direct sums (the FP64 accuracy oracle), same kernel conventions as the traversal in
 * consistent mode: Coulomb sum q/sqrt(r^2+del) skipping r^2+del <= eps; screened
 * -sum q e^{-kr}/r (src/tree3d.cpp:1966-2016); regularised screened +sum q e^{-kR}/R.
 * ----------------------------------------------------------------------------------*/
void orc_direct(int n, const double* x, const double* y, const double* z, const double* q,
                const orc_params* P, int nt, const int* p, const double* tx,
                const double* ty, const double* tz, double* pot, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int pi = p ? p[i] : -1;
    double X = pi >= 0 ? x[pi] : tx[i], Y = pi >= 0 ? y[pi] : ty[i], Z = pi >= 0 ? z[pi] : tz[i];
    double acc = 0.0;
    for (int j = 0; j < n; j++) {
      if (j == pi) continue;
      double dx = X - x[j], dy = Y - y[j], dz = Z - z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (P->kernel == ORC_COULOMB) {
        r2 += P->del;
        if (r2 > EPS_NEAR) acc += q[j] / sqrt(r2);
      } else if (P->kernel == ORC_SCREENED) {
        if (pi == -1 && !(r2 > EPS_NEAR)) continue;
        double r = sqrt(r2);
        acc += q[j] * exp(-P->kappa * r) / r;
      } else {
        r2 += P->del;
        if (r2 > EPS_NEAR) {
          double r = sqrt(r2);
          acc += q[j] * exp(-P->kappa * r) / r;
        }
      }
    }
    pot[i] = P->kernel == ORC_SCREENED ? -acc : acc;
  }
}

void orc_direct_force(int n, const double* x, const double* y, const double* z,
                      const double* q, double del, int kernel_order, int nt, const int* p,
                      double* fx, double* fy, double* fz, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int ind = p[i];
    double a = 0, b = 0, c = 0;
    for (int j = 0; j < n; j++) {
      if (j == ind) continue;
      double dx = x[j] - x[ind], dy = y[j] - y[ind], dz = z[j] - z[ind];
      double rs = dx * dx + dy * dy + dz * dz + del;
      double gx, gy, gz;
      grad_reg(dx, dy, dz, rs, del, kernel_order, &gx, &gy, &gz);
      a += q[j] * gx; b += q[j] * gy; c += q[j] * gz;
    }
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
}

/* ------------------------------------------------------------------------------------
 * GMRES
 * ----------------------------------------------------------------------------------*/

/* solver::gmres (src/solver.h:157-260) with minimize() (:266-310): full GMRES from x=0,
 * modified Gram-Schmidt Arnoldi, least squares by Gram-Schmidt QR of the Hessenberg,
 * stop when the max relative change of x is below 1e-5 (checked every odd step). */
int orc_gmres_dense_ref(int n, const double* A, const double* b, double* x) {
  const int ld = n + 2;
  double* Q = (double*)calloc((size_t)n * ld, sizeof(double));  /* Q[i*ld + j] */
  double* H = (double*)calloc((size_t)(n + 2) * ld, sizeof(double));
  double* V2 = (double*)calloc((size_t)(n + 2) * ld, sizeof(double));
  double* Q2 = (double*)calloc((size_t)(n + 2) * ld, sizeof(double));
  double* R2 = (double*)calloc((size_t)(n + 2) * ld, sizeof(double));
  double* v = (double*)calloc((size_t)n, sizeof(double));
  double* yv = (double*)calloc((size_t)ld, sizeof(double));
#define QQ(i, j) Q[(long)(i) * ld + (j)]
#define HH(i, j) H[(long)(i) * ld + (j)]
#define VV(i, j) V2[(long)(i) * ld + (j)]
#define QT(i, j) Q2[(long)(i) * ld + (j)]
#define RR(i, j) R2[(long)(i) * ld + (j)]
  double bnorm = 0.0;
  for (int i = 0; i < n; i++) bnorm += b[i] * b[i];
  bnorm = sqrt(bnorm);
  for (int i = 0; i < n; i++) QQ(i, 0) = b[i] / bnorm;
  int go = 1, nn = 0, breakdown = 0;
  while (go) {
    int n1 = nn + 1;
    for (int i = 0; i < n; i++) {
      v[i] = 0.0;
      for (int j = 0; j < n; j++) v[i] += A[(long)i * n + j] * QQ(j, nn);
    }
    for (int j = 0; j < n1; j++) {
      HH(j, nn) = 0.0;
      for (int i = 0; i < n; i++) HH(j, nn) += QQ(i, j) * v[i];
      for (int i = 0; i < n; i++) v[i] -= HH(j, nn) * QQ(i, j);
    }
    double temp = 0.0;
    for (int i = 0; i < n; i++) temp += v[i] * v[i];
    HH(n1, nn) = sqrt(temp);
    if (n1 < n && HH(n1, nn) < 1e-14) { go = 0; breakdown = 1; }
    for (int i = 0; i < n; i++) QQ(i, n1) = v[i] / HH(n1, nn);
    /* minimize(n1) */
    {
      int m = n1;
      for (int j = 0; j < m; j++)
        for (int i = 0; i < j + 2; i++) VV(i, j) = HH(i, j);
      for (int i = 0; i < m; i++) {
        int ind = i + 2;
        RR(i, i) = 0;
        for (int k = 0; k < ind; k++) RR(i, i) += VV(k, i) * VV(k, i);
        RR(i, i) = sqrt(RR(i, i));
        for (int k = 0; k < ind; k++) QT(k, i) = VV(k, i) / RR(i, i);
        for (int j = i + 1; j < m; j++) {
          RR(i, j) = 0.0;
          for (int k = 0; k < ind; k++) RR(i, j) += QT(k, i) * VV(k, j);
          for (int k = 0; k < ind; k++) VV(k, j) -= RR(i, j) * QT(k, i);
        }
      }
      for (int i = m - 1; i > -1; i--) {
        yv[i] = bnorm * QT(0, i);
        for (int j = i + 1; j < m; j++) yv[i] -= RR(i, j) * yv[j];
        yv[i] /= RR(i, i);
      }
    }
    if (n1 == n) go = 0;
    if (n1 % 2 || !go) {
      double maxerror = 0.0;
      for (int i = 0; i < n; i++) {
        double old = x[i];
        x[i] = 0;
        for (int j = 0; j < n1; j++) x[i] += QQ(i, j) * yv[j];
        double error = fabs((old - x[i]) / old);
        if (error > maxerror) maxerror = error;
      }
      if (maxerror < 1e-5 && nn > 1) go = 0;
    }
    nn++;
  }
#undef QQ
#undef HH
#undef VV
#undef QT
#undef RR
  free(Q); free(H); free(V2); free(Q2); free(R2); free(v); free(yv);
  return breakdown ? -1 : nn;
}

/* Matvec of the boundary-integral operator: y = diag*s + K(w*s), K the treecode. */
static void tc_matvec(orc_tree_view* t, double* mom, double* qbuf, const orc_params* P,
                      double diag, const double* wts, const double* s, double* y,
                      int* pidx, int nthreads) {
  for (int i = 0; i < t->n; i++) qbuf[i] = (wts ? wts[i] : 1.0) * s[i];
  t->q = qbuf;
  t->mom = mom;
  orc_moments(t, mom);
  orc_eval(t, P, t->n, pidx, NULL, NULL, NULL, y, nthreads);
  for (int i = 0; i < t->n; i++) y[i] = diag * s[i] + y[i];
}

/* Restarted GMRES(m), Arnoldi by modified Gram-Schmidt, Givens rotations, stopping on
 * the relative residual ||b - A x|| / ||b|| <= tol.  The library's device GMRES is
 * checked against this. */
int orc_gmres_treecode(orc_tree_view* t, double* mom_work, const orc_params* P, double diag,
                       const double* wts, const double* b, double* x, int m, double tol,
                       int maxit, int nthreads, int* iters, double* relres) {
  const int n = t->n;
  double* V = (double*)malloc(sizeof(double) * (size_t)n * (m + 1));
  double* Hm = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
  double *cs = (double*)malloc(sizeof(double) * m), *sn = (double*)malloc(sizeof(double) * m);
  double* g = (double*)malloc(sizeof(double) * (m + 1));
  double* w = (double*)malloc(sizeof(double) * n);
  double* qb = (double*)malloc(sizeof(double) * n);
  double* yv = (double*)malloc(sizeof(double) * m);
  int* pidx = (int*)malloc(sizeof(int) * n);
  const double* q_save = t->q;
  for (int i = 0; i < n; i++) pidx[i] = i;
  double bn = 0;
  for (int i = 0; i < n; i++) bn += b[i] * b[i];
  bn = sqrt(bn);
  int it = 0, conv = 0;
  double rr = 1.0;
  while (it < maxit && !conv) {
    tc_matvec(t, mom_work, qb, P, diag, wts, x, w, pidx, nthreads);
    double beta = 0;
    for (int i = 0; i < n; i++) { w[i] = b[i] - w[i]; beta += w[i] * w[i]; }
    beta = sqrt(beta);
    rr = beta / bn;
    if (rr <= tol) { conv = 1; break; }
    for (int i = 0; i < n; i++) V[i] = w[i] / beta;
    for (int i = 0; i <= m; i++) g[i] = 0;
    g[0] = beta;
    int k;
    for (k = 0; k < m && it < maxit; k++) {
      it++;
      tc_matvec(t, mom_work, qb, P, diag, wts, V + (long)n * k, w, pidx, nthreads);
      for (int j = 0; j <= k; j++) {
        double h = 0;
        const double* vj = V + (long)n * j;
        for (int i = 0; i < n; i++) h += vj[i] * w[i];
        for (int i = 0; i < n; i++) w[i] -= h * vj[i];
        Hm[j * m + k] = h;
      }
      double hn = 0;
      for (int i = 0; i < n; i++) hn += w[i] * w[i];
      hn = sqrt(hn);
      Hm[(k + 1) * m + k] = hn;
      for (int j = 0; j < k; j++) {
        double a = Hm[j * m + k], c2 = Hm[(j + 1) * m + k];
        Hm[j * m + k] = cs[j] * a + sn[j] * c2;
        Hm[(j + 1) * m + k] = -sn[j] * a + cs[j] * c2;
      }
      double a = Hm[k * m + k], c2 = Hm[(k + 1) * m + k];
      double den = sqrt(a * a + c2 * c2);
      cs[k] = den > 0 ? a / den : 1.0;
      sn[k] = den > 0 ? c2 / den : 0.0;
      Hm[k * m + k] = den;
      Hm[(k + 1) * m + k] = 0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      rr = fabs(g[k + 1]) / bn;
      if (hn > 0)
        for (int i = 0; i < n; i++) V[(long)n * (k + 1) + i] = w[i] / hn;
      if (rr <= tol || hn == 0) { k++; break; }
    }
    for (int i = k - 1; i >= 0; i--) {
      double s = g[i];
      for (int j = i + 1; j < k; j++) s -= Hm[i * m + j] * yv[j];
      yv[i] = s / Hm[i * m + i];
    }
    for (int j = 0; j < k; j++)
      for (int i = 0; i < n; i++) x[i] += yv[j] * V[(long)n * j + i];
  }
  /* true residual */
  tc_matvec(t, mom_work, qb, P, diag, wts, x, w, pidx, nthreads);
  double r2 = 0;
  for (int i = 0; i < n; i++) { double d = b[i] - w[i]; r2 += d * d; }
  *relres = sqrt(r2) / bn;
  *iters = it;
  t->q = q_save;
  free(V); free(Hm); free(cs); free(sn); free(g); free(w); free(qb); free(yv); free(pidx);
  return *relres <= tol * 10 ? 0 : 1;
}
