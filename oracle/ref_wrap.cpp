// TEST INFRASTRUCTURE (oracle) -- never part of the shipped library.
//
// C-ABI wrapper around the UNMODIFIED reference treecode (ongbw/bit,
// src/tree3d.cpp + src/solver.h).  The reference sources are not copied: the
// recipe in oracle/Makefile puts the reference's src/ directory on the include
// path and this translation unit includes tree3d.cpp from there.
//
// The reference fixes DEL/ACC/KERNEL_ORDER at compile time in src/problem.h:11-13.
// problem.h is guarded by `problem_h`, so defining that guard here and giving the
// three constants first lets one recipe build one library per DEL value
// (BIT_REF_DEL) without touching the reference tree.
//
// Only tests/, __graft_entry__.smoke() and bench.py's reference arm load the
// resulting oracle/_ref/*.so, and only as the checker / CPU baseline.

#define problem_h 1
const double ACC = 0.5;
#ifndef BIT_REF_DEL
#error "BIT_REF_DEL must be defined by the recipe"
#endif
const double DEL = BIT_REF_DEL;
#ifndef BIT_REF_KORDER
#define BIT_REF_KORDER 0
#endif
const int KERNEL_ORDER = BIT_REF_KORDER;

#include "tree3d.cpp"
// solver's work arrays are private members (src/solver.h:31-42); the GMRES test reads its
// Hessenberg after a solve to count the Arnoldi steps, so this translation unit declares
// the class with public members.  Every header solver.h includes (<cmath>, <iostream>) is
// already included above, so the macro touches only the solver class itself.
#define class struct
#include "solver.h"
#undef class

#include <omp.h>
#include <vector>

namespace {

struct RefTree {
  int n = 0, nterms = 0, maxmemb = 0, numtree = 0, cap = 0, mom_dim = 0;
  PARTICLE* part = nullptr;
  TREE* tree = nullptr;
};

// treemoments() allocates nterms^3 moment arrays when `moments` is NULL
// (src/tree3d.cpp:2660-2669).  treetaylorpotential() reads moment[i][k][m] for
// i+k+m <= nterms (src/tree3d.cpp:4632-4638), one past that allocation.  We
// pre-allocate (nterms+1)^3 zero-filled arrays instead: treemoments() then only
// zeroes/fills the i,j,k < nterms block, and every read of the potential sum
// stays in bounds and sees 0 for degree nterms -- which is the defined meaning
// of those terms (they are never accumulated).  No reference code is changed.
void alloc_padded_moments(RefTree* t) {
  const int d = t->nterms + 1;
  t->mom_dim = d;
  for (int ind = 0; ind < t->numtree; ind++) {
    double*** m = new double**[d];
    for (int i = 0; i < d; i++) {
      m[i] = new double*[d];
      for (int j = 0; j < d; j++) {
        m[i][j] = new double[d];
        for (int k = 0; k < d; k++) m[i][j][k] = 0.0;
      }
    }
    t->tree[ind].moments = m;
  }
}

void free_moments(RefTree* t) {
  if (!t->mom_dim) return;
  for (int ind = 0; ind < t->numtree; ind++) {
    double*** m = t->tree[ind].moments;
    if (!m) continue;
    for (int i = 0; i < t->mom_dim; i++) {
      for (int j = 0; j < t->mom_dim; j++) delete[] m[i][j];
      delete[] m[i];
    }
    delete[] m;
    t->tree[ind].moments = nullptr;
  }
  t->mom_dim = 0;
}

}  // namespace

extern "C" {

double ref_del(void) { return DEL; }
int ref_kernel_order(void) { return KERNEL_ORDER; }

// boxparticles() fixture of the reference tests (src/tree3d.cpp:1698-1740,
// srand(100) + glibc rand()).  Returns x, y, z, tot_charge and weight.
void ref_boxparticles(int n, double dlength, double dheight, double ddepth,
                      double density, double* x, double* y, double* z,
                      double* q, double* w) {
  PARTICLE* p = new PARTICLE[n];
  boxparticles(n, dlength, dheight, ddepth, p, density);
  for (int i = 0; i < n; i++) {
    x[i] = p[i].x; y[i] = p[i].y; z[i] = p[i].z;
    q[i] = p[i].tot_charge; w[i] = p[i].weight;
  }
  delete[] p;
}

// treemake (src/tree3d.cpp:1345) on caller particles.  `cap` TREE slots are
// default-constructed (nummemb = 0, NULL pointers) as the tests do
// (tests/treecode.cpp:24-38).  Returns an opaque handle.
void* ref_tree_build(int n, const double* x, const double* y, const double* z,
                     const double* q, const double* w, int nterms, int maxmemb,
                     int cap) {
  RefTree* t = new RefTree;
  t->n = n; t->nterms = nterms; t->maxmemb = maxmemb; t->cap = cap;
  t->part = new PARTICLE[n];
  for (int i = 0; i < n; i++) {
    PARTICLE& p = t->part[i];
    p.charge = 0; p.u = p.v = p.w = 0; p.xforce = p.yforce = p.zforce = 0;
    p.x = x[i]; p.y = y[i]; p.z = z[i];
    p.tot_charge = q[i];
    p.weight = w ? w[i] : 1.0;
  }
  t->tree = new TREE[cap];
  for (int i = 0; i < cap; i++) { t->tree[i].members = nullptr; t->tree[i].moments = nullptr; }
  t->numtree = treemake(n, nterms, maxmemb, t->part, t->tree);
  return t;
}

int ref_tree_numtree(void* h) { return static_cast<RefTree*>(h)->numtree; }

// Overwrite the charges (e.g. for a new matvec) without touching the tree.
void ref_tree_set_charges(void* h, const double* q) {
  RefTree* t = static_cast<RefTree*>(h);
  for (int i = 0; i < t->n; i++) t->part[i].tot_charge = q[i];
}

// treemoments (src/tree3d.cpp:2631) with padded moment storage.
void ref_tree_moments(void* h) {
  RefTree* t = static_cast<RefTree*>(h);
  if (!t->mom_dim) alloc_padded_moments(t);
  treemoments(t->numtree, t->nterms, t->tree, t->part);
}

// Per node: nummemb, children[8], 13 doubles (x0 x1 y0 y1 z0 z1 xmid ymid zmid
// aspxy aspxz aspyz sqradius) and the member list (concatenated in node order).
void ref_tree_export(void* h, int* nummemb, int* children, double* fields,
                     int* members) {
  RefTree* t = static_cast<RefTree*>(h);
  long off = 0;
  for (int i = 0; i < t->numtree; i++) {
    const TREE& n = t->tree[i];
    nummemb[i] = n.nummemb;
    for (int c = 0; c < NUMCHILD; c++) children[8 * i + c] = n.children[c];
    double* f = fields + 13 * (long)i;
    f[0] = n.x0; f[1] = n.x1; f[2] = n.y0; f[3] = n.y1; f[4] = n.z0; f[5] = n.z1;
    f[6] = n.xmid; f[7] = n.ymid; f[8] = n.zmid;
    f[9] = n.aspectxy; f[10] = n.aspectxz; f[11] = n.aspectyz; f[12] = n.sqradius;
    if (members) {
      for (int j = 0; j < n.nummemb; j++) members[off + j] = n.members[j];
      off += n.nummemb;
    }
  }
}

// Moments of node `ind` as a dense nterms^3 block, [i][j][k] row-major.
void ref_tree_node_moments(void* h, int ind, double* out) {
  RefTree* t = static_cast<RefTree*>(h);
  const int n = t->nterms;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++)
        out[(i * n + j) * n + k] = t->tree[ind].moments[i][j][k];
}

// Targets: p[t] >= 0 is a particle index (coordinates taken from it, self
// handled as the reference does); p[t] == -1 is an external point (tx,ty,tz).
// One OpenMP `parallel for` over targets, as tests/treecode_mp.cpp:83-95.
void ref_eval_potential(void* h, double acc, int nt, const int* p,
                        const double* tx, const double* ty, const double* tz,
                        double* pot, int nthreads) {
  RefTree* t = static_cast<RefTree*>(h);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int pi = p ? p[i] : -1;
    double x = pi >= 0 ? t->part[pi].x : tx[i];
    double y = pi >= 0 ? t->part[pi].y : ty[i];
    double z = pi >= 0 ? t->part[pi].z : tz[i];
    double v = 0.0;
    treepotential(0, pi, t->nterms, x, y, z, acc, &v, t->tree, t->part);
    pot[i] = v;
  }
}

void ref_eval_screened(void* h, double kappa, double acc, int nt, const int* p,
                       const double* tx, const double* ty, const double* tz,
                       double* pot, int nthreads) {
  RefTree* t = static_cast<RefTree*>(h);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int pi = p ? p[i] : -1;
    double x = pi >= 0 ? t->part[pi].x : tx[i];
    double y = pi >= 0 ? t->part[pi].y : ty[i];
    double z = pi >= 0 ? t->part[pi].z : tz[i];
    double v = 0.0;
    // The trailing mesh arguments only feed an unused local (src/tree3d.cpp:3577-3579).
    shielded_treepot(0, pi, t->nterms, x, y, z, kappa, acc, &v, t->tree, t->part,
                     1, 1, 1, 1.0, 1.0, 1.0);
    pot[i] = v;
  }
}

void ref_eval_force(void* h, double acc, int nt, const int* p, const double* tx,
                    const double* ty, const double* tz, double* fx, double* fy,
                    double* fz, int nthreads) {
  RefTree* t = static_cast<RefTree*>(h);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int pi = p ? p[i] : -1;
    double x = pi >= 0 ? t->part[pi].x : tx[i];
    double y = pi >= 0 ? t->part[pi].y : ty[i];
    double z = pi >= 0 ? t->part[pi].z : tz[i];
    double a = 0.0, b = 0.0, c = 0.0;
    treeforce(0, pi, t->nterms, x, y, z, acc, &a, &b, &c, t->tree, t->part);
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
}

void ref_tree_free(void* h) {
  RefTree* t = static_cast<RefTree*>(h);
  if (!t) return;
  free_moments(t);
  for (int i = 0; i < t->numtree; i++) {
    delete[] t->tree[i].members;
    t->tree[i].members = nullptr;
  }
  delete[] t->tree;
  delete[] t->part;
  delete t;
}

// Direct sums (src/tree3d.cpp:298-330, 1966-2016) over all n particles for the
// listed particle targets.
void ref_ds_force_reg(int n, const double* x, const double* y, const double* z,
                      const double* q, int nt, const int* p, double* fx,
                      double* fy, double* fz, int nthreads) {
  std::vector<PARTICLE> part(n);
  for (int i = 0; i < n; i++) {
    part[i].x = x[i]; part[i].y = y[i]; part[i].z = z[i]; part[i].tot_charge = q[i];
  }
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double a = 0, b = 0, c = 0;
    force_particle_ds_reg(p[i], n, part.data(), &a, &b, &c);
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
}

void ref_ds_screened_pot(int n, const double* x, const double* y, const double* z,
                         const double* q, double kappa, int nt, const int* p,
                         double* pot, int nthreads) {
  std::vector<PARTICLE> part(n);
  for (int i = 0; i < n; i++) {
    part[i].x = x[i]; part[i].y = y[i]; part[i].z = z[i]; part[i].tot_charge = q[i];
  }
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double v = 0;
    shielded_pot_particle_ds(p[i], n, part.data(), &v, kappa);
    pot[i] = v;
  }
}

void ref_eval_grad_kernel(double dx, double dy, double dz, double rs, int reg,
                          double* out3) {
  if (reg) eval_grad_kernel_reg(dx, dy, dz, rs, &out3[0], &out3[1], &out3[2]);
  else eval_grad_kernel_noreg(dx, dy, dz, rs, &out3[0], &out3[1], &out3[2]);
}

// solver::gmres (src/solver.h:157-260) on a dense row-major n x n matrix.
// x must hold the caller's initial values (only used by the stopping test).  Returns the
// number of Arnoldi steps taken: gmres() zeroes the (n+2) x (n+1) Hessenberg first
// (:174-177) and step j writes column j, whose subdiagonal h[j+1][j] = |v| is nonzero
// unless v vanished exactly.
int ref_gmres_dense(int n, const double* A, const double* b, double* x) {
  std::vector<double*> rows(n);
  std::vector<double> a(A, A + (long)n * n);
  for (int i = 0; i < n; i++) rows[i] = a.data() + (long)i * n;
  std::vector<double> bb(b, b + n);
  solver s;
  s.makeFram(n + 1);
  s.gmres(rows.data(), bb.data(), x, n);
  int steps = 0;
  for (int j = 0; j < n; j++)
    for (int i = 0; i <= j + 1; i++)
      if (s.h[i][j] != 0.0) steps = j + 1;
  return steps;
}

// shielded_treeforce (src/tree3d.cpp:3268-3408) at particle (p >= 0) or point targets.
void ref_eval_screened_field(void* h, double kappa, double acc, int nt, const int* p,
                             const double* tx, const double* ty, const double* tz,
                             double* fx, double* fy, double* fz, int nthreads) {
  RefTree* t = static_cast<RefTree*>(h);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int pi = p ? p[i] : -1;
    double x = pi >= 0 ? t->part[pi].x : tx[i];
    double y = pi >= 0 ? t->part[pi].y : ty[i];
    double z = pi >= 0 ? t->part[pi].z : tz[i];
    double a = 0.0, b = 0.0, c = 0.0;
    shielded_treeforce(0, pi, t->nterms, x, y, z, kappa, acc, &a, &b, &c, t->tree, t->part);
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
}

// force_particle_ds_noreg (src/tree3d.cpp:182-213) for the listed particle targets.
void ref_ds_force_noreg(int n, const double* x, const double* y, const double* z,
                        const double* q, int nt, const int* p, double* fx, double* fy,
                        double* fz, int nthreads) {
  std::vector<PARTICLE> part(n);
  for (int i = 0; i < n; i++) {
    part[i].x = x[i]; part[i].y = y[i]; part[i].z = z[i]; part[i].tot_charge = q[i];
  }
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double a = 0, b = 0, c = 0;
    force_particle_ds_noreg(p[i], n, part.data(), &a, &b, &c);
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
}

// setboundaries (src/tree3d.cpp:3764-3934): the box's boundary panels, 17 doubles each
// (x0 x1 y0 y1 z0 z1 str xnrm ynrm znrm refpot midx midy midz type orientation area).
// Returns the panel count.
int ref_setboundaries(int xp, int yp, int zp, double dl, double dh, double dd, double* out) {
  const int numpan = 2 * (xp * yp + zp * yp + xp * zp);
  std::vector<PANEL> pan(numpan);
  setboundaries(xp, yp, zp, dl, dh, dd, pan.data());
  for (int i = 0; i < numpan; i++) {
    const PANEL& q = pan[i];
    const double v[17] = {q.x0, q.x1, q.y0, q.y1, q.z0, q.z1, q.str, q.xnrm, q.ynrm, q.znrm,
                          q.refpot, q.midx, q.midy, q.midz, (double)q.type,
                          (double)q.orientation, q.area};
    for (int k = 0; k < 17; k++) out[17L * i + k] = v[k];
  }
  return numpan;
}

// panelconstantsreal (src/tree3d.cpp:4054-4078) on panels from ref_setboundaries; A is
// row-major numpan x numpan.
void ref_panelconstantsreal(int xp, int yp, int zp, double dl, double dh, double dd, double* A) {
  const int numpan = 2 * (xp * yp + zp * yp + xp * zp);
  std::vector<PANEL> pan(numpan);
  setboundaries(xp, yp, zp, dl, dh, dd, pan.data());
  std::vector<double*> rows(numpan);
  for (int i = 0; i < numpan; i++) rows[i] = A + (long)i * numpan;
  panelconstantsreal(numpan, pan.data(), rows.data());
}

// output_potential (src/tree3d.cpp:4918-4937) on caller arrays.
void ref_output_potential(int n, const double* x, const double* y, const double* z,
                          const double* pot, const char* filename) {
  std::vector<PARTICLE> p(n);
  for (int i = 0; i < n; i++) { p[i].x = x[i]; p[i].y = y[i]; p[i].z = z[i]; }
  std::vector<double> pv(pot, pot + n);
  output_potential(n, p.data(), pv.data(), std::string(filename));
}

}  // extern "C"
