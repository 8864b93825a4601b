// libtree3d_b200.so: the reference's tree3d.h / solver.h entry points (include/
// tree3d_b200.h) over the C ABI of bit_b200.h.  Host C++ only; every computation runs in
// libbit_b200.so on the GPU.
#include "tree3d_b200.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "bit_b200.h"

double bit_tree3d_del = 0.01;
double bit_tree3d_mac_del = 0.01;
int bit_tree3d_kernel_order = 0;
int bit_tree3d_precision = 0;

namespace {

// Results of one whole-tree evaluation, valid for exactly the parameters they were computed
// with: a later call with any other acc, kappa, kernel, del, screened MAC offset or
// precision recomputes them (moments reset them, so nterms is covered too).
struct Cached {
  bool valid = false;
  double acc = 0, kappa = 0, del = 0, mac_del = 0;
  int kind = -1;  // 0 coulomb, 1 screened, 2 force, 3 screened field
  int prec = -1, korder = -1;
  std::vector<double> a, b, c;
  bool matches(int k, double ac, double ka) const {
    return valid && kind == k && acc == ac && kappa == ka && del == bit_tree3d_del &&
           mac_del == bit_tree3d_mac_del && prec == bit_tree3d_precision &&
           korder == bit_tree3d_kernel_order;
  }
  void mark(int k, double ac, double ka) {
    valid = true;
    kind = k; acc = ac; kappa = ka;
    del = bit_tree3d_del; mac_del = bit_tree3d_mac_del; prec = bit_tree3d_precision;
    korder = bit_tree3d_kernel_order;
  }
};

struct Entry {
  bit_tree* tree = nullptr;
  int n = 0, nterms = 0;
  int mom_dim = 0;  // edge of the moment arrays this library allocated (0: none)
  std::vector<double> x, y, z;
  Cached pot[2], force, sfield;
};

// Direct sums of one particle array (one per kind): a snapshot of the particles, the
// results of every target, and which targets this sweep has served.
struct DirectSweep {
  bool valid = false;
  int n = 0, korder = 0;
  double param = 0;  // del (force) or alpha (screened)
  std::vector<double> x, y, z, q;
  std::vector<double> a, b, c;
  std::vector<char> served;
};

std::mutex mu;
bit_ctx* g_ctx = nullptr;
std::map<const TREE*, Entry> g_trees;
// kind: 0 force_particle_ds_reg, 1 force_particle_ds_noreg, 2 shielded_pot_particle_ds
std::map<std::pair<const PARTICLE*, int>, DirectSweep> g_direct;
thread_local std::string g_err;

bit_ctx* ctx() {
  if (!g_ctx) {
    bit_ctx_opts o{0, nullptr, 0};
    if (bit_ctx_create(&g_ctx, &o) != BIT_OK) g_ctx = nullptr;
  }
  return g_ctx;
}

// Every failure is reported on stderr as well as through bit_tree3d_last_error(): the
// reference's void entry points give a caller no other way to notice one.
void complain(const std::string& m) {
  g_err = m;
  std::fprintf(stderr, "[tree3d_b200] %s\n", m.c_str());
}

bool ok(bit_status s, const char* what) {
  if (s == BIT_OK) return true;
  g_err = std::string(what) + ": " + bit_status_string(s) + " -- " +
          (g_ctx ? bit_ctx_last_error(g_ctx) : "");
  std::fprintf(stderr, "[tree3d_b200] %s\n", g_err.c_str());
  return false;
}

bit_eval_params prm(int kernel, double acc, double kappa) {
  bit_eval_params p{};
  p.kernel = (bit_kernel)kernel;
  p.mode = BIT_MODE_REFERENCE;
  p.precision = (bit_precision)bit_tree3d_precision;
  p.del = bit_tree3d_del;
  p.mac_del = bit_tree3d_mac_del;
  p.kappa = kappa;
  p.acc = acc;
  p.intg = -0.0000483811229725;  // src/tree3d.cpp:3585
  return p;
}

}  // namespace

const char* bit_tree3d_last_error() { return g_err.c_str(); }

// treemake (src/tree3d.cpp:1345-1551): nodes, boxes, children and member lists written
// into the caller's TREE[] exactly as the reference fills them.
int treemake(int num, int nterms, int maxmemb, PARTICLE* part, TREE* tree) {
  std::lock_guard<std::mutex> lk(mu);
  bit_ctx* c = ctx();
  if (!c) { complain("no CUDA device"); return -1; }
  Entry e;
  e.n = num;
  e.nterms = nterms;
  e.x.resize(num); e.y.resize(num); e.z.resize(num);
  for (int i = 0; i < num; i++) { e.x[i] = part[i].x; e.y[i] = part[i].y; e.z[i] = part[i].z; }
  if (!ok(bit_tree_build(c, num, e.x.data(), e.y.data(), e.z.data(), maxmemb, &e.tree), "treemake"))
    return -1;
  int nt = 0;
  bit_tree_info(e.tree, &nt, nullptr, nullptr);
  std::vector<int> nm(nt), ch(8LL * nt), mem;
  std::vector<double> f(13LL * nt);
  bit_tree_export(e.tree, nm.data(), ch.data(), f.data(), nullptr);
  long long total = 0;
  for (int i = 0; i < nt; i++) total += nm[i];
  mem.resize(total);
  bit_tree_export(e.tree, nullptr, nullptr, nullptr, mem.data());
  long long off = 0;
  for (int i = 0; i < nt; i++) {
    TREE& t = tree[i];
    t.nummemb = nm[i];
    const double* g = &f[13LL * i];
    t.x0 = g[0]; t.x1 = g[1]; t.y0 = g[2]; t.y1 = g[3]; t.z0 = g[4]; t.z1 = g[5];
    t.xmid = g[6]; t.ymid = g[7]; t.zmid = g[8];
    t.aspectxy = g[9]; t.aspectxz = g[10]; t.aspectyz = g[11]; t.sqradius = g[12];
    for (int k = 0; k < NUMCHILD; k++) t.children[k] = ch[8LL * i + k];
    t.members = new int[nm[i]];
    std::memcpy(t.members, &mem[off], nm[i] * sizeof(int));
    off += nm[i];
  }
  auto it = g_trees.find(tree);
  if (it != g_trees.end() && it->second.tree) bit_tree_destroy(it->second.tree);
  g_trees[tree] = std::move(e);
  return nt;
}

// treemoments (src/tree3d.cpp:2631-2711): computed on the GPU and copied into the
// caller's moment arrays (allocated nterms^3 as the reference does when NULL).
void treemoments(int numtree, int nterms, TREE* tree, PARTICLE* part) {
  std::lock_guard<std::mutex> lk(mu);
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { complain("treemoments: tree not built by treemake"); return; }
  Entry& e = it->second;
  std::vector<double> q(e.n), w(e.n);
  for (int i = 0; i < e.n; i++) { q[i] = part[i].tot_charge; w[i] = part[i].weight; }
  if (!ok(bit_tree_set_charges(e.tree, q.data(), w.data()), "treemoments")) return;
  if (!ok(bit_tree_moments(e.tree, nterms), "treemoments")) return;
  e.nterms = nterms;
  e.pot[0] = Cached(); e.pot[1] = Cached(); e.force = Cached(); e.sfield = Cached();
  const int T = nterms * (nterms + 1) * (nterms + 2) / 6;
  std::vector<double> m((size_t)numtree * T);
  if (!ok(bit_tree_export_moments(e.tree, m.data()), "treemoments")) return;
  for (int ind = 0; ind < numtree; ind++) {
    TREE& t = tree[ind];
    if (!t.moments) {
      e.mom_dim = nterms;
      t.moments = new double**[nterms];
      for (int i = 0; i < nterms; i++) {
        t.moments[i] = new double*[nterms];
        for (int j = 0; j < nterms; j++) t.moments[i][j] = new double[nterms];
      }
    }
    int idx = 0;
    for (int i = 0; i < nterms; i++)
      for (int j = 0; j < nterms; j++)
        for (int k = 0; k < nterms; k++) t.moments[i][j][k] = 0.0;
    for (int i = 0; i < nterms; i++)
      for (int j = 0; j < nterms - i; j++)
        for (int k = 0; k < nterms - i - j; k++) t.moments[i][j][k] = m[(size_t)ind * T + idx++];
  }
}

void treeempty(int numtree, TREE* tree) {
  std::lock_guard<std::mutex> lk(mu);
  if (!tree) return;
  auto it = g_trees.find(tree);
  const int dim = it != g_trees.end() ? it->second.mom_dim : 0;
  for (int i = 0; i < numtree; i++) {
    delete[] tree[i].members;
    tree[i].members = nullptr;
    if (tree[i].moments && dim) {
      for (int a = 0; a < dim; a++) {
        for (int b = 0; b < dim; b++) delete[] tree[i].moments[a][b];
        delete[] tree[i].moments[a];
      }
      delete[] tree[i].moments;
      tree[i].moments = nullptr;
    }
  }
  if (it != g_trees.end()) {
    if (it->second.tree) bit_tree_destroy(it->second.tree);
    g_trees.erase(it);
  }
}

static double serve_potential(int kernel, int ind, int p, double x, double y, double z,
                              double kappa, double acc, double* pot, TREE* tree) {
  std::lock_guard<std::mutex> lk(mu);
  if (ind != 0) {
    complain("only ind == 0 (the whole tree) is served on the GPU");
    return -1;
  }
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { complain("tree not built by treemake"); return -1; }
  Entry& e = it->second;
  bit_eval_params P = prm(kernel, acc, kappa);
  const bool same_point = p >= 0 && p < e.n && x == e.x[p] && y == e.y[p] && z == e.z[p];
  if (!same_point) {
    double v = 0.0;
    if (!ok(bit_eval_points(e.tree, &P, 1, &x, &y, &z, &v), "evaluate point")) return -1;
    *pot += v;
    return 0;
  }
  Cached& C = e.pot[kernel == BIT_KERNEL_SCREENED];
  if (!C.matches(kernel, acc, kappa)) {
    C.valid = false;
    C.a.assign(e.n, 0.0);
    if (!ok(bit_eval_particles(e.tree, &P, C.a.data()), "evaluate particles")) return -1;
    C.mark(kernel, acc, kappa);
  }
  *pot += C.a[p];
  return 0;
}

double treepotential(int ind, int p, int nterms, double x, double y, double z, double acc,
                     double* pot, TREE* tree, PARTICLE*) {
  (void)nterms;
  return serve_potential(BIT_KERNEL_COULOMB, ind, p, x, y, z, 0.0, acc, pot, tree);
}

double shielded_treepot(int ind, int p, int nterms, double x, double y, double z, double alpha,
                        double acc, double* pot, TREE* tree, PARTICLE*, int, int, int, double,
                        double, double) {
  (void)nterms;
  return serve_potential(BIT_KERNEL_SCREENED, ind, p, x, y, z, alpha, acc, pot, tree);
}

double treeforce(int ind, int p, int nterms, double x, double y, double z, double acc,
                 double* xfor, double* yfor, double* zfor, TREE* tree, PARTICLE*) {
  (void)nterms;
  std::lock_guard<std::mutex> lk(mu);
  if (ind != 0) { complain("only ind == 0 is served on the GPU"); return -1; }
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { complain("tree not built by treemake"); return -1; }
  Entry& e = it->second;
  if (!(p >= 0 && p < e.n && x == e.x[p] && y == e.y[p] && z == e.z[p])) {
    complain("treeforce at a point that is not the particle p is not supported");
    return -1;
  }
  Cached& C = e.force;
  if (!C.matches(2, acc, 0.0)) {
    C.valid = false;
    C.a.assign(e.n, 0.0); C.b.assign(e.n, 0.0); C.c.assign(e.n, 0.0);
    bit_field_params F{};
    F.kind = BIT_FIELD_COULOMB;
    F.precision = (bit_precision)bit_tree3d_precision;
    F.del = bit_tree3d_del;
    F.acc = acc;
    F.kernel_order = bit_tree3d_kernel_order;
    if (!ok(bit_eval_field(e.tree, &F, C.a.data(), C.b.data(), C.c.data()), "treeforce"))
      return -1;
    C.mark(2, acc, 0.0);
  }
  *xfor += C.a[p]; *yfor += C.b[p]; *zfor += C.c[p];
  return 0;
}

// shielded_treeforce (src/tree3d.cpp:3268-3408): the reference accumulates fx, fy and
// assigns fz = 0 wherever it adds a term.
double shielded_treeforce(int ind, int p, int nterms, double x, double y, double z,
                          double alpha, double acc, double* xfor, double* yfor, double* zfor,
                          TREE* tree, PARTICLE*) {
  (void)nterms;
  std::lock_guard<std::mutex> lk(mu);
  if (ind != 0) { complain("only ind == 0 is served on the GPU"); return -1; }
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { complain("tree not built by treemake"); return -1; }
  Entry& e = it->second;
  if (!(p >= 0 && p < e.n && x == e.x[p] && y == e.y[p] && z == e.z[p])) {
    complain("shielded_treeforce at a point that is not the particle p is not supported");
    return -1;
  }
  Cached& C = e.sfield;
  if (!C.matches(3, acc, alpha)) {
    C.valid = false;
    C.a.assign(e.n, 0.0); C.b.assign(e.n, 0.0); C.c.assign(e.n, 0.0);
    bit_field_params F{};
    F.kind = BIT_FIELD_SCREENED;
    F.precision = (bit_precision)bit_tree3d_precision;
    F.mac_del = bit_tree3d_mac_del;
    F.kappa = alpha;
    F.acc = acc;
    if (!ok(bit_eval_field(e.tree, &F, C.a.data(), C.b.data(), C.c.data()), "shielded_treeforce"))
      return -1;
    C.mark(3, acc, alpha);
  }
  *xfor += C.a[p]; *yfor += C.b[p]; *zfor = 0.0;
  return 0;
}

// shielded_freespace_particles_tree (src/tree3d.cpp:2368-2436)
void shielded_freespace_particles_tree(int npart, PARTICLE* part, double alpha, int nterms,
                                       double acc, TREE* tree, int numtree, int maxmemb) {
  numtree = treemake(npart, nterms, maxmemb, part, tree);
  if (numtree < 0) return;
  treemoments(numtree, nterms, tree, part);
  for (int i = 0; i < npart; i++) {
    double xf = 0, yf = 0, zf = 0;
    if (shielded_treeforce(0, i, nterms, part[i].x, part[i].y, part[i].z, alpha, acc, &xf, &yf,
                           &zf, tree, part))
      return;
    part[i].xforce = xf * charge_constant * part[i].tot_charge;
    part[i].yforce = yf * charge_constant * part[i].tot_charge;
    part[i].zforce = zf * charge_constant * part[i].tot_charge;
  }
  treeempty(numtree, tree);
}

// ---- direct sums ----------------------------------------------------------------------
namespace {

// The sweep of (part, kind) that serves target ind: the current one while ind has not been
// served yet and the target still matches the snapshot, else a fresh GPU evaluation of
// every target from the current particles.  Caller holds mu.
DirectSweep* direct_sweep(int kind, int ind, int npart, PARTICLE* part, double param) {
  if (!part || npart < 1 || ind < 0 || ind >= npart) {
    complain("direct sum: invalid particle index or count");
    return nullptr;
  }
  DirectSweep& S = g_direct[{part, kind}];
  const int korder = kind == 0 ? bit_tree3d_kernel_order : 0;
  const PARTICLE& t = part[ind];
  const bool fresh = S.valid && S.n == npart && S.param == param && S.korder == korder &&
                     !S.served[ind] && S.x[ind] == t.x && S.y[ind] == t.y && S.z[ind] == t.z &&
                     S.q[ind] == t.tot_charge;
  if (fresh) return &S;
  bit_ctx* c = ctx();
  if (!c) { complain("no CUDA device"); return nullptr; }
  S.valid = false;
  S.n = npart; S.param = param; S.korder = korder;
  S.x.resize(npart); S.y.resize(npart); S.z.resize(npart); S.q.resize(npart);
  for (int i = 0; i < npart; i++) {
    S.x[i] = part[i].x; S.y[i] = part[i].y; S.z[i] = part[i].z; S.q[i] = part[i].tot_charge;
  }
  std::vector<int> tg(npart);
  for (int i = 0; i < npart; i++) tg[i] = i;
  S.a.assign(npart, 0.0);
  bit_status st;
  if (kind == 2) {
    bit_eval_params P{};
    P.kernel = BIT_KERNEL_SCREENED;
    P.mode = BIT_MODE_REFERENCE;
    P.precision = BIT_PREC_FP64;
    P.kappa = param;
    st = bit_direct_potential(c, npart, S.x.data(), S.y.data(), S.z.data(), S.q.data(), &P, npart,
                              tg.data(), S.a.data());
  } else {
    S.b.assign(npart, 0.0);
    S.c.assign(npart, 0.0);
    st = bit_direct_field(c, npart, S.x.data(), S.y.data(), S.z.data(), S.q.data(), kind == 0,
                          param, korder, npart, tg.data(), S.a.data(), S.b.data(), S.c.data());
  }
  if (!ok(st, "direct sum")) return nullptr;
  S.served.assign(npart, 0);
  S.valid = true;
  return &S;
}

}  // namespace

void force_particle_ds_reg(int ind, int npart, PARTICLE* part, double* xfor, double* yfor,
                           double* zfor) {
  std::lock_guard<std::mutex> lk(mu);
  DirectSweep* S = direct_sweep(0, ind, npart, part, bit_tree3d_del);
  if (!S) return;
  S->served[ind] = 1;
  *xfor = S->a[ind]; *yfor = S->b[ind]; *zfor = S->c[ind];
}

void force_particle_ds_noreg(int ind, int npart, PARTICLE* part, double* xfor, double* yfor,
                             double* zfor) {
  std::lock_guard<std::mutex> lk(mu);
  DirectSweep* S = direct_sweep(1, ind, npart, part, 0.0);
  if (!S) return;
  S->served[ind] = 1;
  *xfor = S->a[ind]; *yfor = S->b[ind]; *zfor = S->c[ind];
}

void shielded_pot_particle_ds(int ind, int npart, PARTICLE* part, double* pot, double alpha) {
  std::lock_guard<std::mutex> lk(mu);
  DirectSweep* S = direct_sweep(2, ind, npart, part, alpha);
  if (!S) return;
  S->served[ind] = 1;
  *pot = S->a[ind];
}

// ---- the reference tests' fixture --------------------------------------------------------
// RandL and boxparticles (src/tree3d.cpp:13-15, 1698-1740): the same rand() draws in the same
// order, so the particles equal the reference's on the same C library.
double RandL(void) { return std::rand() / (double)RAND_MAX; }

void boxparticles(int npart, double dlength, double dheight, double ddepth, PARTICLE* part,
                  double density) {
  const double weight = density * dlength * dheight * ddepth / npart;
  std::srand(100);
  const double hx = dlength / 2, hy = dheight / 2, hz = ddepth / 2;
  for (int i = 0; i < npart; i++) {
    PARTICLE& p = part[i];
    p.charge = -1.0;
    p.weight = weight;
    p.x = hx / 2 + RandL() * hx;
    p.y = hy / 2 + RandL() * hy;
    p.z = hz / 2 + RandL() * hz;
    p.u = (RandL() - 0.5) * 1e6;
    p.v = (RandL() - 0.5) * 1e6;
    p.w = (RandL() - 0.5) * 1e6;
    p.tot_charge = p.charge * p.weight * elec;
  }
}

// freespace_particles_tree (src/tree3d.cpp:2268-2335)
void freespace_particles_tree(int npart, PARTICLE* part, int nterms, double acc, TREE* tree,
                              int numtree, int maxmemb) {
  numtree = treemake(npart, nterms, maxmemb, part, tree);
  if (numtree < 0) return;
  treemoments(numtree, nterms, tree, part);
  for (int i = 0; i < npart; i++) {
    double xf = 0, yf = 0, zf = 0;
    if (treeforce(0, i, nterms, part[i].x, part[i].y, part[i].z, acc, &xf, &yf, &zf, tree, part))
      return;
    part[i].xforce = xf * charge_constant * part[i].tot_charge;
    part[i].yforce = yf * charge_constant * part[i].tot_charge;
    part[i].zforce = zf * charge_constant * part[i].tot_charge;
  }
  treeempty(numtree, tree);
}

// vel_update / loc_update (src/tree3d.cpp:4842-4888): host loops over the caller's
// particle array, as in the reference (bit_pic_steps is the device-resident loop).
int vel_update(int npart, PARTICLE* part, double dt) {
  for (int i = 0; i < npart; i++) {
    part[i].u += dt * part[i].xforce * invmass;
    part[i].v += dt * part[i].yforce * invmass;
    part[i].w += dt * part[i].zforce * invmass;
  }
  return 0;
}

// output_potential (src/tree3d.cpp:4918-4937) through bit_write_potential, which writes
// the reference's bytes; a file that cannot be written is reported by
// bit_tree3d_last_error() (the reference's ofstream fails silently).
void output_potential(int npart, PARTICLE* part, double* pot, std::string filename) {
  std::vector<double> x(npart), y(npart), z(npart);
  for (int i = 0; i < npart; i++) {
    x[i] = part[i].x;
    y[i] = part[i].y;
    z[i] = part[i].z;
  }
  const bit_status st = bit_write_potential(filename.c_str(), npart, x.data(), y.data(),
                                            z.data(), pot);
  if (st != BIT_OK) complain("output_potential: cannot write " + filename);
}

int loc_update(int npart, PARTICLE* part, double dt) {
  for (int i = 0; i < npart; i++) {
    part[i].x += dt * part[i].u;
    part[i].y += dt * part[i].v;
    part[i].z += dt * part[i].w;
  }
  return 0;
}

// solver::gmres (src/solver.h:157-260) on the device
int solver::gmres(double** a, double* b, double* x, int num) {
  std::lock_guard<std::mutex> lk(mu);
  bit_ctx* c = ctx();
  if (!c) return -1;
  std::vector<double> A((size_t)num * num);
  for (int i = 0; i < num; i++) std::memcpy(&A[(size_t)i * num], a[i], num * sizeof(double));
  bit_status s = bit_gmres_dense(c, num, A.data(), b, x, &iters_);
  if (s == BIT_ERR_BREAKDOWN) std::fprintf(stderr, "ERROR: Breakdown!  Quitting...\n");
  else ok(s, "solver::gmres");
  return 0;
}
