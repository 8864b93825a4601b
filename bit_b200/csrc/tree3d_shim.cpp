// libtree3d_b200.so: the reference's tree3d.h / solver.h entry points (include/
// tree3d_b200.h) over the C ABI of bit_b200.h.  Host C++ only; every computation runs in
// libbit_b200.so on the GPU.
#include "tree3d_b200.h"

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "bit_b200.h"

double bit_tree3d_del = 0.01;
double bit_tree3d_mac_del = 0.01;
int bit_tree3d_precision = 0;

namespace {

struct Cached {
  double acc = -1, kappa = -1;
  int kind = -1;  // 0 coulomb, 1 screened, 2 force
  std::vector<double> a, b, c;
};

struct Entry {
  bit_tree* tree = nullptr;
  int n = 0, nterms = 0;
  int mom_dim = 0;  // edge of the moment arrays this library allocated (0: none)
  std::vector<double> x, y, z;
  Cached pot[2], force;
};

std::mutex mu;
bit_ctx* g_ctx = nullptr;
std::map<const TREE*, Entry> g_trees;
thread_local std::string g_err;

bit_ctx* ctx() {
  if (!g_ctx) {
    bit_ctx_opts o{0, nullptr, 0};
    if (bit_ctx_create(&g_ctx, &o) != BIT_OK) g_ctx = nullptr;
  }
  return g_ctx;
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
  if (!c) { g_err = "no CUDA device"; return -1; }
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
  if (it == g_trees.end()) { g_err = "treemoments: tree not built by treemake"; return; }
  Entry& e = it->second;
  std::vector<double> q(e.n), w(e.n);
  for (int i = 0; i < e.n; i++) { q[i] = part[i].tot_charge; w[i] = part[i].weight; }
  if (!ok(bit_tree_set_charges(e.tree, q.data(), w.data()), "treemoments")) return;
  if (!ok(bit_tree_moments(e.tree, nterms), "treemoments")) return;
  e.nterms = nterms;
  e.pot[0] = Cached(); e.pot[1] = Cached(); e.force = Cached();
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
    g_err = "only ind == 0 (the whole tree) is served on the GPU";
    return -1;
  }
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { g_err = "tree not built by treemake"; return -1; }
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
  if (C.acc != acc || C.kappa != kappa || C.kind != kernel) {
    C.a.assign(e.n, 0.0);
    if (!ok(bit_eval_particles(e.tree, &P, C.a.data()), "evaluate particles")) return -1;
    C.acc = acc; C.kappa = kappa; C.kind = kernel;
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
  if (ind != 0) { g_err = "only ind == 0 is served on the GPU"; return -1; }
  auto it = g_trees.find(tree);
  if (it == g_trees.end()) { g_err = "tree not built by treemake"; return -1; }
  Entry& e = it->second;
  if (!(p >= 0 && p < e.n && x == e.x[p] && y == e.y[p] && z == e.z[p])) {
    g_err = "treeforce at a point that is not the particle p is not supported";
    return -1;
  }
  Cached& C = e.force;
  if (C.acc != acc) {
    C.a.assign(e.n, 0.0); C.b.assign(e.n, 0.0); C.c.assign(e.n, 0.0);
    if (!ok(bit_eval_force(e.tree, bit_tree3d_del, acc, (bit_precision)bit_tree3d_precision,
                           C.a.data(), C.b.data(), C.c.data()), "treeforce"))
      return -1;
    C.acc = acc;
  }
  *xfor += C.a[p]; *yfor += C.b[p]; *zfor += C.c[p];
  return 0;
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
  if (st != BIT_OK) g_err = "output_potential: cannot write " + filename;
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
