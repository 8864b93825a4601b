// A program written against the reference's treecode interface (it follows the shape of
// the reference's tests/treecode.cpp and tests/treecode_mp.cpp), compiled against
// include/tree3d_b200.h and linked with libtree3d_b200.so instead of libtree3d.
//   1. treemake + treemoments + treeforce for every particle; the max error against an
//      FP64 direct sum is non-increasing in nterms = 1..4 (tests/treecode.cpp:84-127);
//   2. every TREE field is filled and member lists partition the particles;
//   3. solver::gmres solves a small dense system.
// Prints PASSED / FAILED and returns 0 / 1 like the reference's tests.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tree3d_b200.h"

static double urand(unsigned long long* s) {
  *s = *s * 6364136223846793005ULL + 1442695040888963407ULL;
  return ((*s >> 11) & ((1ULL << 53) - 1)) / 9007199254740992.0;
}

int main() {
  const int npart = 6000, maxmemb = 100;
  std::vector<PARTICLE> part(npart);
  unsigned long long seed = 100;
  for (int i = 0; i < npart; i++) {
    part[i].x = 0.25 + 0.5 * urand(&seed);
    part[i].y = 0.25 + 0.5 * urand(&seed);
    part[i].z = 0.25 + 0.5 * urand(&seed);
    part[i].weight = 1.0 / npart;
    part[i].charge = -1.0;
    part[i].tot_charge = part[i].charge * part[i].weight * elec;
  }
  bit_tree3d_del = 0.01;
  // direct sum with the regularised kernel (force_particle_ds_reg)
  std::vector<double> fx(npart), fy(npart), fz(npart);
  for (int i = 0; i < npart; i++) {
    double a = 0, b = 0, c = 0;
    for (int j = 0; j < npart; j++) {
      if (j == i) continue;
      double dx = part[j].x - part[i].x, dy = part[j].y - part[i].y, dz = part[j].z - part[i].z;
      double rs = dx * dx + dy * dy + dz * dz + bit_tree3d_del;
      double t = 1.0 / (std::sqrt(rs) * rs);
      a += part[j].tot_charge * -dx * t;
      b += part[j].tot_charge * -dy * t;
      c += part[j].tot_charge * -dz * t;
    }
    fx[i] = a; fy[i] = b; fz[i] = c;
  }
  int fail = 0;
  double errstore = 0;
  const int maxtrees = 3 * npart / maxmemb + 1000;
  for (int nterms = 1; nterms < 5; nterms++) {
    TREE* tree = new TREE[maxtrees];
    int numtree = treemake(npart, nterms, maxmemb, part.data(), tree);
    if (numtree <= 0) { std::printf("treemake failed: %s\n", bit_tree3d_last_error()); return 1; }
    long long covered = 0;
    for (int i = 0; i < numtree; i++)
      if (tree[i].children[0] == -1) covered += tree[i].nummemb;
    if (covered != npart) { std::printf("leaves do not partition the particles\n"); fail = 1; }
    treemoments(numtree, nterms, tree, part.data());
    double ex = 0, ey = 0, ez = 0;
    for (int i = 0; i < npart; i++) {
      double a = 0, b = 0, c = 0;
      if (treeforce(0, i, nterms, part[i].x, part[i].y, part[i].z, 0.5, &a, &b, &c, tree,
                    part.data()) != 0) {
        std::printf("treeforce failed: %s\n", bit_tree3d_last_error());
        return 1;
      }
      ex = std::fmax(ex, std::fabs(a - fx[i]));
      ey = std::fmax(ey, std::fabs(b - fy[i]));
      ez = std::fmax(ez, std::fabs(c - fz[i]));
    }
    double errnew = ex + ey + ez;
    std::printf("nterms = %d, err = %.6e\n", nterms, errnew);
    if (nterms > 1 && errnew > errstore) fail = 1;
    errstore = errnew;
    treeempty(numtree, tree);
    delete[] tree;
  }
  // solver::gmres on a diagonally dominant dense system
  const int n = 64;
  std::vector<std::vector<double>> A(n, std::vector<double>(n));
  std::vector<double*> rows(n);
  std::vector<double> bvec(n), x(n, 1.0);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) A[i][j] = (i == j ? 4.0 : 0.0) + 0.1 * (urand(&seed) - 0.5);
    rows[i] = A[i].data();
    bvec[i] = urand(&seed) - 0.5;
  }
  solver s;
  s.makeFram(n + 1);
  s.gmres(rows.data(), bvec.data(), x.data(), n);
  double res = 0, bn = 0;
  for (int i = 0; i < n; i++) {
    double r = bvec[i];
    for (int j = 0; j < n; j++) r -= A[i][j] * x[j];
    res += r * r;
    bn += bvec[i] * bvec[i];
  }
  std::printf("gmres iterations = %d, relres = %.3e\n", s.iterations(), std::sqrt(res / bn));
  if (!(std::sqrt(res / bn) < 1e-4)) fail = 1;
  std::printf(fail ? "Test FAILED\n" : "Test PASSED\n");
  return fail;
}
