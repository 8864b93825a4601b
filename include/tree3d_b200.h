/*
 * tree3d_b200.h -- drop-in replacement for the treecode surface of the reference's
 * src/tree3d.h (ongbw/bit), implemented on the GPU by libtree3d_b200.so over the C ABI of
 * bit_b200.h.  A program written against the reference's tree3d.h / constants.h /
 * problem.h / solver.h switches by including this header instead and linking
 * -ltree3d_b200 -lbit_b200.
 *
 * Types and signatures are the reference's (src/tree3d.h:33-74, 115-126, 197-298,
 * src/solver.h:31-315); the physical constants are the values of src/constants.h:12-22 so
 * that results scale identically.  DEL / ACC / KERNEL_ORDER are the reference's
 * compile-time problem constants (src/problem.h:11-13); here DEL is read at run time from
 * bit_tree3d_del (default 0.01, the reference's value).
 *
 * Semantics that differ (documented, never silent):
 *  - treepotential / shielded_treepot / treeforce called with ind == 0 and a particle
 *    index p evaluate ALL particles of the tree on the GPU on the first call for a given
 *    (tree, acc, kernel) and serve later calls from that result; p == -1 evaluates the one
 *    point on the GPU.  ind != 0 (an internal recursion step of the reference) returns -1
 *    without touching *pot.
 *  - treemake reports failure by returning -1 (the reference never returns on >maxmemb
 *    coincident particles) and a message from bit_tree3d_last_error().
 *  - KERNEL_ORDER > 0 and the screened 2-D field are FP64 only: with
 *    bit_tree3d_precision = 1 those calls report an error.
 *
 * A program written against the reference compiles unchanged with include/tree3d_compat
 * first on its include path: its tree3d.h and constants.h there include this header,
 * and the program's own problem.h sets DEL and KERNEL_ORDER at start-up.
 */
#ifndef TREE3D_B200_H
#define TREE3D_B200_H

#include <cstdio>
#include <string>

const int MAXPART = 1000000;  /* src/constants.h:8  */
const int NUMCHILD = 8;       /* src/constants.h:9  */
const int MAXTERM = 12;       /* src/constants.h:10 */
const int MAXCHILD = 100000;  /* src/constants.h:11 */
const double pi = 3.14159265359;
const double inv2pi = 0.5 / pi;
const double perm = 8.85418781762e-12;
const double elec = 1.60217733e-19;
const double charge_constant = inv2pi / perm;
const double invmass = 1.0 / 9.1093897e-31; /* src/constants.h:19 */
const double eps = 1e-14;

/* src/tree3d.h:33-47 */
struct PARTICLE {
  double charge;
  double x, y, z;
  double u, v, w;
  double xforce, yforce, zforce;
  double weight;
  double tot_charge;
};

/* src/tree3d.h:51-74 */
struct TREE {
  int nummemb;
  double x0, x1, y0, y1, z0, z1;
  double xmid, ymid, zmid;
  double aspectxy, aspectxz, aspectyz;
  double sqradius;
  int children[NUMCHILD];
  int* members;
  double*** moments;
  TREE() : nummemb(0), members(0x0), moments(0x0) {}
};

/* run-time problem constants (the reference's src/problem.h:11-13) */
extern double bit_tree3d_del;
extern double bit_tree3d_mac_del;   /* screened MAC offset; the reference uses DEL */
extern int bit_tree3d_kernel_order; /* KERNEL_ORDER (0 = the one-parameter kernel)   */
extern int bit_tree3d_precision;    /* 0 = FP64 (default), 1 = mixed FP32 */
const char* bit_tree3d_last_error();

/* src/tree3d.cpp:13-15 and 1698-1740: the reference tests' fixture, npart particles
 * uniform in the middle half of a dlength x dheight x ddepth box from srand(100) / rand()
 * (the same draws in the same order, so the same particles on the same C library),
 * charge -1, weight density * volume / npart, tot_charge = charge * weight * elec. */
double RandL(void);
void boxparticles(int npart, double dlength, double dheight, double ddepth, PARTICLE* part,
                  double density);

int treemake(int num, int nterms, int maxmemb, PARTICLE* part, TREE* tree);
void treeempty(int numtree, TREE* tree);
void treemoments(int numtree, int nterms, TREE* tree, PARTICLE* part);
double treepotential(int ind, int p, int nterms, double x, double y, double z, double acc,
                     double* pot, TREE* tree, PARTICLE* part);
double shielded_treepot(int ind, int p, int nterms, double x, double y, double z,
                        double alpha, double acc, double* pot, TREE* tree, PARTICLE* part,
                        int Nx, int Ny, int Nz, double dlength, double dheight,
                        double ddepth);
double treeforce(int ind, int p, int nterms, double x, double y, double z, double acc,
                 double* xfor, double* yfor, double* zfor, TREE* tree, PARTICLE* part);
void freespace_particles_tree(int npart, PARTICLE* part, int nterms, double acc, TREE* tree,
                              int numtree, int maxmemb);
/* src/tree3d.cpp:3268-3408 and 2368-2436: the screened 2-D field (FP64) and its driver;
 * served like treeforce. */
double shielded_treeforce(int ind, int p, int nterms, double x, double y, double z,
                          double alpha, double acc, double* xfor, double* yfor, double* zfor,
                          TREE* tree, PARTICLE* part);
void shielded_freespace_particles_tree(int npart, PARTICLE* part, double alpha, int nterms,
                                       double acc, TREE* tree, int numtree, int maxmemb);

/* Direct sums (src/tree3d.cpp:298-330, 182-213, 1966-2016), assigning the field or
 * potential of particle ind from all others.  On the GPU: the first call evaluates every
 * particle of part[] and later calls are served from that result until a target is asked
 * for a second time or its own position or charge differs from the snapshot; then the
 * sums are evaluated afresh from the current part[].  A caller that changes the particles
 * between two complete sweeps over the targets therefore sees the new values. */
void force_particle_ds_reg(int ind, int npart, PARTICLE* part, double* xfor, double* yfor,
                           double* zfor);
void force_particle_ds_noreg(int ind, int npart, PARTICLE* part, double* xfor, double* yfor,
                             double* zfor);
void shielded_pot_particle_ds(int ind, int npart, PARTICLE* part, double* pot, double alpha);
/* src/tree3d.cpp:4842-4850 and :4880-4888: explicit velocity and position updates */
int vel_update(int npart, PARTICLE* part, double dt);
int loc_update(int npart, PARTICLE* part, double dt);
/* src/tree3d.cpp:4918-4937: "i\tx\ty\tz\tpot" per particle, 14 significant digits */
void output_potential(int npart, PARTICLE* part, double* pot, std::string filename);

/* src/solver.h:31-315: dense GMRES, on the device */
class solver {
 public:
  solver() {}
  void makeFram(int) {}
  int gmres(double** a, double* b, double* x, int num);
  int minimize(int) { return 0; }
  int iterations() const { return iters_; }

 private:
  int iters_ = 0;
};

#endif
