/* TEST INFRASTRUCTURE (oracle) -- CPU restatement of the BIT treecode hot path.
 *
 * Used only by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline / reference
 * arm) as the checker.  The shipped library never links or calls this code.
 *
 * Every function restates the reference (ongbw/bit) algorithm it names, in plain C with
 * FP64 arithmetic and no FMA contraction, so that trees and interaction lists are
 * identical to the reference's and values agree to the last bit where the reference
 * itself is well defined.
 */
#ifndef BIT_ORACLE_H
#define BIT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Kernels and modes (same numbering as the library's C ABI). */
enum { ORC_COULOMB = 0, ORC_SCREENED = 1, ORC_SCREENED_REG = 2 };
enum { ORC_MODE_REFERENCE = 0, ORC_MODE_CONSISTENT = 1 };

/* Error codes of orc_tree_build. */
enum { ORC_ERR_CAPACITY = -1, ORC_ERR_DEGENERATE = -2, ORC_ERR_INVALID = -3 };

/* Flat tree: node i owns perm[start[i] .. start[i]+nummemb[i]); a node's children
 * occupy consecutive sub-ranges of it in slot order, and every node's members appear
 * in ascending original index (the reference's member order).  fields holds 13
 * doubles per node: x0 x1 y0 y1 z0 z1 xmid ymid zmid aspxy aspxz aspyz sqradius. */
typedef struct {
  int n, numtree, nterms;
  const double *x, *y, *z, *q, *w;
  const int *nummemb, *start, *children, *perm;
  const double *fields;
  const double *mom; /* T(nterms) doubles per node, packed (i, j, k) with i outermost */
} orc_tree_view;

typedef struct {
  int kernel, mode;
  double del;     /* Coulomb / regularised-screened delta^2 (reference DEL)            */
  double mac_del; /* screened MAC offset: accept iff sqradius < acc*(r^2 - mac_del)    */
  double kappa;
  double acc;
  double intg;    /* screened self term q*intg/w in reference mode                     */
} orc_params;

int orc_nterms_max(void);
int orc_num_terms(int nterms);                /* T(nterms) = nterms(nterms+1)(nterms+2)/6 */
int orc_moment_index(int nterms, int i, int j, int k);
double orc_aspect_limit(void);

int orc_tree_build(int n, const double* x, const double* y, const double* z, int maxmemb,
                   int cap, int* nummemb, int* start, int* children, int* level,
                   int* parent, double* fields, int* perm);
void orc_moments(const orc_tree_view* t, double* mom);

/* Targets: p[t] >= 0 is a particle (coordinates from it), -1 an external point. */
void orc_eval(const orc_tree_view* t, const orc_params* prm, int nt, const int* p,
              const double* tx, const double* ty, const double* tz, double* pot,
              int nthreads);
void orc_eval_force(const orc_tree_view* t, double del, double acc, int kernel_order,
                    int nt, const int* p, const double* tx, const double* ty,
                    const double* tz, double* fx, double* fy, double* fz, int nthreads);
void orc_count(const orc_tree_view* t, const orc_params* prm, int nt, const int* p,
               const double* tx, const double* ty, const double* tz, long long* nfar,
               long long* nnear_pairs, long long* nnear_leaves, int nthreads);
int orc_target_lists(const orc_tree_view* t, const orc_params* prm, int p, double x,
                     double y, double z, int* node, int* kind, int cap);

void orc_direct(int n, const double* x, const double* y, const double* z, const double* q,
                const orc_params* prm, int nt, const int* p, const double* tx,
                const double* ty, const double* tz, double* pot, int nthreads);
void orc_direct_force(int n, const double* x, const double* y, const double* z,
                      const double* q, double del, int kernel_order, int nt, const int* p,
                      double* fx, double* fy, double* fz, int nthreads);

int orc_gmres_dense_ref(int n, const double* A, const double* b, double* x);
int orc_gmres_treecode(orc_tree_view* t, double* mom_work, const orc_params* prm,
                       double diag, const double* wts, const double* b, double* x,
                       int restart, double tol, int maxit, int nthreads, int* iters,
                       double* relres);

#ifdef __cplusplus
}
#endif
#endif
