/*
 * bit_b200.h -- C ABI of the B200-native BIT treecode.
 *
 * Plain C types only (pointers, sizes, enums, POD structs); no CUDA or C++ types cross
 * this boundary.  Every entry point returns a bit_status; none aborts or throws.  A
 * context owns one CUDA stream on one device and is not thread-safe: use one context per
 * host thread.  Trees are owned by the context that built them and keep their device
 * memory (particles, nodes, moments, interaction lists) resident until destroyed.
 *
 * Each entry point names the reference (ongbw/bit) interface it replaces, as file:line.
 */
#ifndef BIT_B200_H
#define BIT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BIT_ABI_VERSION 1
#define BIT_NTERMS_MAX 10 /* nterms = p + 1; the reference caps it via MAXTERM=12 (src/constants.h:10) */

typedef struct bit_ctx bit_ctx;
typedef struct bit_tree bit_tree;

typedef enum {
  BIT_OK = 0,
  BIT_ERR_INVALID_ARGUMENT = 1,
  BIT_ERR_CUDA = 2,
  BIT_ERR_OUT_OF_MEMORY = 3,
  BIT_ERR_CAPACITY = 4,     /* a node / list / stack capacity was exceeded              */
  BIT_ERR_DEGENERATE = 5,   /* > maxmemb coincident particles: the reference loops forever */
  BIT_ERR_BREAKDOWN = 6,    /* GMRES breakdown (src/solver.h:220-225)                    */
  BIT_ERR_NOT_CONVERGED = 7,
  BIT_ERR_NO_DEVICE = 8,
  BIT_ERR_BUDGET = 9,       /* the request does not fit the context's HBM budget         */
  BIT_ERR_STATE = 10        /* call order violated (e.g. evaluation before moments)      */
} bit_status;

typedef enum {
  BIT_KERNEL_COULOMB = 0,      /* 1/sqrt(r^2 + del)          treepotential, src/tree3d.cpp:4679 */
  BIT_KERNEL_SCREENED = 1,     /* -exp(-kappa r)/r           shielded_treepot, src/tree3d.cpp:3448 */
  BIT_KERNEL_SCREENED_REG = 2  /* exp(-kappa R)/R, R^2 = r^2 + del (new; no reference routine) */
} bit_kernel;

typedef enum {
  BIT_PREC_FP64 = 0,  /* plain FP64 everywhere                                         */
  BIT_PREC_MIXED = 1  /* FP32 near/far arithmetic in cluster-centred coordinates with
                         compensated per-target accumulation; FP64 MAC and moments   */
} bit_precision;

typedef enum {
  /* Exactly the reference's conventions: Coulomb particle targets drop del in the near
   * field (src/tree3d.cpp:4765); screened particle targets add q*intg/w for themselves
   * (:3575-3596); screened point targets add the near field with + (:3558). */
  BIT_MODE_REFERENCE = 0,
  /* One kernel everywhere: near field uses the same kernel as the far field and the
   * direct sum (src/tree3d.cpp:298-330, 1966-2016); self excluded. */
  BIT_MODE_CONSISTENT = 1
} bit_mode;

typedef struct {
  int device;        /* CUDA device ordinal                                  */
  void* stream;      /* cudaStream_t to use; NULL: the context creates one   */
  size_t hbm_budget; /* bytes the context may allocate; 0 = no limit         */
} bit_ctx_opts;

typedef struct {
  bit_kernel kernel;
  bit_mode mode;
  bit_precision precision;
  double del;      /* delta^2 of the regularised kernels (the reference's DEL, src/problem.h:12) */
  double mac_del;  /* screened kernel only: accept iff sqradius < acc*(r^2 - mac_del)
                      (the reference subtracts DEL, src/tree3d.cpp:3473)                  */
  double kappa;    /* screening parameter (the reference's alpha / kappa)                 */
  double acc;      /* MAC: accept iff sqradius < acc * distance^2 (src/tree3d.cpp:866)    */
  double intg;     /* reference-mode screened self term constant (src/tree3d.cpp:3585)    */
} bit_eval_params;

/* Device time (seconds, CUDA events on the context stream) of the last call's phases and
 * the interaction counts of its lists. */
typedef struct {
  double t_build, t_moments, t_lists, t_far, t_near, t_total;
  long long far_pairs;   /* (target, cluster) Taylor evaluations   */
  long long near_pairs;  /* (target, source) direct interactions   */
  long long far_entries, near_entries, batches;
  int numtree, nleaves, depth, nterms;
  int far_launches, near_launches;
  int list_fallback; /* the last list build used the count / scan / fill passes */
  int lists_shared;  /* the last evaluation reused lists built for another MAC (the
                        context's previous one): every acceptance decision of that
                        traversal was also checked under this MAC and agreed, so the
                        lists are the ones this MAC's own traversal would build */
} bit_stats;

const char* bit_status_string(bit_status s);
int bit_abi_version(void);
/* Number of CUDA kernels this library has launched in this process (all contexts). */
long long bit_kernel_launches(void);

bit_status bit_ctx_create(bit_ctx** ctx, const bit_ctx_opts* opts);
bit_status bit_ctx_destroy(bit_ctx* ctx);
const char* bit_ctx_last_error(const bit_ctx* ctx);
bit_status bit_ctx_synchronize(bit_ctx* ctx);
/* Leaf packing, a tuning knob (bit_b200.autotune): 0 (default) evaluates each leaf as its
 * own group of targets; 32..1024 evaluates runs of consecutive small leaves together, up
 * to that many targets (one traversal, shared source tiles).  Results do not depend on it
 * beyond FP32 summation order. */
bit_status bit_ctx_set_group_size(bit_ctx* ctx, int targets);
/* Evaluations whose systems fall into several (nterms, kernel) classes (forests): 1
 * (default) runs the far field and the near field each as ONE persistent kernel whose CTAs
 * take (system, target group) items from a device work queue in decreasing-work order;
 * 0 launches once per class.  Results are identical either way. */
bit_status bit_ctx_set_work_queue(bit_ctx* ctx, int on);
/* Near-field tuning knobs (bit_b200.autotune): `tile` source records per TMA tile (a power
 * of two, 128..2048; clamped to 256..2048 for the mixed path and 128..1024 for FP64; 0: the
 * default, 1024 mixed / 512 FP64) and the cap on threads that share one target's sources
 * (a power of two, 1..32; 0: the default rule).  Results change only in FP rounding order. */
bit_status bit_ctx_set_near_config(bit_ctx* ctx, int tile, int threads_per_target);
bit_status bit_ctx_stream(const bit_ctx* ctx, void** stream);
/* Bytes currently allocated by the context and its trees. */
bit_status bit_ctx_memory(const bit_ctx* ctx, size_t* in_use, size_t* peak);
/* Give back to the device the freed blocks the context keeps for reuse, largest first,
 * until the bytes it holds (live + cached) are at most `keep`; live buffers are never
 * freed.  Waits for the context's stream.  For a long-lived process that moves from one
 * workload to another (e.g. a large batch, then serving) so that the next one finds the
 * memory free.  No reference counterpart. */
bit_status bit_ctx_trim(bit_ctx* ctx, size_t keep);

/* treemake (src/tree3d.cpp:1345-1551): build the aspect-ratio bisection tree of the n
 * particles.  x, y, z are host arrays (original order).  The node numbering, children
 * order and member sets equal the reference's.  Returns BIT_ERR_DEGENERATE where the
 * reference would never terminate. */
bit_status bit_tree_build(bit_ctx* ctx, int n, const double* x, const double* y,
                          const double* z, int maxmemb, bit_tree** tree);
/* Same with device pointers (resident inputs). */
bit_status bit_tree_build_device(bit_ctx* ctx, int n, const double* x, const double* y,
                                 const double* z, int maxmemb, bit_tree** tree);
/* treeempty (src/tree3d.cpp:990-1004). */
bit_status bit_tree_destroy(bit_tree* tree);
bit_status bit_tree_info(const bit_tree* tree, int* numtree, int* nleaves, int* depth);

/* Charges (the reference's tot_charge) and weights (the reference's weight, used only by
 * the reference-mode screened self term; NULL = 1) in original particle order. */
bit_status bit_tree_set_charges(bit_tree* tree, const double* q, const double* w);
bit_status bit_tree_set_charges_device(bit_tree* tree, const double* q, const double* w);
/* treemoments (src/tree3d.cpp:2631-2711), FP64, for nterms = p + 1 (1..BIT_NTERMS_MAX). */
bit_status bit_tree_moments(bit_tree* tree, int nterms);

/* Copy the tree out in the reference's TREE terms (src/tree3d.h:51-74): per node
 * nummemb, children[8] (-1 = none), 13 doubles (x0 x1 y0 y1 z0 z1 xmid ymid zmid aspectxy
 * aspectxz aspectyz sqradius); members concatenated in node order, each node's list in
 * ascending index (the reference's order).  Any output pointer may be NULL. */
bit_status bit_tree_export(const bit_tree* tree, int* nummemb, int* children,
                           double* fields, int* members);
/* Moments, T = nterms(nterms+1)(nterms+2)/6 per node, packed with i (x power)
 * outermost, then j, then k. */
bit_status bit_tree_export_moments(const bit_tree* tree, double* mom);

/* treepotential (src/tree3d.cpp:4679) / shielded_treepot (:3448) at every particle
 * (targets = sources, p = particle index).  pot: host array, original order. */
bit_status bit_eval_particles(bit_tree* tree, const bit_eval_params* prm, double* pot);
bit_status bit_eval_particles_device(bit_tree* tree, const bit_eval_params* prm,
                                     double* pot);
/* Same at m external points (the reference's p = -1 path).  Host arrays. */
bit_status bit_eval_points(bit_tree* tree, const bit_eval_params* prm, int m,
                           const double* x, const double* y, const double* z, double* pot);
/* treeforce (src/tree3d.cpp:851-971) at every particle: the field sum q grad G with the
 * regularised Coulomb kernel (del), KERNEL_ORDER = 0.  Host arrays, original order. */
bit_status bit_eval_force(bit_tree* tree, double del, double acc, bit_precision prec,
                          double* fx, double* fy, double* fz);

/* Fields at every particle, generalising bit_eval_force.  Host arrays, original order. */
#define BIT_KERNEL_ORDER_MAX 8
typedef enum {
  /* treeforce (src/tree3d.cpp:851-971) with treetaylorforce (:456-810) and
   * eval_grad_kernel_reg (:73-97): the field of 1/sqrt(r^2 + del), regularised by the
   * reference's KERNEL_ORDER family (src/problem.h:13) of order kernel_order. */
  BIT_FIELD_COULOMB = 0,
  /* shielded_treeforce (src/tree3d.cpp:3268-3408) with shielded_treetaylorforce
   * (:2745-2973): the reference's screened 2-D field, fx = -d/dy, fy = d/dx of
   * q e^{-kappa r}/r summed over the sources, fz = 0; r^2 without del, the screened MAC
   * sqradius < acc (r^2 - mac_del) (:3279-3283); no eps check at particle targets. */
  BIT_FIELD_SCREENED = 1
} bit_field_kind;
typedef struct {
  bit_field_kind kind;
  bit_precision precision; /* MIXED only for BIT_FIELD_COULOMB with kernel_order 0 */
  double del;              /* COULOMB: DEL of r^2 + del                                */
  double mac_del;          /* SCREENED: the MAC offset (the reference subtracts DEL)   */
  double kappa;            /* SCREENED: the screening parameter (alpha)               */
  double acc;              /* MAC parameter                                            */
  int kernel_order;        /* COULOMB: 0..BIT_KERNEL_ORDER_MAX                        */
} bit_field_params;
bit_status bit_eval_field(bit_tree* tree, const bit_field_params* prm, double* fx, double* fy,
                          double* fz);

/* Time stepping of the reference's particle loop, device-resident: every step rebuilds
 * the tree from the current positions and runs freespace_particles_tree
 * (src/tree3d.cpp:2268-2335: treemake, treemoments, treeforce, F = field * charge_constant
 * * q), then vel_update (:4842-4850, u += dt F invmass) and loc_update (:4880-4888,
 * x += dt u).  x..w are device arrays in original order, updated in place; fx, fy, fz
 * (device, may all be NULL) receive F of the last step. */
typedef struct {
  int steps, nterms, maxmemb;
  double dt, del, acc;
  double charge_constant, invmass; /* src/constants.h:22 / :30 and :19 / :29 */
  bit_precision precision;
} bit_pic_opts;
bit_status bit_pic_steps(bit_ctx* ctx, int n, double* x, double* y, double* z, double* u,
                         double* v, double* w, const double* q, const bit_pic_opts* opts,
                         double* fx, double* fy, double* fz);

/* Whole pipeline through host buffers, the analogue of treemake + treemoments + a loop of
 * treepotential / shielded_treepot over all particles (tests/treecode_mp.cpp:57-95). */
bit_status bit_treecode_potential(bit_ctx* ctx, int n, const double* x, const double* y,
                                  const double* z, const double* q, const double* w,
                                  int nterms, int maxmemb, const bit_eval_params* prm,
                                  double* pot);

/* FP64 direct sum at m particle targets (indices into the n sources; each target skips
 * itself by index): shielded_pot_particle_ds (src/tree3d.cpp:1966-2016), -sum q e^{-kappa r}/r,
 * for BIT_KERNEL_SCREENED; sum q / sqrt(r^2 + del) for BIT_KERNEL_COULOMB; and
 * sum q e^{-kappa R}/R with R = sqrt(r^2 + del) for BIT_KERNEL_SCREENED_REG, the two
 * regularised sums skipping r^2 + del <= 1e-14 (src/constants.h:35).  The accuracy
 * reference of every treecode result.  pot[i] belongs to targets[i].  Host arrays; the
 * _device variant takes device pointers (an out-of-range device target index is reported
 * by the next synchronising call). */
bit_status bit_direct_potential(bit_ctx* ctx, int n, const double* x, const double* y,
                                const double* z, const double* q, const bit_eval_params* prm,
                                int m, const int* targets, double* pot);
bit_status bit_direct_potential_device(bit_ctx* ctx, int n, const double* x, const double* y,
                                       const double* z, const double* q,
                                       const bit_eval_params* prm, int m, const int* targets,
                                       double* pot);

/* FP64 field direct sum at m particle targets (indices into the n sources; each target
 * skips itself by index), fx/fy/fz[i] for targets[i]: with regularised != 0,
 * force_particle_ds_reg (src/tree3d.cpp:298-330): sum q_j G(x_j - x), G(d) = -d t,
 * t = 1/(r rs) plus the KERNEL_ORDER terms of eval_grad_kernel_reg (:73-97), rs = |d|^2 + del;
 * with regularised == 0, force_particle_ds_noreg (:182-213): t = 1/(rs sqrt(rs)),
 * rs = |d|^2 (coincident particles give inf / NaN, as in the reference).  Host arrays. */
bit_status bit_direct_field(bit_ctx* ctx, int n, const double* x, const double* y,
                            const double* z, const double* q, int regularised, double del,
                            int kernel_order, int m, const int* targets, double* fx, double* fy,
                            double* fz);

/* Measured CUDA-core FMA throughput of the context's device in flop/s (2 per FMA): FP32
 * (BIT_PREC_MIXED) or FP64 (BIT_PREC_FP64), from a dense FMA-chain kernel timed with CUDA
 * events (best of 3 launches of about 0.1 s).  The denominator of the near- and
 * far-field rooflines; no reference counterpart. */
bit_status bit_device_fma_peak(bit_ctx* ctx, bit_precision prec, double* flops_per_s);

/* Largest difference, in ulps of CUDA's result, between the FP64 near field's own exp and
 * rsqrt and CUDA's exp and rsqrt over n seeded arguments (exp: [-707, 0], and (-8, 0] for
 * its small-argument form, the larger of the two; rsqrt: [1e-12, 1e6], log-uniform).  A
 * diagnostic of the device math; no reference counterpart. */
bit_status bit_device_fp64_math_error(bit_ctx* ctx, long long n, double* exp_ulps,
                                      double* rsqrt_ulps);

/* The kernels' give-up path for a device-side wait, exercised on its own: one CTA waits,
 * with the same bounded mbarrier wait the near and far fields use (at most `limit`
 * attempts), on a barrier that nothing ever completes, combines the outcome for the CTA
 * and raises the context's device error flag.  Returns BIT_ERR_CUDA ("a device-side wait
 * gave up", flag 16) with the flag then cleared, so the context stays usable for later
 * calls.  No copy is in flight, nothing faults and nothing hangs.  A diagnostic of the
 * failure path; no reference counterpart. */
bit_status bit_device_wait_check(bit_ctx* ctx, int limit);

bit_status bit_tree_stats(const bit_tree* tree, bit_stats* st);

/* Per-target interaction lists of the last evaluation, in the reference's traversal
 * order, for particle index p: kind 0 = far (Taylor) cluster, 1 = near (direct) leaf.
 * Returns the count in *n (entries beyond cap are dropped). */
bit_status bit_tree_target_lists(bit_tree* tree, const bit_eval_params* prm, int p,
                                 int* node, int* kind, int cap, int* n);

/* ---------------------------------------------------------------------------------
 * Forests: many independent systems in one tree, built, expanded and evaluated by the
 * same launches (no reference counterpart: the reference handles one system per
 * treemake / treepotential loop, src/tree3d.cpp:1345, 4679; this replaces a host loop of
 * those calls over many systems).
 * System s owns particles [o_s, o_s + n[s]) of x, y, z, q (o_s = n[0] + ... + n[s-1]).
 * Its subtree is the tree treemake builds for those particles alone with maxmemb[s] (same
 * nodes, children order and members), rooted at node s; its moments, MAC and kernel are
 * its own, so every system's result equals a separate single-system evaluation.
 * ------------------------------------------------------------------------------- */
bit_status bit_forest_build(bit_ctx* ctx, int nsys, const int* n, const int* maxmemb,
                            const double* x, const double* y, const double* z,
                            bit_tree** tree);
bit_status bit_forest_build_device(bit_ctx* ctx, int nsys, const int* n, const int* maxmemb,
                                   const double* x, const double* y, const double* z,
                                   bit_tree** tree);
/* Moments of every system: nterms[s] (1..BIT_NTERMS_MAX) per system. */
bit_status bit_forest_moments(bit_tree* tree, const int* nterms);
/* Potential at every particle with params[s] for system s (one precision for all).
 * pot: host array (bit_forest_eval) or device array (bit_forest_eval_device), original
 * order. */
bit_status bit_forest_eval(bit_tree* tree, const bit_eval_params* params, double* pot);
bit_status bit_forest_eval_device(bit_tree* tree, const bit_eval_params* params, double* pot);
/* Number of systems; first node of system s is its root, node s. */
bit_status bit_forest_systems(const bit_tree* tree, int* nsys);

/* ---------------------------------------------------------------------------------
 * GMRES with the treecode as its matvec (no reference counterpart: the reference's
 * solver::gmres, src/solver.h:157-260, takes a dense matrix).
 * Solves (diag*I + K) s = f, (K s)_i = sum_{j != i} G(x_i, x_j) w_j s_j, G from prm.
 * ------------------------------------------------------------------------------- */
typedef struct {
  int restart;             /* GMRES(m)                                                */
  int maxit;               /* cap on inner iterations (matvecs)                       */
  double tol;              /* target relative residual ||f - A s|| / ||f|| (FP64 A)   */
  bit_precision precision; /* FP64: FP64 matvecs.  MIXED: FP32 matvecs inside FP64
                              iterative refinement with FP64 true residuals            */
  double inner_tol;        /* MIXED: relative tolerance of each inner solve (0: 1e-4) */
  int max_refinements;     /* MIXED: outer refinement steps cap (0: 10)               */
} bit_gmres_opts;

typedef struct {
  int iterations;  /* inner GMRES iterations (all refinement steps) */
  int refinements; /* outer refinement steps (MIXED)                */
  int matvecs_fp64, matvecs_fp32;
  double relres;   /* final true relative residual in FP64          */
  double seconds;  /* device time of the solve                      */
} bit_gmres_info;

/* ---------------------------------------------------------------------------------
 * Boundary panels (PANEL, src/tree3d.h:77-95) and the panel solve.
 * ------------------------------------------------------------------------------- */
typedef struct {
  double x0, x1, y0, y1, z0, z1;
  double str;                /* panel strength sigma (set by bit_panel_solve) */
  double xnrm, ynrm, znrm;
  double refpot;             /* Dirichlet value                                */
  double midx, midy, midz;   /* quadrature point                               */
  int type;                  /* 0: Dirichlet                                   */
  int orientation;           /* 1: xy, 2: xz, 3: yz                            */
  double area;
} bit_panel;

/* setboundaries (src/tree3d.cpp:3764-3934): the faces of a dlength x dheight x ddepth box
 * centred at the origin, in the reference's panel order.  *numpan gets
 * 2 (xp yp + zp yp + xp zp); pan (that many entries) may be NULL to ask for the count. */
bit_status bit_panels_box(int xpanels, int ypanels, int zpanels, double dlength,
                          double dheight, double ddepth, bit_panel* pan, int* numpan);
/* panelconstantsreal (src/tree3d.cpp:4054-4078) on the device, bit-exact:
 * A[i*n + j] = -1 / sqrt(|mid_i - mid_j|^2 + del) / 2 * inv2pi * area_j. */
bit_status bit_panel_matrix(bit_ctx* ctx, int n, const bit_panel* pan, double del, double* A);
/* The panel solve the reference left commented out (panel_solve_tree,
 * src/tree3d.cpp:4351-4438) on the treecode: b_i = refpot_i + 0.5 sum_j q_j / r_ij over the
 * np particles (FP64 direct sum), then A sigma = b for A as in bit_panel_matrix, solved as
 * (I/sqrt(del) + K) (area sigma) = -4 pi b with the regularised Coulomb treecode K over
 * the panel midpoints (nterms, acc, maxmemb) and GMRES(m) (opts).  Sets pan[i].str. */
bit_status bit_panel_solve(bit_ctx* ctx, int npan, bit_panel* pan, int np, const double* x,
                           const double* y, const double* z, const double* q, double del,
                           int nterms, double acc, int maxmemb, const bit_gmres_opts* opts,
                           bit_gmres_info* info);

/* output_potential (src/tree3d.cpp:4918-4937): one line per particle,
 * "i\tx\ty\tz\tpot", 14 significant digits.  Host arrays. */
bit_status bit_write_potential(const char* path, int n, const double* x, const double* y,
                               const double* z, const double* pot);
/* The same from device arrays, streamed to the file in chunks (device-to-host copies of the
 * next chunk overlap the formatting of the current one). */
bit_status bit_write_potential_device(bit_ctx* ctx, const char* path, int n, const double* x,
                                      const double* y, const double* z, const double* pot);

/* ---------------------------------------------------------------------------------
 * Serving (no reference counterpart: the reference has no request layer).
 * A server owns `slots` contexts on one device, each with its own stream, and a FIFO of
 * evaluate and solve requests.  A request starts when a slot is free and its estimated
 * device memory fits in what running requests leave of the HBM budget (the head of the
 * queue is never overtaken); requests in different slots overlap on the device.  Inputs
 * are copied at submission; results are identical to the single-request calls
 * (bit_treecode_potential, bit_bie_solve) whatever else runs.  The functions are safe to
 * call from several host threads.
 * ------------------------------------------------------------------------------- */
typedef struct bit_server bit_server;

typedef struct {
  int device;
  int slots;          /* requests on the device at once (1..64)                  */
  size_t hbm_budget;  /* bytes the running requests may hold (0: 90% of free)     */
} bit_server_opts;

typedef struct {
  bit_status status;
  int slot;
  double t_submit, t_start, t_done;  /* seconds on the server's clock          */
  size_t bytes_reserved;             /* admission estimate                      */
  size_t peak_bytes;                 /* device memory the request's slot peaked at */
  bit_gmres_info gmres;              /* solve requests                          */
} bit_request_info;

typedef struct {
  long long submitted, completed, queued;
  int running, max_running, slots;
  size_t budget, reserved, max_reserved;
  double now;  /* seconds since the server was created */
} bit_server_info;

bit_status bit_server_create(bit_server** server, const bit_server_opts* opts);
/* Finishes every submitted request, then releases the device. */
bit_status bit_server_destroy(bit_server* server);
/* Potential at every particle (treemake + treemoments + treepotential /
 * shielded_treepot for all p); returns the request id.  BIT_ERR_BUDGET if the request
 * alone exceeds the budget. */
bit_status bit_server_submit_eval(bit_server* server, int n, const double* x, const double* y,
                                  const double* z, const double* q, int nterms, int maxmemb,
                                  const bit_eval_params* prm, long long* id);
/* (diag*I + K) s = f with weights w, as bit_bie_solve. */
bit_status bit_server_submit_solve(bit_server* server, int n, const double* x, const double* y,
                                   const double* z, const double* w, const double* f,
                                   int nterms, int maxmemb, const bit_eval_params* prm,
                                   double diag, const bit_gmres_opts* opts, long long* id);
/* Block until the request is done; out gets its n results (original order).  Returns the
 * request's status.  Each id can be waited for once. */
bit_status bit_server_wait(bit_server* server, long long id, double* out,
                           bit_request_info* info);
bit_status bit_server_poll(bit_server* server, long long id, int* done);
bit_status bit_server_stats(bit_server* server, bit_server_info* info);
const char* bit_server_last_error(const bit_server* server);

bit_status bit_bie_solve(bit_tree* tree, const bit_eval_params* prm, int nterms, double diag,
                         const double* w, const double* f, double* s,
                         const bit_gmres_opts* opts, bit_gmres_info* info);

/* solver::gmres (src/solver.h:157-310) on a dense row-major n x n matrix, on the device:
 * full GMRES from zero, modified Gram-Schmidt, least squares by Gram-Schmidt QR of the
 * Hessenberg, stop when the max relative change of x < 1e-5 every odd step.  x holds the
 * initial values used by that stopping test.  Returns BIT_ERR_BREAKDOWN on h < 1e-14. */
bit_status bit_gmres_dense(bit_ctx* ctx, int n, const double* a, const double* b, double* x,
                           int* iterations);

/* bit_gmres_dense without any allocation at call time, for callers that cannot allocate:
 * code running where cudaMalloc is forbidden or unsafe (inside a caller's own memory pool
 * or allocator hook, a real-time loop with a fixed memory plan, or a host that has
 * reserved all device memory up front).  No reference counterpart; it gives the same
 * results as bit_gmres_dense with the same kernels.
 * Scratch is one file-scope device array (about 4.2 MB, held by every GPU that loads this
 * library until the process exits) sized for n <= BIT_GMRES_STATIC_MAX, plus file-scope
 * host arrays; no cudaMalloc / cudaFree and no allocating library call is made.
 * n > BIT_GMRES_STATIC_MAX returns BIT_ERR_CAPACITY with a message.  Runs in the CUDA
 * context current on the calling thread, on `stream` (a cudaStream_t; NULL = the default
 * stream), with host arrays a (row-major n x n), b, x (initial values in, solution out);
 * b = 0 returns x = 0.  A message for any error goes to err (errlen bytes, NUL-terminated;
 * may be NULL).
 * Every call looks up the scratch's address in the current context (cudaGetSymbolAddress).
 * The first call in a context may load this library's device code (CUDA lazy loading),
 * which creates the array: make one warm-up call per device outside any region that must
 * not allocate, and before any stream capture.
 * Calls that overlap in time share the scratch and race: serialise them. */
#define BIT_GMRES_STATIC_MAX 512
bit_status bit_gmres_dense_static(void* stream, int n, const double* a, const double* b,
                                  double* x, int* iterations, char* err, int errlen);

#ifdef __cplusplus
}
#endif
#endif /* BIT_B200_H */
