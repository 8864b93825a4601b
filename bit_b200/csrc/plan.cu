// Evaluation plans: per-system parameters of one call, the MAC its lists need, and the
// launch classes of the far / near kernels.
//
// A tree may hold several independent systems (a forest), each with its own kernel,
// parameters and expansion order.  Kernels read a group's parameters from the system's
// SysEval entry; the template parameters of a launch (nterms, kernel, precision) are the
// same for every group of one launch class, so a forest is evaluated by one far launch
// per distinct (nterms, kernel) and one near launch per distinct (kernel, eps check).
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace bit {

SysEval make_sys_eval(const bit_eval_params& p, int nterms, int points, int force,
                      int kernel_order) {
  SysEval s{};
  s.kernel = force == 1 ? BIT_KERNEL_COULOMB : (force == 2 ? BIT_KERNEL_SCREENED : p.kernel);
  s.nterms = nterms;
  s.acc = p.acc;
  s.kappa = p.kappa;
  s.intg = p.intg;
  s.particles = !points;
  const bool ref = p.mode == BIT_MODE_REFERENCE;
  // MAC, src/tree3d.cpp:4688-4692 (Coulomb: + del - del), 3472-3476 (screened: - mac_del)
  if ((!force && p.kernel == BIT_KERNEL_SCREENED) || force == 2) {
    s.mac_add = 0.0;
    s.mac_sub = p.mac_del;
  } else {
    s.mac_add = p.del;
    s.mac_sub = p.del;
  }
  if (force == 2) {
    // shielded_treeforce (src/tree3d.cpp:3268-3408): r^2 without del in both fields, the
    // screened MAC with its del offset (:3279-3283), no eps check for particles (:3378-3398)
    s.far_add = 0.0;
    s.far_sign = 1.0;
    s.near_del = 0.0;
    s.near_sign = 1;
    s.eps_check = 0;
    s.particles = 1;
    return s;
  }
  if (force) {
    s.kernel_order = kernel_order;
    // treeforce (src/tree3d.cpp:851-971): r^2 + del in both fields
    s.far_add = p.del;
    s.far_sign = 1.0;
    s.near_del = p.del;
    s.near_sign = 1;
    s.eps_check = 0;
    s.particles = 1;
    return s;
  }
  switch (p.kernel) {
    case BIT_KERNEL_COULOMB:
      s.far_add = p.del;
      s.far_sign = 1.0;
      // src/tree3d.cpp:4744-4772: points use del, particles drop it (reference mode)
      s.near_del = (points || !ref) ? p.del : 0.0;
      s.eps_check = 1;
      s.near_sign = 1;
      break;
    case BIT_KERNEL_SCREENED:
      s.far_add = 0.0;
      s.far_sign = -1.0;                            // src/tree3d.cpp:3222 subtracts
      s.near_del = 0.0;
      s.eps_check = points ? 1 : 0;                 // :3557 / :3604-3619
      s.near_sign = (points && ref) ? 1 : -1;       // :3558 adds, :3619 subtracts
      s.self_term = (!points && ref) ? 1 : 0;       // :3575-3596
      break;
    default:  // regularised screened: one kernel with del everywhere
      s.far_add = p.del;
      s.far_sign = 1.0;
      s.near_del = p.del;
      s.eps_check = 1;
      s.near_sign = 1;
      break;
  }
  return s;
}

void plan_sys(Tree* t, EvalPlan* P, const std::vector<bit_eval_params>& prm, int points,
              int force, int kernel_order) {
  const int ns = t->nsys;
  if (prm.empty() || ((int)prm.size() != 1 && (int)prm.size() != ns))
    fail(BIT_ERR_INVALID_ARGUMENT, "one parameter set, or one per system, expected");
  if (points && ns != 1) fail(BIT_ERR_INVALID_ARGUMENT, "external points need a single-system tree");
  if (!t->has_moments) fail(BIT_ERR_STATE, "moments not computed (call bit_tree_moments)");
  for (const auto& p : prm)
    if (p.precision != prm[0].precision)
      fail(BIT_ERR_INVALID_ARGUMENT, "all systems of one call share a precision");
  std::vector<SysEval> h(ns);
  for (int s = 0; s < ns; s++)
    h[s] = make_sys_eval(prm[prm.size() == 1 ? 0 : s], t->h_sys_nterms[s], points, force,
                         kernel_order);
  P->f32 = prm[0].precision == BIT_PREC_MIXED;
  P->force = force;
  const bool same = P->sys.p && P->h_sys.size() == h.size() &&
                    std::equal(h.begin(), h.end(), P->h_sys.begin(), [](const SysEval& a, const SysEval& b) {
                      return std::memcmp(&a, &b, sizeof(SysEval)) == 0;
                    });
  if (same) return;
  P->h_sys = h;
  P->sys.ensure(t->ctx, ns);
  BIT_CUDA(cudaMemcpyAsync(P->sys.p, P->h_sys.data(), ns * sizeof(SysEval), cudaMemcpyHostToDevice,
                           t->ctx->stream));
  P->lists_version = -1;
}

ListKey plan_key(const Tree* t, const EvalPlan& P, int points) {
  ListKey k;
  k.points = points;
  k.group = t->ctx->group_targets;
  k.gen = t->gen;
  const SysEval& s0 = P.h_sys[0];
  k.acc = s0.acc;
  k.add_del = s0.mac_add;
  k.sub_del = s0.mac_sub;
  if (P.h_sys.size() > 1)
    for (const auto& s : P.h_sys) {
      k.sysmac.push_back(s.acc);
      k.sysmac.push_back(s.mac_add);
      k.sysmac.push_back(s.mac_sub);
    }
  return k;
}

namespace {
long long far_class_of(const SysEval& s) { return s.nterms * 2 + (s.kernel == BIT_KERNEL_COULOMB ? 0 : 1); }
long long near_class_of(const SysEval& s) { return (s.kernel == BIT_KERNEL_COULOMB ? 0 : 2) + s.eps_check; }

// Groups ordered by class, then by decreasing work; one LaunchClass per class present.
void order_by_class(const Lists* L, const std::vector<long long>& gcls, const EvalPlan& P,
                    std::vector<int>& ord, std::vector<LaunchClass>& cls, bool far) {
  const int ng = L->ngroups;
  ord.resize(ng);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    if (gcls[a] != gcls[b]) return gcls[a] < gcls[b];
    return L->h_work[a] > L->h_work[b];
  });
  cls.clear();
  for (int i = 0; i < ng; i++) {
    if (i == 0 || gcls[ord[i]] != gcls[ord[i - 1]]) {
      const SysEval& s = P.h_sys[L->h_g_sys[ord[i]]];
      cls.push_back(LaunchClass{far ? s.nterms : 0, s.kernel, s.eps_check, i, 0});
    }
    cls.back().count++;
  }
}
}  // namespace

void plan_classes(Tree* t, Lists* L, EvalPlan* P) {
  const int ns = (int)P->h_sys.size();
  std::vector<long long> key(2 * ns);
  for (int s = 0; s < ns; s++) {
    key[2 * s] = far_class_of(P->h_sys[s]);
    key[2 * s + 1] = near_class_of(P->h_sys[s]);
  }
  if (P->lists_version == L->version && P->class_key == key) return;
  bool one_far = true, one_near = true;
  for (int s = 1; s < ns; s++) {
    one_far &= key[2 * s] == key[0];
    one_near &= key[2 * s + 1] == key[1];
  }
  const int ng = L->ngroups;
  Ctx* c = t->ctx;
  cudaStream_t st = c->stream;
  std::vector<long long> gf(ng), gn(ng);
  for (int g = 0; g < ng; g++) {
    gf[g] = key[2 * L->h_g_sys[g]];
    gn[g] = key[2 * L->h_g_sys[g] + 1];
  }
  std::vector<int> ord;
  const SysEval& s0 = P->h_sys[0];
  if (one_far) {
    P->far_classes.assign(1, LaunchClass{s0.nterms, s0.kernel, s0.eps_check, 0, ng});
    P->far_ord = L->order.p;
  } else {
    order_by_class(L, gf, *P, ord, P->far_classes, true);
    P->far_order.ensure(c, ng);
    BIT_CUDA(cudaMemcpyAsync(P->far_order.p, ord.data(), ng * sizeof(int), cudaMemcpyHostToDevice, st));
    P->far_ord = P->far_order.p;
  }
  if (one_near) {
    P->near_classes.assign(1, LaunchClass{0, s0.kernel, s0.eps_check, 0, ng});
    P->near_ord = L->order.p;
  } else {
    order_by_class(L, gn, *P, ord, P->near_classes, false);
    P->near_order.ensure(c, ng);
    BIT_CUDA(cudaMemcpyAsync(P->near_order.p, ord.data(), ng * sizeof(int), cudaMemcpyHostToDevice, st));
    P->near_ord = P->near_order.p;
  }
  if (!one_far || !one_near) BIT_CUDA(cudaStreamSynchronize(st));
  P->lists_version = L->version;
  P->class_key = key;
}

// Particle-target lists for this call's MAC: the tree's own lists when they were built
// for it, or built for another MAC and checked against this one; else a new build, which
// also checks the context's previous MAC (an evaluation that alternates two kernels on
// each new tree then walks the tree once per tree when their decisions agree).
void prepare_particles(Tree* t, const std::vector<bit_eval_params>& prm, int force,
                       int kernel_order) {
  plan_sys(t, &t->pplan, prm, 0, force, kernel_order);
  const ListKey k = plan_key(t, t->pplan, 0);
  Lists& L = t->plists;
  Ctx* c = t->ctx;
  const bool own = L.valid && L.key == k;
  const bool shared = !own && L.valid && L.alt_valid && L.alt_key == k;
  t->lists_built = !own && !shared;
  if (t->lists_built) {
    const ListKey alt = c->mac_hint;
    const bool check = alt.acc >= 0 && !alt.same_mac(k);
    if (t->ev[4]) BIT_CUDA(cudaEventRecord(t->ev[4], c->stream));
    build_lists(t, &L, k, t->n, t->sx.p, t->sy.p, t->sz.p, t->pplan.sys.p, check ? &alt : nullptr);
    if (t->ev[5]) BIT_CUDA(cudaEventRecord(t->ev[5], c->stream));
  }
  L.shared = shared;
  c->mac_hint = k;
  plan_classes(t, &L, &t->pplan);
}

}  // namespace bit
