"""Generate the golden fixtures in this directory from the UNMODIFIED reference treecode.

    make -C oracle ref && python tests/golden/make_golden.py

Runs the reference's own treemake / treemoments / treepotential / shielded_treepot /
treeforce / setboundaries / panelconstantsreal / output_potential (ongbw/bit src/tree3d.cpp, built by
oracle/Makefile from the reference sources)
on seeded inputs and stores inputs and outputs as .npz.  The Coulomb potential runs with
moment arrays padded to (nterms+1)^3 (oracle/ref_wrap.cpp) so its degree-nterms reads stay
in bounds.  Only the reference's outputs are stored; nothing of the reference source is.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from bit_b200 import workloads  # noqa: E402


def tree_record(R):
    nm, ch, f, mem = R.export()
    T = R.nterms * (R.nterms + 1) * (R.nterms + 2) // 6
    mom = np.zeros((R.numtree, T))
    order = [(i, j, k) for i in range(R.nterms) for j in range(R.nterms - i)
             for k in range(R.nterms - i - j)]
    for node in range(R.numtree):
        m = R.node_moments(node)
        mom[node] = [m[a, b, c] for (a, b, c) in order]
    return dict(nummemb=nm, children=ch, fields=f, members=mem, moments=mom)


def case(name, x, y, z, q, w, nterms, maxmemb, del_, acc, kappa):
    R = ref.RefTree(x, y, z, q, nterms, maxmemb, del_=del_, w=w)
    R.moments()
    rec = tree_record(R)
    rng = np.random.default_rng(7)
    pts = rng.uniform(-1.3, 1.3, (64, 3))
    out = dict(x=x, y=y, z=z, q=q, w=w if w is not None else np.ones(len(x)),
               nterms=nterms, maxmemb=maxmemb, del_=del_, acc=acc, kappa=kappa, points=pts,
               coulomb=R.potential(acc), screened=R.screened(kappa, acc),
               coulomb_points=R.potential(acc, points=pts),
               screened_points=R.screened(kappa, acc, points=pts))
    fx, fy, fz = R.force(acc)
    out.update(force=np.stack([fx, fy, fz]))
    out.update(rec)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    R.close()
    print(name, "numtree", rec["nummemb"].shape[0])


def panel_case(name, xp, yp, zp, dl, dh, dd, del_):
    """setboundaries + panelconstantsreal of the reference build with DEL = del_."""
    panels = ref.setboundaries(xp, yp, zp, dl, dh, dd, del_=del_)
    A = ref.panelconstantsreal(xp, yp, zp, dl, dh, dd, del_=del_)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), xp=xp, yp=yp, zp=zp, dl=dl, dh=dh,
                        dd=dd, del_=del_, panels=panels, A=A)
    print(name, panels.shape, A.shape)


def output_case(name, n, seed):
    """output_potential of the reference on seeded values (incl. signed zeros, tiny, huge)."""
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    pot = rng.standard_normal(n) * 10.0 ** rng.integers(-20, 20, n)
    pot[:4] = [0.0, -0.0, 1.0, -1234567.891011121314]
    ref.output_potential(x, y, z, pot, os.path.join(HERE, name + ".txt"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), x=x, y=y, z=z, pot=pot)
    print(name, n)


def main():
    # the reference tests' own fixture (tests/treecode.cpp:41), smaller N
    x, y, z, q, w = ref.boxparticles(2000)
    # 20 z-panels over depth 12 put one ring of panels in 4 < z < 5 (refpot 0)
    panel_case("panels_box", 3, 2, 20, 2.0, 3.0, 12.0, 1e-4)
    output_case("output_potential", 300, 41)
    case("box2000", x, y, z, q, w, nterms=5, maxmemb=100, del_=0.01, acc=0.5, kappa=1.0)
    # uniform cube, regularised Coulomb delta = 0.01 (DEL = 1e-4)
    x, y, z, q = workloads.uniform_cube(3000, seed=3)
    case("uniform3000", x, y, z, q, None, nterms=7, maxmemb=100, del_=1e-4, acc=0.5, kappa=1.0)
    # clustered blobs, delta = 0.005 (DEL = 2.5e-5), p = 8, theta = 0.7
    x, y, z, q = workloads.clustered_blobs(4000, seed=4)
    case("clustered4000", x, y, z, q, None, nterms=9, maxmemb=100, del_=2.5e-5, acc=0.7,
         kappa=1.0)
    # a thin slab: y/z-only split branches and the z-split of a sibling slot
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, 2500); y = rng.uniform(-0.3, 0.3, 2500); z = rng.uniform(-0.05, 0.05, 2500)
    q = rng.uniform(-1, 1, 2500)
    case("slab2500", x, y, z, q, None, nterms=4, maxmemb=60, del_=0.01, acc=0.6, kappa=2.0)


if __name__ == "__main__":
    main()
