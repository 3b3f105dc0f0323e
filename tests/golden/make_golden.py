"""Regenerate the golden plan fixtures (run in a container with the reference).

For each seeded scene it runs the REFERENCE's own maximin ordering
(src/maxmin.h create_ordering_3d) and kd-tree pattern (src/nanoflann.hpp),
compiled into oracle/_ref/libref.so by oracle/Makefile, checks that the CPU
oracle reproduces them bit for bit, and stores inputs and outputs:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from fastmbcui_b200 import scenes as S  # noqa: E402

SCENES = {
    "sphere_ico4": lambda: S.sphere_scene(),
    "ellipsoids3_mixed": lambda: S.ellipsoids_scene(3, [400, 700, 900], seed=11),
    "coin1x1500": lambda: S.coins_scene(n_coins=1, pts=1500),
}


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libref.so missing (needs the reference tree)"
    for name, make in SCENES.items():
        sc = make()
        P, s = O.ref_order(sc.y)
        ptr, ind = O.ref_pattern(sc.y, P, s, sc.rho)
        pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
        assert np.array_equal(P, pl["P"]) and np.array_equal(s, pl["scale"]), name
        assert np.array_equal(ptr, pl["ptr"]) and np.array_equal(ind, pl["ind"]), name
        np.savez_compressed(os.path.join(HERE, f"plan_{name}.npz"),
                            y=sc.y.astype(np.float32), rho=np.float32(sc.rho), lam=sc.lam,
                            max_super=sc.max_super, P=P, scale=s, ptr=ptr, ind=ind,
                            sup_ptr=pl["sup_ptr"], sup_ind=pl["sup_ind"], sup_parent=pl["sup_parent"],
                            lptr=pl["lptr"], lind=pl["lind"])
        print(name, sc.n, "nnz", ptr[-1], "supernodes", pl["n_super"])


if __name__ == "__main__":
    main()
