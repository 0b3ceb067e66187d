"""Which copy of a point shared across a coarse-fine face is the primary one (the value every copy
takes after a fill, and the one a sum counts). TreeAMR, whose fill the reference uses, is not
vendored and its documents leave the choice open (CODE.md:434-444); this library takes the
coarsest leaf holding the point, the choice with which the reference's driver record on a
refined hole is met (tests/test_gpu_driver_golden.py). Checked on the oracle's fill of a
two-level mesh whose blocks hold different markers: a point of the interface that lies on the
coarse lattice takes the coarse block's value in the fine block; a point only the fine block
holds keeps the fine value; a face between two fine blocks takes the value of the block holding
it on its lower face."""
import numpy as np

from helpers import two_level_forest


def test_the_coarsest_leaf_is_the_primary_copy(oracle, tgh):
    case = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=0.0)
    N, q = 8, 4
    f = two_level_forest(tgh, case, N=N)
    O = oracle.problem(case, f, q)
    N1, G = N + 1, q // 2 + 1
    W = N1 + 2 * G
    u = np.zeros(O.L)
    S = N1 ** 3
    for b in range(f.nblocks):
        u[b * 20 * S:(b + 1) * 20 * S] = b + 1.0
    O.prepare(u, 0.0)
    w = O.work().reshape(f.nblocks, 20, W, W, W)  # (block, variable, z, y, x)

    def block(level, corner):
        for b in range(f.nblocks):
            if int(f.level[b]) == level and tuple(int(c) for c in f.corner[b]) == corner:
                return b
        raise AssertionError((level, corner))

    fine = block(1, (N, 0, 0))      # upper x face at level-1 coordinate 2N = level-0 N
    coarse = block(0, (N, 0, 0))    # holds that face on its lower x face
    fine_lo = block(1, (0, 0, 0))   # holds the face x = N (level 1) on its upper face
    # on the coarse lattice (even fine indices): the coarse block's value
    assert w[fine, 0, G + 2, G + 4, G + N] == coarse + 1.0
    assert w[coarse, 0, G + 1, G + 2, G + 0] == coarse + 1.0
    # held by the fine block alone (odd fine index): its own value
    assert w[fine, 0, G + 2, G + 3, G + N] == fine + 1.0
    # between two fine blocks: the one holding it on its lower face
    assert w[fine_lo, 0, G + 2, G + 3, G + N] == fine + 1.0
