"""The reference's G5 mesh from hole_forest (test/hole_runs.jl:2416-2435): Harmonic(1, 7/10) on
[-5/4, 5/4]^3, N = 8, one root, radii 10, 8/5, 13/10, 1 give the 2472 blocks of 8^3, 1,265,664
points and finest h = 5/256 the reference states for its G5 chart (SINGULARITY_HANDLING.md:1066,
1272)."""
import numpy as np


def test_g5_mesh_is_the_references(tgh):
    case = tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=1.25, r0=0.8, r1=1.0, variant="fitted")
    f = tgh.hole_forest(case, 8, 1, [10.0, 1.6, 1.3, 1.0])
    assert f.nblocks == 2472 and f.points() == 1265664
    assert f.h0 / 2 ** int(f.level.max()) == 5.0 / 256.0
    assert list(np.bincount(f.level)) == [0, 0, 0, 232, 2240]
