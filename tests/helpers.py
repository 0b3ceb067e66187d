"""Shared helpers for the parity tests: the reference's comparison metric and the cases."""
import numpy as np


def rhs_scale(work, forest, q):
    """Per owned point, max(1, max_{v,d} |D2_d u_v| / h^2, max_v |u_v|) from a working array
    (test/evolution_tests.jl:97-108); returns [nblocks, N1, N1, N1] (z, y, x order)."""
    N, G = forest.N, q // 2 + 1
    W, N1 = N + 2 * G + 1, N + 1
    r = q // 2
    from fractions import Fraction  # noqa: F401
    w2 = {2: [1, -2, 1], 4: [-1 / 12, 4 / 3, -5 / 2, 4 / 3, -1 / 12],
          6: [1 / 90, -3 / 20, 3 / 2, -49 / 18, 3 / 2, -3 / 20, 1 / 90],
          8: [-1 / 560, 8 / 315, -1 / 5, 8 / 5, -205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560]}[q]
    w = work.reshape(forest.nblocks, 20, W, W, W)
    out = np.ones((forest.nblocks, N1, N1, N1))
    for b in range(forest.nblocks):
        h = forest.h0 / 2 ** int(forest.level[b])
        own = w[b, :, G:G + N1, G:G + N1, G:G + N1]
        s = np.max(np.abs(own), axis=0)
        for axis in range(3):
            acc = 0.0
            for k, wk in enumerate(w2):
                off = k - r
                sl = [slice(None), slice(G, G + N1), slice(G, G + N1), slice(G, G + N1)]
                ax = 3 - axis  # arrays are (v, z, y, x)
                sl[ax] = slice(G + off, G + off + N1)
                acc = acc + wk * w[b][tuple(sl)]
            s = np.maximum(s, np.max(np.abs(acc), axis=0) / h ** 2)
        out[b] = np.maximum(s, 1.0)
    return out


def rhs_error(du_gpu, du_ref, scale, forest):
    """max over points of max_v |du_gpu - du_ref| / rhs_scale."""
    N1 = forest.N + 1
    a = du_gpu.reshape(forest.nblocks, 20, N1, N1, N1)
    b = du_ref.reshape(forest.nblocks, 20, N1, N1, N1)
    return float(np.max(np.max(np.abs(a - b), axis=1) / scale))


N_ROWS = 22


def cases(tgh):
    """(name, case, forest, q, t) rows the GPU parity tests run on."""
    rows = []
    c = tgh.perturbed_minkowski_case()
    rows.append(("perturbed_minkowski_q4", c, tgh.gh_forest(c, 8, 2), 4, 0.0))
    for q in (2, 4, 6, 8):
        c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
        rows.append((f"gauge_wave_q{q}", c, tgh.gh_forest(c, 10 if q < 8 else 10, 2), q, 0.25))
    c = tgh.gauge_wave_case(eps_ko=0.0, gamma0=0.0, gamma2=0.0)
    rows.append(("gauge_wave_q4_nodiss_nodamp", c, tgh.gh_forest(c, 8, 2), 4, 0.25))
    c = tgh.shifted_minkowski_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    rows.append(("shifted_minkowski_sampled", c, tgh.gh_forest(c, 8, 2), 4, 0.125))
    for variant in ("damped", "frozen", "pasted"):
        c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, variant=variant, gauge="sampled")
        rows.append((f"kerr_schild_{variant}", c, tgh.gh_forest(c, 8, 2), 4, 0.0))
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    rows.append(("kerr_schild_algebraic", c, tgh.gh_forest(c, 8, 2), 4, 0.0))
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    rows.append(("kerr_schild_moving", c, tgh.gh_forest(c, 8, 2), 4, 0.3))
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic",
                             eps_ko={"eps_out": 0.5, "eps_in": 2.0, "r_1": 1.3, "r_h": 1.7, "c0": (0, 0, 0)})
    rows.append(("kerr_schild_horizon_dissipation", c, tgh.gh_forest(c, 8, 2), 4, 0.0))
    # blocks of N = 32, the size the kernels are also compiled for with fixed strides
    for q in (2, 4, 6, 8):
        c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
        rows.append((f"gauge_wave_q{q}_n32", c, tgh.gh_forest(c, 32, 2), q, 0.25))
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    rows.append(("kerr_schild_damped_n32", c, tgh.gh_forest(c, 32, 2), 4, 0.0))
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    rows.append(("kerr_schild_algebraic_n32", c, tgh.gh_forest(c, 32, 2), 4, 0.0))
    # a moving boosted hole on a four-level hierarchy of 8^3 blocks (levels 1-3 populated,
    # prolongation at two interfaces): the hierarchy workload's physics at a size the
    # oracle steps in seconds
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.hole_forest(c, 8, 2, [3.0, 1.8, 1.4], path=((0.0, 0.0, 0.0), (0.05, 0.0, 0.0)))
    rows.append(("kerr_schild_hierarchy_moving", c, f, 4, 0.3))
    # Kerr in harmonic coordinates (no gauge source), at rest and moving
    c = tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.9, r1=1.4)
    rows.append(("harmonic_kerr_damped", c, tgh.gh_forest(c, 8, 2), 4, 0.0))
    c = tgh.harmonic_kerr_case(M=1.0, a=0.7, v=0.1, halfwidth=2.0, r0=0.9, r1=1.4)
    rows.append(("harmonic_kerr_moving", c, tgh.gh_forest(c, 8, 2), 4, 0.3))
    assert len(rows) == N_ROWS
    return rows


def two_level_forest(tgh, case, N=8):
    """A 2^3 root grid with one root block refined (the interface test's mesh,
    test/interface_tests.jl:64-113)."""
    import numpy as np  # noqa: F811
    f = tgh.gh_forest(case, N, 2)
    leaves = [(0, tuple(int(v) for v in c)) for c in f.corner if tuple(c) != (0, 0, 0)]
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                leaves.append((1, (dx * N, dy * N, dz * N)))
    leaves.sort()
    lv = np.array([l for l, _ in leaves], dtype=np.int32)
    cn = np.array([c for _, c in leaves], dtype=np.int32)
    return tgh.Forest(N, f.lo, f.h0, f.cells0, f.periodic, lv, cn)
