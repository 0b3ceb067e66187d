"""The allocation-free speed entry point, tgh_max_speed_noalloc, through the C ABI.

It is for callers that cannot allocate device memory (another allocator owns the device,
or the loop asking for the time step may not allocate): it keeps its scratch in a fixed
device array inside the library instead. Its answer must be the speed tgh_max_speed gives
for the same state, call after call (the shared array keeps the previous call's contents,
so a second call checks that what must start at zero is cleared). This file is collected
last so that a stopping run has executed every other test before it.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc_speed(tgh, case, forest, q, u, t):
    lib = tgh.load_library()
    cfg = case.config(q)
    mesh = forest.mesh()
    lam = ctypes.c_double()
    err = ctypes.create_string_buffer(256)
    st = lib.tgh_max_speed_noalloc(ctypes.byref(cfg), ctypes.byref(mesh), ctypes.c_void_p(u.data_ptr()), float(t),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(lam), err,
                                   256)
    return st, lam.value, err.value.decode()


def test_noalloc_speed_matches_max_speed_twice(tgh):
    # a hole with an interior (the mask matters) and a flat periodic case, alternated, so that
    # the second call on each sees the other's leftovers in the shared array
    rows = []
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    rows.append((c, tgh.gh_forest(c, 8, 2), 0.0))
    c = tgh.perturbed_minkowski_case()
    rows.append((c, tgh.gh_forest(c, 8, 2), 0.0))
    probs = []
    for case, forest, t in rows:
        P = tgh.GHProblem(case, forest, 4, margin_check=False)
        u = P.initial_state(P.statevector(), t)
        if case.interior is None:
            u += torch.from_numpy(tgh.perturbation(forest, amplitude=1e-3)).cuda()
        probs.append((case, forest, t, P, u, P.max_speed(u, t)))
    for _ in range(2):
        for case, forest, t, P, u, lam in probs:
            st, got, msg = _noalloc_speed(tgh, case, forest, 4, u, t)
            assert st == tgh._abi.TGH_OK, msg
            assert got == pytest.approx(lam, rel=1e-15)


def test_noalloc_speed_refuses_nonfinite_and_large_meshes(tgh):
    c = tgh.minkowski_case(L=1.0)
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4)
    u = P.initial_state(P.statevector(), 0.0)
    u[77] = float("nan")
    st, _, msg = _noalloc_speed(tgh, c, f, 4, u, 0.0)
    assert st == tgh._abi.TGH_ERR_NONFINITE and "not finite" in msg
    u[77] = 0.0
    st, lam, _ = _noalloc_speed(tgh, c, f, 4, u, 0.0)
    assert st == tgh._abi.TGH_OK and lam == pytest.approx(3 ** 0.5, rel=1e-15)
    big = tgh.gh_forest(tgh.minkowski_case(L=1.0), 8, 21)  # 9261 blocks > the fixed table
    st, _, msg = _noalloc_speed(tgh, c, big, 4, u, 0.0)
    assert st == tgh._abi.TGH_ERR_ARG and "at most" in msg
