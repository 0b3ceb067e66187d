"""Forests of closed vertex-centered blocks: the leaves a problem runs on.

A leaf is (level, integer corner) with N cells per edge; level l has spacing h0 / 2^l. The
builders mirror the reference's gh_forest (uniform roots) and hole_forest (nested shells of
refinement around a hole, src/initialdata.jl:1370-1515), with 2:1 balance across faces,
edges and corners, which is what TreeAMR's regrid guarantees.
"""
from dataclasses import dataclass
import ctypes

import numpy as np

from . import _abi


@dataclass
class Forest:
    N: int
    lo: tuple
    h0: float
    cells0: tuple
    periodic: tuple
    level: np.ndarray       # int32 [nblocks]
    corner: np.ndarray      # int32 [nblocks, 3]

    @property
    def nblocks(self):
        return int(self.level.shape[0])

    @property
    def nlevels(self):
        return int(self.level.max()) + 1

    def points(self):
        """Owned points counted N^3 per block (the reference's point count)."""
        return self.nblocks * self.N ** 3

    def mesh(self):
        m = _abi.Mesh()
        m.N = self.N
        m.nblocks = self.nblocks
        for d in range(3):
            m.lo[d] = self.lo[d]
            m.cells0[d] = self.cells0[d]
            m.periodic[d] = 1 if self.periodic[d] else 0
        m.h0 = self.h0
        self._lv = np.ascontiguousarray(self.level, dtype=np.int32)
        self._cn = np.ascontiguousarray(self.corner.reshape(-1), dtype=np.int32)
        m.level = self._lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        m.corner = self._cn.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        return m

    def block_positions(self, b):
        """Positions (x, y, z) of block b's (N+1)^3 owned points, x fastest."""
        h = self.h0 / 2 ** int(self.level[b])
        idx = np.arange(self.N + 1, dtype=np.float64)
        xs = [self.lo[d] + (self.corner[b, d] + idx) * h for d in range(3)]
        z, y, x = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        return x, y, z


def gh_forest(case, N, roots):
    """roots^3 level-0 blocks of N cells over the case's box (gh_forest)."""
    r = (roots,) * 3 if np.isscalar(roots) else tuple(roots)
    lo = tuple(b[0] for b in case.box)
    ext = [case.box[d][1] - case.box[d][0] for d in range(3)]
    h0 = ext[0] / (r[0] * N)
    for d in range(3):
        if abs(ext[d] / (r[d] * N) - h0) > 1e-14 * h0:
            raise ValueError("the box must have the same spacing along every axis")
    corners = np.array([(i * N, j * N, k * N) for k in range(r[2]) for j in range(r[1]) for i in range(r[0])],
                       dtype=np.int32)
    return Forest(N, lo, h0, tuple(ri * N for ri in r), tuple(case.periodic),
                  np.zeros(len(corners), dtype=np.int32), corners)


def _balance(leaves, N, cells0):
    """Refine until neighbouring leaves (faces, edges, corners) differ by at most one level."""
    changed = True
    while changed:
        changed = False
        byl = {}
        for (l, c) in leaves:
            byl.setdefault(l, set()).add(c)
        maxl = max(byl)
        refine = set()
        for (l, c) in leaves:
            # a leaf at level l must not touch a leaf at level >= l + 2
            for lf in range(l + 2, maxl + 1):
                s = 2 ** (lf - l)
                bc = tuple(ci // N for ci in c)
                # the leaf's box in level-lf block coordinates, grown by one block
                lo = [bc[d] * s - 1 for d in range(3)]
                hi = [(bc[d] + 1) * s for d in range(3)]
                for c2 in byl.get(lf, ()):
                    b2 = tuple(ci // N for ci in c2)
                    if all(lo[d] <= b2[d] <= hi[d] for d in range(3)):
                        refine.add((l, c))
                        break
                if (l, c) in refine:
                    break
        if refine:
            changed = True
            new = []
            for (l, c) in leaves:
                if (l, c) in refine:
                    for dz in (0, 1):
                        for dy in (0, 1):
                            for dx in (0, 1):
                                new.append((l + 1, (2 * c[0] + dx * N, 2 * c[1] + dy * N, 2 * c[2] + dz * N)))
                else:
                    new.append((l, c))
            leaves = new
    return leaves


def hole_forest(case, N, roots, radii, centre=(0.0, 0.0, 0.0), path=None):
    """Nested refinement around a hole: level l's leaves whose box comes within radii[l] of the
    centre (or of the segment `path` = (start, end) the centre sweeps) are refined, level by
    level, then the forest is 2:1 balanced (hole_forest, src/initialdata.jl:1469-1515)."""
    base = gh_forest(case, N, roots)
    leaves = [(0, tuple(int(v) for v in c)) for c in base.corner]
    p0 = np.array(centre if path is None else path[0], dtype=float)
    p1 = np.array(centre if path is None else path[1], dtype=float)

    def dist_box(lo, hi):
        # distance from the segment p0-p1 to the box, sampled along the segment
        best = np.inf
        for s in np.linspace(0.0, 1.0, 33):
            c = p0 + s * (p1 - p0)
            d = np.maximum(0.0, np.maximum(lo - c, c - hi))
            best = min(best, float(np.sqrt((d * d).sum())))
        return best

    for l, R in enumerate(radii):
        h = base.h0 / 2 ** l
        new = []
        for (lv, c) in leaves:
            if lv == l:
                lo = np.array(base.lo) + np.array(c) * h
                hi = lo + N * h
                if dist_box(lo, hi) < R:
                    for dz in (0, 1):
                        for dy in (0, 1):
                            for dx in (0, 1):
                                new.append((l + 1, (2 * c[0] + dx * N, 2 * c[1] + dy * N, 2 * c[2] + dz * N)))
                    continue
            new.append((lv, c))
        leaves = _balance(new, N, base.cells0)
    leaves.sort()
    level = np.array([l for (l, c) in leaves], dtype=np.int32)
    corner = np.array([c for (l, c) in leaves], dtype=np.int32)
    return Forest(N, base.lo, base.h0, base.cells0, base.periodic, level, corner)
