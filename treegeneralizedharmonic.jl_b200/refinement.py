"""The refinement criterion: the masked Loehner indicator reduced to one mark per block, with a
level floor around the horizon and a level ceiling at the outer boundary (src/refinement.jl).

The per-point work runs on the GPU (include/tgh.h, "the refinement indicator"): the masked
reference amplitude (field_scales), tau at every owned point into the diag field set, its
maximum, and the two firing sweeps (per block: how many points exceed a threshold, and the
bounding box of their nodes). What is per block runs here, as the reference runs it on the
host at regrid cadence: the level bounds (pure functions of position), the four marks,
the travelling margin and the refinement centroid.

The mesh package the reference flags for (TreeAMR 0.3) is not vendored; its firing_boxes and
buffered_flags are restated from the reference's own description of them
(src/refinement.jl:670-830, test/refinement_tests.jl:143-215): a block's box is in cell
indices, the cells touching the firing nodes, max(1, lo - 1):min(N, hi) (1-based), and the
margin widens every reported box by `buffer` cells and promotes the leaves it reaches to the
level its source asks for (the source's level + 1 for Refine, its own for Keep).
"""
import math
from dataclasses import dataclass

import numpy as np

REFINE, KEEP, COARSEN = "Refine", "Keep", "Coarsen"
MAX_LEVEL = 30


@dataclass(frozen=True)
class Refinement:
    """Refinement(refine_tol, coarsen_tol, maxlevel_cap, floor_margin, ceiling_cells=1,
    ceiling_level=0, eps=1/100): the thresholds, the cap the indicator may reach, the floor's
    margin beyond the horizon, the ceiling's margin in coarse cells and its level, and the
    Loehner noise floor's coefficient (src/refinement.jl:91-152, with its checks)."""
    refine_tol: float
    coarsen_tol: float
    maxlevel_cap: int
    floor_margin: float
    ceiling_cells: int = 1
    ceiling_level: int = 0
    eps: float = 1 / 100

    def __post_init__(self):
        if not 0 < self.coarsen_tol < self.refine_tol:
            raise ValueError("the thresholds must satisfy 0 < coarsen_tol < refine_tol: the gap between them is "
                             f"the hysteresis dead band (coarsen_tol = {self.coarsen_tol}, "
                             f"refine_tol = {self.refine_tol})")
        if not self.refine_tol < 1:
            raise ValueError(f"refine_tol = {self.refine_tol}, but tau lies in [0, 1] by construction, so a "
                             "threshold at or above 1 can never fire")
        if self.maxlevel_cap < 0:
            raise ValueError(f"maxlevel_cap must be non-negative, got {self.maxlevel_cap}")
        if self.floor_margin < 0:
            raise ValueError(f"the floor's margin cannot be negative, got {self.floor_margin}")
        if self.ceiling_cells < 0:
            raise ValueError(f"the ceiling's margin is a number of coarse cells, got {self.ceiling_cells}")
        if not 0 <= self.ceiling_level <= self.maxlevel_cap:
            raise ValueError(f"the ceiling's level must lie between 0 and maxlevel_cap = {self.maxlevel_cap}, "
                             f"got {self.ceiling_level}")
        if not self.eps > 0:
            raise ValueError(f"the Loehner noise floor's coefficient must be positive, got {self.eps}")


def lohner(um, u0, up, scale, eps=1 / 100):
    """|u+ - 2 u0 + u-| / (|u+ - u0| + |u0 - u-| + 4 eps |scale|), 0 where the denominator is
    (src/refinement.jl:179-183); the device computes the same, rounded the same way."""
    num = abs(up - 2 * u0 + um)
    den = abs(up - u0) + abs(u0 - um) + 4 * eps * abs(scale)
    return 0.0 if den == 0 else num / den


# ---- where a block is ----
def spacing(forest, level):
    return forest.h0 / 2 ** int(level)


def block_extent(forest, b):
    """((lo, hi) x 3) of leaf b, the closed box its nodes span."""
    h = spacing(forest, forest.level[b])
    return tuple((forest.lo[d] + int(forest.corner[b][d]) * h, forest.lo[d] + (int(forest.corner[b][d]) + forest.N) * h)
                 for d in range(3))


def horizon_radii(case):
    """(r_h,min, r_h,max): the smallest and largest coordinate radius of the hole's horizon
    about the hole's center (src/interior.jl:756-800). A boost contracts the rest frame's
    horizon ellipsoid x^T A x = 1 along the velocity; the smallest radius is then
    1 / sqrt(largest eigenvalue of L A L), L the boost's spatial matrix."""
    bg = case.background
    if bg.get("kind") not in ("kerr_schild", "harmonic_kerr"):
        raise ValueError("the level floor needs a hole: a Kerr-Schild or harmonic Kerr background")
    M, a = bg["M"], bg.get("a", 0.0)
    # the horizon's spheroidal radius: r_+ in Kerr-Schild, r_+ - M in the harmonic chart
    r_min = (M if bg["kind"] == "kerr_schild" else 0.0) + math.sqrt(M * M - a * a)
    r_max = math.sqrt(r_min * r_min + a * a)
    v = np.array(bg.get("boost", (0.0, 0.0, 0.0)), dtype=float)
    b2 = float(v @ v)
    if b2 == 0.0:
        return r_min, r_max
    contracted = r_min * math.sqrt(1.0 - b2)
    A = np.diag([1.0 / (r_min * r_min + a * a), 1.0 / (r_min * r_min + a * a), 1.0 / (r_min * r_min)])
    vh = v / math.sqrt(b2)
    if vh @ A @ vh >= (1 - 1e-12) / r_min ** 2:
        return contracted, r_max
    g = 1.0 / math.sqrt(1.0 - b2)
    L = np.eye(3) + (g - 1.0) / b2 * np.outer(v, v)
    lam = np.linalg.eigvalsh(L @ A @ L)
    return 1.0 / math.sqrt(lam.max()), r_max


def horizon_floor_level(forest, case, G):
    """The coarsest level whose spacing meets both interior radius requirements,
    h <= (r_h,min - r_1) / m and h <= (r_1 - r_0) / (2 (G + 1)) (src/refinement.jl:448-485)."""
    it = case.interior
    r_h, _ = horizon_radii(case)
    r0, r1, m = it["r0"], it["r1"], it.get("margin", 8)
    if not r_h > r1:
        raise ValueError(f"the layer's outer radius r_1 = {r1} is not inside the horizon's smallest coordinate "
                         f"radius r_h,min = {r_h}: no refinement level can satisfy r_1 <= r_h,min - m h")
    need = min((r_h - r1) / m, (r1 - r0) / (2 * (G + 1)))
    lev, h = 0, spacing(forest, 0)
    while h > need and lev < MAX_LEVEL:
        lev += 1
        h /= 2
    return lev


@dataclass
class LevelBounds:
    """Where the floor and the ceiling apply (src/refinement.jl:402-414): the hole's center, the
    floor's shell [floor_lo, floor_hi] (empty when floor_hi < floor_lo) and level, the box, its
    periodic axes, the ceiling's margin and level, and the cap."""
    forest: object
    center: tuple
    floor_lo: float
    floor_hi: float
    floor_level: int
    box: tuple
    periodic: tuple
    ceiling_margin: float
    ceiling_level: int
    maxlevel_cap: int


def level_bounds(case, forest, t, G, ref, travel=0.0):
    """The floor and the ceiling at time t (src/refinement.jl:514-590): the floor's shell
    r_1 - travel <= r <= r_h,max + floor_margin + travel around the hole's center at t, at
    horizon_floor_level; the ceiling ceiling_cells root cells in from every non-periodic face."""
    it = case.interior
    if it is None:
        c, lo, hi, L = (0.0, 0.0, 0.0), 0.0, -1.0, 0
    else:
        c = tuple(it["c0"][d] + t * it.get("v", (0, 0, 0))[d] for d in range(3))
        lo = max(it["r1"] - travel, 0.0)
        hi = horizon_radii(case)[1] + ref.floor_margin + travel
        L = horizon_floor_level(forest, case, G)
    if L > ref.maxlevel_cap:
        raise ValueError(f"the interior's radius requirements need level {L} around this hole, but maxlevel_cap "
                         f"is {ref.maxlevel_cap}: raise the cap, start from a finer root grid, or move the layer's "
                         "radii outward")
    return LevelBounds(forest, c, lo, hi, L, case.box, case.periodic, ref.ceiling_cells * spacing(forest, 0),
                       ref.ceiling_level, ref.maxlevel_cap)


def _box_radii(ext, c):
    near, far = 0.0, 0.0
    for d in range(3):
        lo, hi = ext[d]
        gap = max(lo - c[d], c[d] - hi, 0.0)
        near += gap * gap
        far += max((c[d] - lo) ** 2, (hi - c[d]) ** 2)
    return math.sqrt(near), math.sqrt(far)


def _box_meets_shell(ext, c, lo, hi):
    if hi < lo:
        return False
    near, far = _box_radii(ext, c)
    return near <= hi and far >= lo


def _box_near_boundary(ext, box, periodic, margin):
    for d in range(3):
        if periodic[d]:
            continue
        if ext[d][0] - box[d][0] <= margin or box[d][1] - ext[d][1] <= margin:
            return True
    return False


def block_level_bounds(lb, b):
    """(floor, ceiling) of leaf b (src/refinement.jl:638-668); a floor above the ceiling is refused."""
    ext = block_extent(lb.forest, b)
    flo = lb.floor_level if lb.floor_level > 0 and _box_meets_shell(ext, lb.center, lb.floor_lo, lb.floor_hi) else 0
    cap = lb.ceiling_level if _box_near_boundary(ext, lb.box, lb.periodic, lb.ceiling_margin) else lb.maxlevel_cap
    if flo > cap:
        raise ValueError(f"the level floor and the ceiling disagree about the block {ext}: the horizon shell asks "
                         f"for level {flo} there and the boundary margin caps it at {cap}; widen the box, shrink "
                         "the floor's margin, or lower the ceiling's margin")
    return flo, cap


# ---- the marks ----
def cell_box(forest, lo, hi):
    """The cells touching the firing nodes lo..hi (0-based), as 1-based inclusive ranges."""
    N = forest.N
    return tuple((max(1, int(lo[d])), min(N, int(hi[d]) + 1)) for d in range(3))


def _mark_level(mark, lev):
    kind = mark[0] if isinstance(mark, tuple) else mark
    return lev + 1 if kind == REFINE else (max(lev - 1, 0) if kind == COARSEN else lev)


def refine_flags(forest, lb, ref, counts, boxes, buffer=0):
    """The four marks per leaf (src/refinement.jl:738-780) from the two firing sweeps, counts[b]
    and boxes[b] for (refine_tol, coarsen_tol) in that order:
        tau > refine_tol somewhere, level < cap  -> (Refine, box)
        the coarsen_tol sweep fired               -> (Keep, box)
        nothing fired, level > 0                  -> Coarsen
        otherwise                                 -> Keep
    each request clamped between the block's floor and ceiling; the box is the coarsen_tol
    sweep's. With buffer > 0 the travelling margin is applied and the bounds again."""
    marks = []
    for b in range(len(forest.level)):
        lev = int(forest.level[b])
        flo, cap = block_level_bounds(lb, b)
        nref, nbox = int(counts[b][0]), int(counts[b][1])
        box = cell_box(forest, boxes[b][1][:3], boxes[b][1][3:]) if nbox > 0 else None
        if nref > 0 and lev < cap:
            request = lev + 1
        elif nbox > 0:
            request = lev
        else:
            request = max(lev - 1, 0)
        target = min(max(request, flo), cap)
        if target > lev:
            marks.append((REFINE, box) if nbox > 0 else REFINE)
        elif target < lev:
            marks.append(COARSEN)
        else:
            marks.append((KEEP, box) if nbox > 0 else KEEP)
    return buffered_marks(lb, marks, buffer) if buffer > 0 else marks


def buffered_marks(lb, marks, buffer):
    """The travelling margin (src/refinement.jl:797-830): every reported box widened by `buffer`
    cells promotes the leaves it reaches to the level its source asks for (level + 1 for Refine,
    level for Keep); the marks come out bare, and the floor and the ceiling are applied again."""
    f = lb.forest
    nb = len(f.level)
    want = [_mark_level(m, int(f.level[b])) for b, m in enumerate(marks)]
    ext = [block_extent(f, b) for b in range(nb)]
    for s, m in enumerate(marks):
        if not isinstance(m, tuple) or m[1] is None:
            continue
        lev = int(f.level[s])
        h = spacing(f, lev)
        o = [e[0] for e in ext[s]]
        wide = tuple((o[d] + (m[1][d][0] - 1 - buffer) * h, o[d] + (m[1][d][1] + buffer) * h) for d in range(3))
        ask = lev + 1 if m[0] == REFINE else lev
        for b in range(nb):
            if b == s:
                continue
            if all(max(wide[d][0], ext[b][d][0]) < min(wide[d][1], ext[b][d][1]) for d in range(3)):
                want[b] = max(want[b], ask)
    out = []
    for b in range(nb):
        lev = int(f.level[b])
        flo, cap = block_level_bounds(lb, b)
        target = min(max(want[b], flo), cap)
        out.append(REFINE if target > lev else (COARSEN if target < lev else KEEP))
    return out


def refinement_centroid(forest, counts, boxes):
    """The volume-weighted centroid of the coarsen_tol sweep's boxes (src/refinement.jl:875-930):
    each firing block's box center, o + ((first + last)/2 - 1/2) h per axis, weighted by its
    firing count and cell volume; None when nothing fired."""
    num, den = np.zeros(3), 0.0
    for b in range(len(forest.level)):
        n = int(counts[b][1])
        if n == 0:
            continue
        h = spacing(forest, forest.level[b])
        o = [e[0] for e in block_extent(forest, b)]
        box = cell_box(forest, boxes[b][1][:3], boxes[b][1][3:])
        x = np.array([o[d] + ((box[d][0] + box[d][1]) / 2 - 0.5) * h for d in range(3)])
        w = n * h ** 3
        num += w * x
        den += w
    return None if den == 0 else num / den


def refinement_buffer(forest, maxlevel_cap, travel):
    """The margin in cells that covers a feature moving `travel` between regrids, at the cap's
    spacing: ceil(travel / h) + 1, at most N (src/refinement.jl:931-945)."""
    h = spacing(forest, maxlevel_cap)
    cells = math.ceil(travel / h) + 1
    if cells > forest.N:
        raise ValueError(f"a hole travelling {travel} between regrids needs a {cells}-cell margin at level "
                         f"{maxlevel_cap} (h = {h}), more than the block width N = {forest.N}: shorten the chunk "
                         "or lower the cap")
    return cells


def regrid_forest(forest, flags):
    """The leaves after one regrid on bare or boxed marks (TreeAMR's regrid! with buffer = 0, as
    the reference's driver calls it): a Refine leaf becomes its eight children; eight siblings
    that are all marked Coarsen become their parent; then the forest is made 2:1 balanced by
    refining (a coarsened parent next to a leaf two levels finer is refined back). Returns a new
    Forest with the leaves sorted by level, then corner with x fastest (gh_forest's order, so
    that a forest that did not change keeps its block numbering)."""
    from .forest import Forest, _balance
    N = forest.N
    leaves = [(int(l), tuple(int(x) for x in c)) for l, c in zip(forest.level, forest.corner)]
    if len(flags) != len(leaves):
        raise ValueError(f"{len(flags)} marks for {len(leaves)} leaves")
    kind = [m[0] if isinstance(m, tuple) else m for m in flags]

    def parent(l, c):
        return l - 1, tuple((ci // N) // 2 * N for ci in c)

    groups = {}
    for (l, c), k in zip(leaves, kind):
        if k == COARSEN and l > 0:
            groups.setdefault(parent(l, c), []).append((l, c))
    whole = {pk for pk, ch in groups.items() if len(ch) == 8}
    new, done = [], set()
    for (l, c), k in zip(leaves, kind):
        if k == REFINE:
            for dz in (0, 1):
                for dy in (0, 1):
                    for dx in (0, 1):
                        new.append((l + 1, (2 * c[0] + dx * N, 2 * c[1] + dy * N, 2 * c[2] + dz * N)))
        elif k == COARSEN and l > 0 and parent(l, c) in whole:
            pk = parent(l, c)
            if pk not in done:
                done.add(pk)
                new.append(pk)
        else:
            new.append((l, c))
    new = sorted(_balance(new, N, forest.cells0), key=lambda lc: (lc[0], lc[1][2], lc[1][1], lc[1][0]))
    return Forest(N, forest.lo, forest.h0, forest.cells0, forest.periodic,
                  np.array([l for l, _ in new], dtype=np.int32), np.array([c for _, c in new], dtype=np.int32))


def regrid(P, u, t, flags):
    """regrid! and the rebuild after it (src/driver.jl:1660-1695): the regridded forest, a new
    problem on it (same case and order; the gauge source is sampled anew), the state transferred
    with this t's hook, and the stage limiter applied to it (the pasted variant's paste; the
    prolongation into a fresh block is unlimited). Returns (problem, state)."""
    from .problem import GHProblem
    f2 = regrid_forest(P.forest, flags)
    P2 = GHProblem(P.case, f2, P.q, margin_check=P.margin_check, precision=P.precision, stream=P.stream)
    u2 = P2.statevector()
    P2.transfer_from(P, u, t, u2)
    P2.stage_limit(u2, t)
    return P2, u2


def indicator_flags(P, case, u, t, ref, G=None, buffer=0, travel=0.0, mask="interior"):
    """indicator_flags / gh_indicator! (src/refinement.jl:973-1025) on a problem's own mesh: the
    masked reference amplitude, tau into the diag field set, then the marks with the level
    bounds. Returns flags, tau_max, centroid, nfiring, scale."""
    G = P.q // 2 + 1 if G is None else G
    r = P.tau(u, t, eps=ref.eps, mask=mask)
    counts, boxes = P.firing([ref.refine_tol, ref.coarsen_tol])
    lb = level_bounds(case, P.forest, t, G, ref, travel=travel)
    flags = refine_flags(P.forest, lb, ref, counts, boxes, buffer=buffer)
    return {"flags": flags, "tau_max": r["tau_max"], "centroid": refinement_centroid(P.forest, counts, boxes),
            "nfiring": int(sum(int(c[1]) for c in counts)), "scale": r["scale"], "scales": r["scales"]}
