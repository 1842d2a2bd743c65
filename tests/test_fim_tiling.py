"""The temporally blocked schedule of the fast iterative method (k_fim_tiled) restated on the CPU: 32 x 32
tiles, each iterating HALO / 2 times on its tile plus a halo of HALO cells read at the launch's start (the
neighbours' values outside the image replaced by the 'large' stand-in), tiles with no active cell in their
image (or, on the first launch, no active tile around them) left unchanged.  After every launch the owned
cells equal the two-phase global iteration's, and after the 10 iterations the oracle's level set, for both
halos the CUDA kernel uses (4 and 20).  CPU only: the schedule, not the kernel."""
import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

F = np.float32
LARGE, EPS, SQ2 = F(1e30), F(1e-6), F(1.41421356237309504880)
NONE, SOURCE, ACTIVE, CONV = 0, 1, 2, 3
TILE = 32


def _sign(v):
    return F(1) if v > 0 else (F(-1) if v < 0 else F(0))


def _quad(get, x, y):  # solve_quadratic_2d (fast_iterative_method/update.wgsl:62-83)
    xm = min(get(x - 1, y), get(x + 1, y))
    ym = min(get(x, y - 1), get(x, y + 1))
    d = F(xm - ym)
    if d > SQ2:
        return F(ym + F(1))
    if d < -SQ2:
        return F(xm + F(1))
    return F(F(0.5) * F(F(xm + ym) + np.sqrt(F(F(2) - F(d * d)))))


def _init(ls1):  # initialize.wgsl, initialize_active_label.wgsl
    H, W = ls1.shape
    S = np.empty_like(ls1)
    lab0 = np.zeros((H, W), np.uint32)
    nb = ((-1, 0), (1, 0), (0, -1), (0, 1))
    for y in range(H):
        for x in range(W):
            lv = ls1[y, x]
            src = any(0 <= x + dx < W and 0 <= y + dy < H and F(lv * ls1[y + dy, x + dx]) <= 0 for dx, dy in nb)
            S[y, x], lab0[y, x] = (lv, SOURCE) if src else (_sign(lv) * LARGE, NONE)
    L = np.where(lab0 == SOURCE, SOURCE, NONE).astype(np.uint32)
    for y in range(H):
        for x in range(W):
            if lab0[y, x] != SOURCE and any(0 <= x + dx < W and 0 <= y + dy < H and lab0[y + dy, x + dx] == SOURCE
                                            for dx, dy in nb):
                L[y, x] = ACTIVE
    return S, L


def _iterate(S, L, iters, box=None):
    """Two-phase iterations in place; box = (x0, y0, x1, y1): only the image, neighbours outside it 'large'."""
    H, W = S.shape
    x0, y0, x1, y1 = box or (0, 0, W, H)
    inside = lambda x, y: max(0, x0) <= x < min(W, x1) and max(0, y0) <= y < min(H, y1)  # noqa: E731
    cells = [(x, y) for y in range(max(0, y0), min(H, y1)) for x in range(max(0, x0), min(W, x1))]
    for _ in range(iters):
        T, LT = S.copy(), L.copy()
        ab = lambda A, x, y: F(abs(A[y, x])) if inside(x, y) else LARGE  # noqa: E731
        for x, y in cells:
            if L[y, x] == ACTIVE:
                p = S[y, x]
                q = F(_quad(lambda a, b: ab(S, a, b), x, y) * _sign(p))
                T[y, x], LT[y, x] = q, (ACTIVE if abs(F(p - q)) > EPS else CONV)
        for x, y in cells:
            lv, tv = LT[y, x], T[y, x]
            if lv == NONE:
                w = next(((x + dx, y + dy) for dx, dy in ((0, 1), (1, 0), (-1, 0), (0, -1))
                          if inside(x + dx, y + dy) and LT[y + dy, x + dx] == CONV), None)
                if w is not None:
                    qn = _quad(lambda a, b: ab(T, a, b), x, y)
                    if F(abs(tv)) > qn:
                        S[y, x], L[y, x] = F(qn * _sign(T[w[1], w[0]])), ACTIVE
                        continue
                S[y, x], L[y, x] = tv, NONE
            else:
                S[y, x], L[y, x] = tv, (NONE if lv == CONV else lv)


def _tiled(S, L, iters, halo):
    H, W = S.shape
    tx, ty = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    flags = np.zeros((ty, tx), bool)
    for y, x in np.argwhere(L == ACTIVE):
        flags[y // TILE, x // TILE] = True
    k = 0
    while k < iters:
        n = min(halo // 2, iters - k)
        S2, L2 = S.copy(), L.copy()  # the launch's output planes; reads see the launch's start
        for by in range(ty):
            for bx in range(tx):
                if k == 0 and not flags[max(0, by - 1):by + 2, max(0, bx - 1):bx + 2].any():
                    continue
                box = (bx * TILE - halo, by * TILE - halo, bx * TILE + TILE + halo, by * TILE + TILE + halo)
                img = (slice(max(0, box[1]), min(H, box[3])), slice(max(0, box[0]), min(W, box[2])))
                if not (L[img] == ACTIVE).any():
                    continue
                Si, Li = S.copy(), L.copy()
                _iterate(Si, Li, n, box)
                own = (slice(by * TILE, min(H, by * TILE + TILE)), slice(bx * TILE, min(W, bx * TILE + TILE)))
                S2[own], L2[own] = Si[own], Li[own]
        S, L = S2, L2
        k += n
    return S, L


@pytest.mark.parametrize("halo", [4, 20])
def test_tiled_schedule_equals_two_phase_and_oracle(oracle_api, halo):
    sc = scenes.batch(1, seed=0xC5, shapes=[(96, 64)]).scenes[0]
    sim = sc.make(oracle_api)
    for _ in range(4):
        sim.step(sc.dt)
    ls1 = sim.get(capi.FIELD_LEVELSET_AIR1).astype(F)
    S, L = _init(ls1)
    Sg, Lg = S.copy(), L.copy()
    _iterate(Sg, Lg, 10)
    assert np.array_equal(Sg, sim.get(capi.FIELD_LEVELSET_AIR).astype(F))  # the restatement is the oracle's
    St, Lt = _tiled(S, L, 10, halo)
    assert np.array_equal(St, Sg) and np.array_equal(Lt, Lg)
    sim.close()
