#!/usr/bin/env python
"""Shared-memory wavefront model of the stage kernel's passes.

Reproduces the layout constants of csrc/dg_stage.cuh: the point-array row
stride (qs_stride), the task order of every pass (TaskOrd) and, at p = 3, the
rotated rows of the coefficient blocks (Lay::cw).

Hardware model (B200 shared memory, 32 banks of 4 bytes, one 128-byte
wavefront per SM and cycle):
  * an 8-byte (FP64) warp access is served per half-warp: 16 lanes, bank pair
    = word % 16; a half-warp costs max over bank pairs of the number of
    distinct words on it (broadcasts are free);
  * a 4-byte (FP32) warp access: 32 lanes, bank = word % 32, same rule.
Each pass is a loop `for (i = tid; i < ntask; i += NT)` whose task i decodes
into coordinates in a chosen order; a warp holds 32 consecutive tasks, so
the count does not depend on NT. Each task's accesses are listed in program
order; the model sums the wavefronts of every warp-wide access.

Passes modelled (per element, E = 1; the face-flux variant, non-row-split
lift): x interpolation (coefficients -> X1), y interpolation (X1 -> X2), z
interpolation in place, pointwise flux (5 rows -> 15 rows), z / y / x
contractions, lift, lift gather into the residual, inverse-mass x and y
passes and the update (z pencils); with the launch option MG the lift gather
and the inverse-mass x pass are one pass (minvxg).

    python tests/bank_model.py 3 8      # p = 3, FP64 work area
    python tests/bank_model.py 5 4 --search

Design tool only: nothing in the library imports it.
"""
from __future__ import annotations

import argparse
import itertools
from collections import defaultdict


def wavefronts(addrs, word):
    """addrs: list of (lane, word address or None) of one warp access."""
    if word == 8:
        tot = 0
        for half in (0, 1):
            grp = [a for t, a in addrs if t // 16 == half and a is not None]
            if grp:
                banks = defaultdict(set)
                for a in grp:
                    banks[a % 16].add(a)
                tot += max(len(s) for s in banks.values())
        return tot
    grp = [a for t, a in addrs if a is not None]
    if not grp:
        return 0
    banks = defaultdict(set)
    for a in grp:
        banks[a % 32].add(a)
    return max(len(s) for s in banks.values())


def ideal_wavefronts(addrs, word):
    lanes = [t for t, a in addrs if a is not None]
    if not lanes:
        return 0
    return len({t // 16 for t in lanes}) if word == 8 else 1


def decode(r, dims, order):
    """task index r -> {name: coordinate}; order lists names fastest first."""
    idx = {}
    for name in order:
        idx[name] = r % dims[name]
        r //= dims[name]
    return idx


def pass_cost(dims, order, accesses):
    """accesses: list of (function task -> list of addresses, word bytes)."""
    ntask = 1
    for n in dims.values():
        ntask *= n
    tasks = [decode(i, dims, order) for i in range(ntask)]
    tot = ideal = 0
    for fn, word in accesses:
        lists = [fn(t) for t in tasks]
        for w0 in range(0, ntask, 32):
            lanes = lists[w0:w0 + 32]
            for k in range(len(lanes[0])):
                a = [(j, lanes[j][k]) for j in range(len(lanes))]
                tot += wavefronts(a, word)
                ideal += ideal_wavefronts(a, word)
    return tot, ideal


# --- the header's constants ---------------------------------------------------

def qs_stride(p, nbytes):
    return {2: 79, 3: 127 if nbytes == 8 else 126, 4: 223 if nbytes == 8 else 231,
            5: 349 if nbytes == 8 else 343}.get(p, ((p + 2) ** 3) | 1)


def order3(code, names):
    """TaskOrd 3-coordinate code f + 3m + 9s -> names fastest first."""
    return (names[code % 3], names[(code // 3) % 3], names[code // 9])


def order2(code, names):
    return (names[0], names[1]) if code == 0 else (names[1], names[0])


def task_orders(p, nbytes):
    """TaskOrd<P, BYTES> of dg_stage.cuh, as name tuples (fastest first)."""
    w8 = nbytes == 8
    x = 1 if p >= 3 or (p == 2 and not w8) else 0
    y = {2: 11, 3: 5, 4: 5 if w8 else 21, 5: 21 if w8 else 11}.get(p, 21)
    z = 1 if p == 5 and w8 else 0
    zc = {2: 0 if w8 else 1, 3: 1, 4: 1 if w8 else 0}.get(p, 0)
    yc = {2: 21 if w8 else 11, 3: 21 if w8 else 5, 4: 21 if w8 else 11, 5: 19 if w8 else 21}.get(p, 7)
    xc = 1 if p >= 3 or (p == 2 and not w8) else 0
    gather = 1 if p == 4 else 0
    minvx = 1 if p >= 2 else 0
    minvy = {2: 11, 3: 7, 4: 11, 5: 7}.get(p, 21)
    minvxg = 0 if p == 5 and w8 else 1
    return {
        "x": order2(x, ("v", "byz")), "y": order3(y, ("v", "qx", "bz")), "z": order2(z, ("qxy", "v")),
        "zc": order2(zc, ("qxy", "v")), "yc": order3(yc, ("v", "qx", "bz")), "xc": order2(xc, ("v", "byz")),
        "gather": order2(gather, ("b", "v")), "minvx": order2(minvx, ("v", "byz")),
        "minvy": order3(minvy, ("v", "bx", "bz")), "upd": ("bxy", "v"), "lift": ("v", "f"), "flux": ("q",),
        "minvxg": order2(minvxg, ("v", "byz")),
    }


def coef_word(p, rotated):
    n = p + 1
    if rotated and n == 4:
        return lambda bx, by, bz: 16 * by + 4 * ((bx + by) & 3) + ((bz + bx) & 3)
    return lambda bx, by, bz: (bz * n + by) * n + bx


# --- the passes -----------------------------------------------------------------

def passes(p, W, VS, X1S, QS, FS, cw):
    """name -> (dims, accesses) of every modelled pass (W: work-area bytes)."""
    N, M = p + 1, p + 2
    NF, N2, NB = M * M, N * N, N ** 3
    X1 = 5 * QS  # X1 rows follow the five X2 rows of the point array
    out = {}
    out["x"] = (dict(v=5, byz=N2), [
        (lambda t: [t["v"] * VS + cw(bx, t["byz"] % N, t["byz"] // N) for bx in range(N)], 8),
        (lambda t: [X1 + t["v"] * X1S + t["byz"] * M + qx for qx in range(M)], W)])
    out["y"] = (dict(v=5, qx=M, bz=N), [
        (lambda t: [X1 + t["v"] * X1S + t["bz"] * N * M + by * M + t["qx"] for by in range(N)], W),
        (lambda t: [t["v"] * QS + t["bz"] * NF + qy * M + t["qx"] for qy in range(M)], W)])
    out["z"] = (dict(qxy=NF, v=5), [
        (lambda t: [t["v"] * QS + bz * NF + t["qxy"] for bz in range(N)]
         + [t["v"] * QS + qz * NF + t["qxy"] for qz in range(M)], W)])
    out["flux"] = (dict(q=M * NF), [
        (lambda t: [v * QS + t["q"] for v in range(5)] + [r * QS + t["q"] for r in range(15)], W)])
    out["zc"] = (dict(qxy=NF, v=5), [
        (lambda t: [(3 * t["v"] + d) * QS + qz * NF + t["qxy"] for qz in range(M) for d in range(3)]
         + [(3 * t["v"] + d) * QS + bz * NF + t["qxy"] for bz in range(N) for d in range(3)], W)])
    out["yc"] = (dict(v=5, qx=M, bz=N), [
        (lambda t: [(3 * t["v"] + d) * QS + t["bz"] * NF + qy * M + t["qx"] for qy in range(M) for d in range(3)]
         + [(3 * t["v"] + d) * QS + t["bz"] * NF + by * M + t["qx"] for by in range(N) for d in range(2)], W)])
    out["xc"] = (dict(v=5, byz=N2), [
        (lambda t: [(3 * t["v"] + d) * QS + (t["byz"] // N) * NF + (t["byz"] % N) * M + qx
                    for qx in range(M) for d in range(2)], W),
        (lambda t: [t["v"] * VS + cw(bx, t["byz"] % N, t["byz"] // N) for bx in range(N)], 8)])
    out["lift"] = (dict(v=5, f=6), [
        (lambda t: [(t["f"] * 5 + t["v"]) * FS + t1 * M + t0 for t1 in range(M) for t0 in range(M)]
         + [30 * FS + (t["f"] * 5 + t["v"]) * FS + b1 * N + b0 for b1 in range(N) for b0 in range(N)], W)])

    def lift_rows(t):
        b, v = t["b"], t["v"]
        bc = (b % N, (b // N) % N, b // N2)
        rows = []
        for f in range(6):
            ax = 0 if f in (2, 4) else (1 if f in (1, 3) else 2)
            sidx = N - 1 if f in (2, 3, 5) else 0
            if bc[ax] == sidx:
                b0 = bc[1] if ax == 0 else bc[0]
                b1 = bc[1] if ax == 2 else bc[2]
                rows.append(30 * FS + f * 5 * FS + v * FS + b1 * N + b0)
            else:
                rows.append(None)
        return rows

    out["gather"] = (dict(b=NB, v=5), [
        (lift_rows, W),
        (lambda t: [t["v"] * VS + cw(t["b"] % N, (t["b"] // N) % N, t["b"] // N2)] * 2, 8)])
    out["minvx"] = (dict(v=5, byz=N2), [
        (lambda t: [t["v"] * VS + cw(k, t["byz"] % N, t["byz"] // N) for k in range(N)] * 2, 8)])

    def minvx_lifts(t):
        # launch option MG: the x pencil, the lifted face fluxes on it (x faces at
        # its ends, y / z faces along it when the pencil lies on them), the pencil
        v, by, bz = t["v"], t["byz"] % N, t["byz"] // N
        lift = lambda f, b0, b1: 30 * FS + f * 5 * FS + v * FS + b1 * N + b0
        rows = [v * VS + cw(k, by, bz) for k in range(N)] + [lift(4, by, bz), lift(2, by, bz)]
        for f, c, sidx in ((1, by, 0), (3, by, N - 1), (0, bz, 0), (5, bz, N - 1)):
            other = bz if f in (1, 3) else by
            rows += [lift(f, k, other) if c == sidx else None for k in range(N)]
        return rows + [v * VS + cw(k, by, bz) for k in range(N)]

    out["minvxg"] = (dict(v=5, byz=N2), [(minvx_lifts, W)])
    out["minvy"] = (dict(v=5, bx=N, bz=N), [
        (lambda t: [t["v"] * VS + cw(t["bx"], k, t["bz"]) for k in range(N)] * 2, 8)])
    out["upd"] = (dict(bxy=N2, v=5), [
        (lambda t: [t["v"] * VS + cw(t["bxy"] % N, t["bxy"] // N, k) for k in range(N)] * 3, 8)])
    return out


def kernel_passes(ps, mg=False):
    """the passes one stage runs: with the launch option MG the lift gather and
    the inverse mass's x pass are one pass (minvxg)"""
    drop = ("gather", "minvx") if mg else ("minvxg",)
    return {k: v for k, v in ps.items() if k not in drop}


def count(p, nbytes, QS=None, orders=None, rotated=True, mg=False):
    """per-pass (wavefronts, ideal) with the given stride and orders."""
    N, M = p + 1, p + 2
    VS, X1S, FS = (N ** 3) | 1, (N * N * M) | 1, (M * M) | 1
    QS = QS if QS is not None else qs_stride(p, nbytes)
    orders = orders or task_orders(p, nbytes)
    ps = kernel_passes(passes(p, nbytes, VS, X1S, QS, FS, coef_word(p, rotated)), mg)
    return {name: pass_cost(dims, orders[name], acc) for name, (dims, acc) in ps.items()}


def search(p, nbytes, rotated=True):
    """best point-array stride (within 16 past the block) and per-pass orders;
    the update keeps its z-pencil order (coalesced global writes)."""
    N, M = p + 1, p + 2
    VS, X1S, FS = (N ** 3) | 1, (N * N * M) | 1, (M * M) | 1
    best = None
    for QS in range(M ** 3, M ** 3 + 17):
        ps = kernel_passes(passes(p, nbytes, VS, X1S, QS, FS, coef_word(p, rotated)))
        total, chosen = 0, {}
        for name, (dims, acc) in ps.items():
            cands = [("bxy", "v")] if name == "upd" else list(itertools.permutations(dims))
            cost, order = min((pass_cost(dims, o, acc)[0], o) for o in cands)
            total += cost
            chosen[name] = order
        if best is None or total < best[0]:
            best = (total, QS, chosen)
    return best


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("order", type=int)
    ap.add_argument("width", type=int, choices=(4, 8), help="work-area bytes: 8 FP64, 4 FP32 residual")
    ap.add_argument("--search", action="store_true", help="also search strides and orders")
    args = ap.parse_args()
    cur = count(args.order, args.width)
    plain = count(args.order, args.width, QS=((args.order + 2) ** 3) | 1, orders=task_orders(0, args.width),
                  rotated=False)
    print(f"p = {args.order}, {args.width}-byte work area: wavefronts per element (committed / x-fastest, "
          f"odd strides, original orders / conflict-free)")
    for name in cur:
        print(f"  {name:7s} {cur[name][0]:6d} {plain[name][0]:6d} {cur[name][1]:6d}")
    print(f"  {'total':7s} {sum(c[0] for c in cur.values()):6d} {sum(c[0] for c in plain.values()):6d} "
          f"{sum(c[1] for c in cur.values()):6d}")
    mg = count(args.order, args.width, mg=True)
    print(f"  with the lifts added in the inverse mass's x pass (MG): minvxg {mg['minvxg'][0]} "
          f"(gather + minvx {cur['gather'][0] + cur['minvx'][0]}), total {sum(c[0] for c in mg.values())}")
    if args.search:
        total, QS, chosen = search(args.order, args.width)
        print(f"search: total {total} with QS = {QS}; orders {chosen}")


if __name__ == "__main__":
    main()
