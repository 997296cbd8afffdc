"""Tile plan of the one-pass normal operator (``tls_normal_tiles``).

The operator y = diag(s) J^T J diag(s) x + lambda x (torchls sparse.py:83-84,
warp_normal.py:125-294) reads each factor's Jacobian once. This module
decides, once per incidence structure, where every contribution goes:

* Factor group k is cut into tiles of ``tile_factors[k]`` consecutive factors
  (the stage of one CTA holds a whole tile's contributions: 72 KB), and the
  tiles are split into contiguous ranges, one per CTA (two CTAs per SM).
* Within a tile, the (slot, factor) pairs are ordered by (target column,
  factor, slot); ``pos`` holds each pair's offset (in doubles) in that order
  and the offset of its target's x values in the tile's compact x buffer
  (each target's x is loaded once per tile); each target's pairs form one
  run, summed in order by one thread.
* A run is *final* when it holds all of the target's contributions (the point
  of a bundle adjustment whose observations all sit in the tile); it goes to
  the CTA's shared *accumulator* when the target recurs in several of the
  CTA's tiles (cameras), up to ``acc_doubles``; otherwise it becomes a
  *partial*. At the end the CTA flushes each accumulator entry as final (all
  of the target's contributions were in the CTA) or as a partial.
* The gather kernel finishes every target that has partials (summed in
  creation order) and every variable no factor touches (y = lambda x).

All orders are fixed here, so the device results are bitwise reproducible.
The plan depends only on the index arrays and the SM count, never on values.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

STAGE_DOUBLES = 9216  # 72 KB contribution stage per CTA
ACC_DOUBLES = 2048    # 16 KB accumulator per CTA
MAX_TILE = 1024
CTAS_PER_SM = 2  # resident CTAs per SM for small factor shapes (r * D <= 18)
MAX_RUN = (1 << 13) - 1
MAX_STAGE = 1 << 14
HEAVY = 32  # partials from which a gather target gets a whole 256-thread block


@dataclass
class FactorGroupShape:
    """The incidence of one factor group: per slot, the first tangent column
    of the variable group, its dimension and the [N] variable indices."""

    count: int
    slots: list  # [(offset, dim, index ndarray)]
    rdim: int = 1


@dataclass
class TilePlan:
    tile_factors: list
    tile_base: list
    cta_base: list
    pos: list  # per group: uint32 [S_k * N_k] (stage offset | x-buffer offset << 16), tile order, or None
    perm: list  # per group: int64 [N_k] factor at each tile position, or None (caller's order)
    cta_tile: np.ndarray
    tile_run: np.ndarray
    run_col: np.ndarray
    run_meta: np.ndarray
    run_dest: np.ndarray
    run_xoff: np.ndarray
    cta_flush: np.ndarray
    flush_col: np.ndarray
    flush_meta: np.ndarray
    flush_dest: np.ndarray
    target_col: np.ndarray
    target_dim: np.ndarray
    target_ptr: np.ndarray
    target_src: np.ndarray
    npartials: int
    gather_lanes: int
    nheavy: int
    xbuf_doubles: int
    stage_doubles: int = STAGE_DOUBLES
    acc_doubles: int = ACC_DOUBLES
    stats: dict = field(default_factory=dict)

    @property
    def ncta(self) -> int:
        return len(self.cta_tile) - 1

    @property
    def ntiles(self) -> int:
        return len(self.tile_run) - 1


def _lanes(mean: float) -> int:
    lanes = 1
    while lanes < mean and lanes < 32:
        lanes *= 2
    return lanes


def tile_size(total_dim: int, stage_doubles: int = STAGE_DOUBLES) -> int:
    """Factors per tile for a group of total dimension D (0: does not fit)."""
    t = min(MAX_TILE, stage_doubles // max(total_dim, 1)) // 32 * 32
    return t if t >= 32 else 0


def _tile_sizes(groups, budget, stage_doubles, max_tile):
    """(factors per tile, tiles, CTAs, tiles per CTA) per group.

    Every CTA of a launch should carry the same number of tiles (a CTA with
    one tile more than the others sets the launch's time). The group with the
    most Jacobian bytes fixes the tiles per CTA from its CTA budget (two per SM
    for r * D <= 18, one above); the other groups get as many CTAs as they
    need to finish in the same number of tiles, and the largest group's budget
    shrinks by that many (the groups may share one launch).
    """
    info = []
    for g in groups:
        D = sum(d for _, d, _ in g.slots)
        tmax = min(tile_size(D, stage_doubles), max_tile)
        if g.count > 0 and (tmax == 0 or not g.slots):
            return None
        cap = budget if g.rdim * D <= 18 else max(1, budget // 2)
        info.append((g.count, max(tmax, 32), cap, g.count * g.rdim * D))

    def fit(count, tmax, ctas, per=None):
        if count == 0:
            return (tmax, 0, 0, 1)
        if per is None:
            per = -(-count // (ctas * tmax))
        T = max(1, min(tmax, -(-count // (ctas * per))))
        nt = -(-count // T)
        return (T, nt, -(-nt // per), per)

    live = [k for k, v in enumerate(info) if v[0] > 0]
    if not live:
        return [fit(0, v[1], 1) for v in info]
    main = max(live, key=lambda k: info[k][3])
    per = fit(info[main][0], info[main][1], info[main][2])[3]
    out = [None] * len(info)
    used = 0
    for k, (count, tmax, cap, _) in enumerate(info):
        if k != main:
            out[k] = fit(count, tmax, max(1, -(-count // (per * tmax))), per)
            used += out[k][2]
    count, tmax, cap, _ = info[main]
    out[main] = fit(count, tmax, max(1, cap - used))
    return out


def _tile_order(g: FactorGroupShape, group_count: dict) -> np.ndarray | None:
    """Factor order for the tiles of one group, or None to keep the caller's.

    Factors are ordered by the smaller (then the larger) index of their slots
    on the largest variable group (the points of a bundle adjustment, the
    poses of a pose graph), so that a tile's factors share targets: a pose
    graph's loop closures, added in random order, then land beside the
    odometry edges of the same poses. The order is stable; a group already in
    that order keeps its own (no copy of J is needed then).
    """
    if g.count == 0 or not g.slots:
        return None
    sizes = [group_count.get(off, 0) for off, _, _ in g.slots]
    big = max(sizes)
    keys = [np.asarray(idx, dtype=np.int64) for (_, _, idx), n in zip(g.slots, sizes) if n == big]
    lo, hi = np.minimum.reduce(keys), np.maximum.reduce(keys)
    if np.all(lo[1:] >= lo[:-1]):
        return None  # already ordered by the primary key: keep it
    return np.lexsort((np.arange(g.count), hi, lo)).astype(np.int64)


def build_tile_plan(groups: list[FactorGroupShape], var_groups: list[tuple[int, int, int]], num_sms: int, *,
                    ctas_per_sm: int = CTAS_PER_SM, stage_doubles: int = STAGE_DOUBLES,
                    acc_doubles: int = ACC_DOUBLES, max_tile: int = MAX_TILE,
                    reorder: bool = True) -> TilePlan | None:
    """Plan for factor groups over variable groups ``(offset, count, dim)``.

    Returns None when a shape does not fit the one-pass kernel (a variable
    dimension above 16, a tile that cannot hold 32 factors, more than 2^31
    columns); the operator then takes the two-pass route. With ``reorder``,
    a group whose factors are not ordered by their main variable gets a tile
    order (``perm[k]``: tile position -> factor); the kernels then read J
    from a copy with its columns in that order (``tls_permute_columns``).
    """
    for k, g in enumerate(groups):
        for s, (_, _, idx) in enumerate(g.slots):
            if len(idx) != g.count:
                raise ValueError(f"factor group {k}, slot {s}: index array of length {len(idx)} for {g.count} factors")
    n = sum(c * d for _, c, d in var_groups)
    if n >= 2**31 or stage_doubles > MAX_STAGE or acc_doubles > 65536:
        return None
    if any(d > 16 for _, _, d in var_groups):
        return None
    budget = max(1, num_sms * ctas_per_sm)
    sizes = _tile_sizes(groups, budget, stage_doubles, max_tile)
    if sizes is None:
        return None
    tile_factors, tile_base, cta_base = [], [], [0]
    cta_tile_parts, pair_parts, perm = [], [], []
    group_count = {off: c for off, c, _ in var_groups}
    ntiles = 0
    for k, g in enumerate(groups):
        T, nt, G, per = sizes[k]
        if g.count == 0:
            perm.append(None)
        tile_factors.append(T)
        tile_base.append(ntiles)
        if G:
            bounds = ntiles + np.minimum(np.arange(G, dtype=np.int64) * per, nt)
            cta_tile_parts.append(bounds)
        cta_base.append(cta_base[-1] + G)
        if g.count:
            f = np.arange(g.count, dtype=np.int64)
            order = _tile_order(g, group_count) if reorder else None
            perm.append(order)
            for s, (off, dim, idx) in enumerate(g.slots):
                idx = np.asarray(idx, dtype=np.int64)
                if order is not None:
                    idx = idx[order]
                pair_parts.append((ntiles + f // T, off + idx * dim, f % T, np.full(g.count, s, np.int64),
                                   np.full(g.count, dim, np.int64), np.full(g.count, k, np.int64), f))
        ntiles += nt
    ncta = cta_base[-1]
    cta_tile = np.concatenate(cta_tile_parts + [np.array([ntiles], np.int64)]).astype(np.int32)
    cta_of_tile = np.zeros(ntiles, np.int64)
    if ntiles:
        cta_of_tile = np.searchsorted(cta_tile[:-1], np.arange(ntiles), side="right") - 1

    if pair_parts:
        tile, col, lf, slot, dim, grp, fac = (np.concatenate(a) for a in zip(*pair_parts))
    else:
        tile = col = lf = slot = dim = grp = fac = np.zeros(0, np.int64)
    order = np.lexsort((slot, lf, col, tile))
    tile, col, slot, dim, grp, fac = (a[order] for a in (tile, col, slot, dim, grp, fac))
    # stage offsets: cumulative dims within the tile
    cum = np.cumsum(dim) - dim
    first_pair = np.searchsorted(tile, np.arange(ntiles), side="left")
    base = cum[first_pair[tile]] if len(tile) else cum
    pos_all = cum - base
    if len(pos_all) and int((pos_all + dim).max()) > stage_doubles:
        return None
    # runs: consecutive pairs of one (tile, col)
    if len(tile):
        new = np.ones(len(tile), bool)
        new[1:] = (tile[1:] != tile[:-1]) | (col[1:] != col[:-1])
        run_first = np.flatnonzero(new)
    else:
        new = np.zeros(0, bool)
        run_first = np.zeros(0, np.int64)
    run_tile = tile[run_first]
    run_col = col[run_first]
    run_dim = dim[run_first]
    run_start = pos_all[run_first]
    run_len = np.diff(np.append(run_first, len(tile)))
    if len(run_len) and int(run_len.max()) > MAX_RUN:
        return None
    # each run's x values sit once per tile in a compact buffer: offset = dims of the tile's earlier runs
    rcum = np.cumsum(run_dim) - run_dim
    tile_first_run = np.searchsorted(run_tile, np.arange(ntiles), side="left")
    run_xoff = rcum - (rcum[tile_first_run[run_tile]] if len(run_first) else rcum)
    xbuf_doubles = int((run_xoff + run_dim).max()) if len(run_first) else 0
    pair_run = np.cumsum(new) - 1
    pair_x = run_xoff[pair_run] if len(tile) else pos_all
    pos = []
    for k, g in enumerate(groups):
        if g.count == 0:
            pos.append(None)
            continue
        arr = np.zeros(len(g.slots) * g.count, np.uint32)
        m = grp == k
        arr[slot[m] * g.count + fac[m]] = pos_all[m] | (pair_x[m] << 16)
        pos.append(arr)
    nruns = len(run_first)
    tile_run = np.searchsorted(run_tile, np.arange(ntiles + 1), side="left").astype(np.int32)
    total = np.bincount(col, minlength=n) if len(col) else np.zeros(n, np.int64)

    run_cta = cta_of_tile[run_tile] if nruns else np.zeros(0, np.int64)
    key = run_cta * n + run_col
    ukey, inv, runs_in_cta = np.unique(key, return_inverse=True, return_counts=True)
    pairs_in_cta = np.bincount(inv, weights=run_len, minlength=len(ukey)).astype(np.int64)
    u_cta, u_col = ukey // max(n, 1), ukey % max(n, 1)
    u_dim = np.zeros(len(ukey), np.int64)
    u_dim[inv] = run_dim
    final_run = run_len == total[run_col]
    # accumulator entries: targets in >= 2 of the CTA's tiles, in column order, up to capacity
    cand = runs_in_cta >= 2
    cdim = np.where(cand, u_dim, 0)
    cta_first = np.searchsorted(u_cta, np.arange(ncta), side="left")
    csum = np.cumsum(cdim)
    before = np.concatenate(([0], csum))[cta_first[u_cta]] if len(ukey) else csum
    acc_end = csum - before
    assigned = cand & (acc_end <= acc_doubles)
    acc_off = acc_end - u_dim
    run_dest = np.full(nruns, -1, np.int64)
    run_acc = assigned[inv] & ~final_run
    run_dest[run_acc] = -2 - acc_off[inv][run_acc]
    run_partial = ~final_run & ~run_acc
    fl = np.flatnonzero(assigned)
    flush_final = pairs_in_cta[fl] == total[u_col[fl]]
    # partial slots in creation order: per CTA, its partial runs in order, then its partial flushes
    p_cta = np.concatenate((run_cta[run_partial], u_cta[fl][~flush_final]))
    p_kind = np.concatenate((np.zeros(int(run_partial.sum()), np.int64), np.ones(int((~flush_final).sum()), np.int64)))
    p_idx = np.concatenate((np.flatnonzero(run_partial), np.flatnonzero(~flush_final)))
    p_col = np.concatenate((run_col[run_partial], u_col[fl][~flush_final]))
    p_dim = np.concatenate((run_dim[run_partial], u_dim[fl][~flush_final]))
    porder = np.lexsort((p_idx, p_kind, p_cta))
    p_off = np.empty(len(porder), np.int64)
    p_off[porder] = np.cumsum(p_dim[porder]) - p_dim[porder]
    npartials = int(p_dim.sum())
    if npartials >= 2**31:
        return None
    nrp = int(run_partial.sum())
    run_dest[run_partial] = p_off[:nrp]
    flush_dest = np.full(len(fl), -1, np.int64)
    flush_dest[~flush_final] = p_off[nrp:]
    cta_flush = np.searchsorted(u_cta[fl], np.arange(ncta + 1), side="left").astype(np.int32)

    # gather targets: columns with partials (sources in creation order), then untouched variables
    seq = np.empty(len(porder), np.int64)
    seq[porder] = np.arange(len(porder))
    gorder = np.lexsort((seq, p_col))
    g_col, g_src, g_dim = p_col[gorder], p_off[gorder], p_dim[gorder]
    tcols, tfirst = np.unique(g_col, return_index=True)
    tdim = g_dim[tfirst]
    counts = np.diff(np.append(tfirst, len(g_col)))
    untouched_c, untouched_d = [], []
    for off, count, d in var_groups:
        cols = off + np.arange(count, dtype=np.int64) * d
        miss = cols[total[cols] == 0] if count else cols
        untouched_c.append(miss)
        untouched_d.append(np.full(len(miss), d, np.int64))
    ucols = np.concatenate(untouched_c) if untouched_c else np.zeros(0, np.int64)
    udims = np.concatenate(untouched_d) if untouched_d else np.zeros(0, np.int64)
    # heavy targets (at least HEAVY partials: the cameras) first, a block each;
    # the rest share `gather_lanes` lanes per target
    heavy = counts >= HEAVY
    horder = np.concatenate((np.flatnonzero(heavy), np.flatnonzero(~heavy)))
    starts = tfirst[horder]
    counts_o = counts[horder]
    new_ptr = np.concatenate(([0], np.cumsum(counts_o)))
    g_src = g_src[np.arange(new_ptr[-1]) - np.repeat(new_ptr[:-1], counts_o) + np.repeat(starts, counts_o)]
    target_col = np.concatenate((tcols[horder], ucols))
    target_dim = np.concatenate((tdim[horder], udims))
    target_ptr = np.concatenate(([0], np.cumsum(np.concatenate((counts_o, np.zeros(len(ucols), np.int64))))))
    nheavy = int(heavy.sum())
    light = counts[~heavy]
    mean = float(light.mean()) if len(light) else 1.0

    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    run_meta = run_start | (run_len << 14) | ((run_dim - 1) << 27)
    flush_meta = acc_off[fl] | ((u_dim[fl] - 1) << 16)
    stats = dict(ntiles=ntiles, ncta=ncta, nruns=nruns, final_runs=int(final_run.sum()),
                 acc_runs=int(run_acc.sum()), partial_runs=nrp, flushes=len(fl),
                 partial_doubles=npartials, targets=len(target_col))
    stage_need = max([T * sum(d for _, d, _ in g.slots) for T, g in zip(tile_factors, groups) if g.count] or [0])
    acc_need = int((acc_off[assigned] + u_dim[assigned]).max()) if assigned.any() else 0
    return TilePlan(tile_factors=tile_factors, tile_base=tile_base, cta_base=cta_base, pos=pos, perm=perm,
                    cta_tile=cta_tile, tile_run=tile_run, run_col=i32(run_col), run_meta=i32(run_meta),
                    run_dest=i32(run_dest), run_xoff=i32(run_xoff), xbuf_doubles=xbuf_doubles, cta_flush=cta_flush,
                    flush_col=i32(u_col[fl]),                    flush_meta=i32(flush_meta), flush_dest=i32(flush_dest), target_col=i32(target_col),
                    target_dim=i32(target_dim), target_ptr=i32(target_ptr), target_src=i32(g_src),
                    npartials=npartials, gather_lanes=_lanes(mean), nheavy=nheavy, stage_doubles=max(stage_need, 1),
                    acc_doubles=max(acc_need, 1), stats=stats)
