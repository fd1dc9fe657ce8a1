"""Oracle of Circuitscape's pairwise mode on rasters -- TEST INFRASTRUCTURE ONLY.

Only the tests (and the bench's CPU leg) import this module, as the checker of the GPU path; nothing in the
product calls it.  A plain-loop restatement of the reference's native code, solving each component's grounded
Laplacian directly (scipy's sparse LU) where the reference uses its own multifrontal Cholesky:

- ``raster_graph``: ``src/cpp/circuit/circuitscape.cpp:145-263`` (node map with short-circuit regions, edges in
  column-major order, duplicates summed in the order met, the Laplacian's diagonal, connected components);
- ``node_currents``: ``graph_node_currents``, ``circuitscape.cpp:38-77``;
- ``pairwise``: ``raster_pairwise``, ``circuitscape.cpp:474-743`` (jobs, grounding at the component's last node,
  per-pair maps, the shortcut of ``update_voltmatrix!`` / ``update_shortcut_resistances!``);
- ``region_polymap`` / ``pairwise_regions``: ``circuitscape.cpp:749-866`` (a graph per pair of focal regions);
- ``node_sums`` / ``resolve`` / ``advanced_many`` / ``multi_advanced``: ``node_sums``, ``resolve`` and
  ``raster_advanced_many`` (``circuitscape.cpp:382-391,881-1083``) and the native ``circuitscape_multi_advanced``
  (``src/cpp/circuit/python.cpp:404-480``): advanced-mode problems with direct and finite grounds, solved per
  component and problem (the reference's Schur-complement shortcut is exact, so a plain solve stands for it);
- ``pairwise_ini``: the pairwise branch of ``circuitscape_ini``, ``src/landschaft/circuit/circuitscape.py:1039-1170``.

The file parsers (ASCII grids, point lists, pair files) are the package's own; the reference's golden outputs of
Circuitscape's pairwise INI cases (``tests/data/reference/circuit/circuitscape.npz``, copied under
``tests/golden/circuitscape``) pin this oracle.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np

NODATA = -9999.0
K_SHIFT = 10 * np.finfo(np.float64).eps
SQRT2 = 1.4142135623730951


def _average(x, y, diagonal, resistances):
    # raster/graph.jl's averages (circuitscape.cpp:31-34); 1/0 is +inf as in C++
    if resistances:
        ix = math.inf if x == 0 else 1 / x
        iy = math.inf if y == 0 else 1 / y
        s = (ix + iy) / 2
        if diagonal:
            return 0.0 if math.isinf(s) else 1 / (SQRT2 * s)
        return 0.0 if math.isinf(s) else 1 / s
    return (x + y) / (2 * SQRT2) if diagonal else (x + y) / 2


def raster_graph(gmap, polymap, avg_resistances, four_neighbors):
    ny, nx = gmap.shape
    g = gmap.ravel()
    n = nx * ny
    label = [0] * n
    nxt = 0
    for x in range(nx):
        for y in range(ny):
            if g[y * nx + x] > 0:
                nxt += 1
                label[y * nx + x] = nxt
    if polymap is not None:
        pm = polymap.ravel()
        first = {}
        for x in range(nx):
            for y in range(ny):
                c = y * nx + x
                if pm[c] != 0 and g[c] > 0 and int(pm[c]) not in first:
                    first[int(pm[c])] = label[c]
        for c in range(n):
            if pm[c] != 0 and int(pm[c]) in first:
                label[c] = first[int(pm[c])]
    labels = sorted(set(v for v in label if v != 0))
    rank = {v: k for k, v in enumerate(labels)}
    nodemap = [-1] * n
    for c in range(n):
        if label[c] != 0:
            nodemap[c] = rank[label[c]]
    n_nodes = len(labels)
    edges = []

    def emit(c, d, diagonal):
        a, b = nodemap[c], nodemap[d]
        if a < 0 or b < 0:
            return
        w = _average(g[c], g[d], diagonal, avg_resistances)
        if a == b:
            return
        edges.append((a, b, w))
        edges.append((b, a, w))

    for x in range(nx):
        for y in range(ny):
            c = y * nx + x
            if nodemap[c] < 0:
                continue
            if x + 1 < nx:
                emit(c, c + 1, False)
            if y + 1 < ny:
                emit(c, c + nx, False)
            if not four_neighbors:
                if y + 1 < ny and x + 1 < nx:
                    emit(c, c + nx + 1, True)
                if y > 0 and x + 1 < nx:
                    emit(c, c - nx + 1, True)
    edges.sort(key=lambda e: (e[0], e[1]))  # stable: duplicates in the order met
    rows = [[] for _ in range(n_nodes)]
    k = 0
    while k < len(edges):
        e = k
        w = None
        while e < len(edges) and edges[e][0] == edges[k][0] and edges[e][1] == edges[k][1]:
            w = edges[e][2] if w is None else w + edges[e][2]
            e += 1
        rows[edges[k][0]].append((edges[k][1], w))
        k = e
    degree = []
    for r in rows:
        d = 0.0
        for _, w in r:
            d += w
        degree.append(d)
    comp = [-1] * n_nodes
    n_comp = 0
    for u in range(n_nodes):
        if comp[u] >= 0:
            continue
        comp[u] = n_comp
        stack = [u]
        while stack:
            v = stack.pop()
            for t, w in rows[v]:
                if w == 0 or comp[t] >= 0:
                    continue
                comp[t] = n_comp
                stack.append(t)
        n_comp += 1
    return {"nx": nx, "ny": ny, "n_nodes": n_nodes, "nodemap": np.array(nodemap, dtype=np.int64), "rows": rows,
            "degree": np.array(degree), "comp": np.array(comp, dtype=np.int64), "n_comp": n_comp}


def node_currents(G, members, v, finite=None):
    """graph_node_currents over the nodes `members` (ascending) with voltages v by node (finite grounds by node
    or None)."""
    with np.errstate(divide="ignore", invalid="ignore"):  # b / 0 is +-inf, as in C++
        return _node_currents(G, members, v, finite)


def _node_currents(G, members, v, finite):
    rows = G["rows"]
    maxin = maxout = -math.inf
    for c in members:
        for r, w in rows[c]:
            b = abs(w) * (v[r] - v[c])
            if r < c:
                if b > maxin:
                    maxin = b
            elif b > maxout:
                maxout = b
    cur = {}
    for c in members:
        inflow = outflow = 0.0
        for r, w in rows[c]:
            b = abs(w) * (v[r] - v[c])
            if b > 0:
                if not (abs(b / maxin) < 1e-8):
                    inflow += b
            elif b < 0:
                if not (abs(b / maxout) < 1e-8):
                    outflow -= b
        if finite is not None:
            f = finite[c] * v[c]
            if f < 0:
                inflow -= f
            elif f > 0:
                outflow += f
        cur[c] = inflow if inflow > outflow else outflow
    return cur


def _component_solver(G, members, ref):
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import splu
    unk = [v for v in members if v != ref]
    loc = {v: k for k, v in enumerate(unk)}
    ri, ci, vals = [], [], []
    for v in unk:
        i = loc[v]
        ri.append(i)
        ci.append(i)
        vals.append(G["degree"][v] + K_SHIFT)
        for t, w in G["rows"][v]:
            if t in loc:
                ri.append(i)
                ci.append(loc[t])
                vals.append(-w)
    m = len(unk)
    if m == 0:
        return loc, None
    lu = splu(csc_matrix((vals, (ri, ci)), shape=(m, m)))
    return loc, lu


def node_sums(G, cells, vals):
    nx = G["nx"]
    order = sorted(range(len(cells)), key=lambda k: (cells[k] % nx, cells[k] // nx))
    s = [0.0] * G["n_nodes"]
    for k in order:
        v = G["nodemap"][cells[k]]
        if v >= 0 and vals[k] != 0:
            s[v] += vals[k]
    return s


def resolve(src, gnd, policy):
    n = len(src)
    src, gnd = list(src), list(gnd)
    finite = [gnd[v] if gnd[v] < math.inf else 0.0 for v in range(n)]
    for v in range(n):
        if not (src[v] != 0 and gnd[v] != 0):
            continue
        if policy in ("rmvsrc", "rmvall"):
            src[v] = 0.0
        elif policy == "rmvgnd":
            gnd[v] = 0.0
    for v in range(n):
        if gnd[v] == math.inf and src[v] > 0:
            gnd[v] = 0.0
    return src, gnd, finite


def advanced_many(G, srcs, gnds, only_nodes, policy):
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import splu
    n = G["n_nodes"]
    comp = G["comp"]
    out = []
    res = [resolve(s, g, policy) for s, g in zip(srcs, gnds)]
    for s, g, _ in res:
        out.append({"voltage": np.zeros(n), "current": np.zeros(n), "solved": False,
                    "active": np.array([v for v in range(n) if s[v] != 0 or g[v] != 0], dtype=np.int32)})
    for k in range(G["n_comp"]):
        members = [v for v in range(n) if comp[v] == k]
        for p, (s, g, fin) in enumerate(res):
            only = only_nodes[p]
            if only == -2 or (only >= 0 and comp[only] != k):
                continue
            ss = tt = 0.0
            for v in members:
                ss += s[v]
                tt += g[v]
            if not (ss != 0 and tt != 0):
                continue
            out[p]["solved"] = True
            unk = [v for v in members if g[v] != math.inf]
            loc = {v: i for i, v in enumerate(unk)}
            ri, ci, vals = [], [], []
            for v in unk:
                i = loc[v]
                ri.append(i)
                ci.append(i)
                vals.append((G["degree"][v] + fin[v]) + K_SHIFT)
                for t_, w in G["rows"][v]:
                    if t_ in loc:
                        ri.append(i)
                        ci.append(loc[t_])
                        vals.append(-w)
            volt = out[p]["voltage"]
            if unk:
                lu = splu(csc_matrix((vals, (ri, ci)), shape=(len(unk), len(unk))))
                x = lu.solve(np.array([s[v] for v in unk]))
                for v in unk:
                    volt[v] = x[loc[v]]
            cn = node_currents(G, members, volt, fin)
            for v in members:
                out[p]["current"][v] = cn[v]
    return out


def multi_advanced(g, poly, avg, four, problems, policy):
    """circuitscape_multi_advanced: (nodemap as a grid, one result dict per problem)."""
    G = raster_graph(g, poly, avg, four)
    srcs, gnds, only = [], [], []
    for q in problems:
        srcs.append(node_sums(G, [int(c) for c in q["src_cells"]], [float(v) for v in q["src_vals"]]))
        gnds.append(node_sums(G, [int(c) for c in q["gnd_cells"]], [float(v) for v in q["gnd_vals"]]))
        o = -1
        if q["check_cell"] >= 0:
            o = int(G["nodemap"][q["check_cell"]])
            if o < 0:
                o = -2
        only.append(o)
    return G["nodemap"].reshape(g.shape), advanced_many(G, srcs, gnds, only, policy)


def pairwise(G, gmap, points, excluded, opts, emit=None):
    """raster_pairwise: resistances (n x n), cum, max (flat, or None)."""
    npt = len(points)
    ncell = G["nx"] * G["ny"]
    g = gmap.ravel()
    R = np.full((npt, npt), -1.0)
    maps = opts.get("volt_maps") or opts.get("cur_maps") or opts.get("cum") or opts.get("max")
    shortcut = not maps and not np.any(excluded)
    voltmatrix = np.zeros((npt, npt))
    S = np.full((npt, npt), -1.0)
    cum = np.zeros(ncell) if opts.get("cum") else None
    mx = np.full(ncell, NODATA) if opts.get("max") else None
    comp = G["comp"]
    positions = {}
    for i, v in enumerate(points):
        if v >= 0:
            positions.setdefault(int(v), []).append(i)
    for k in range(G["n_comp"]):
        members = [v for v in range(G["n_nodes"]) if comp[v] == k]
        csub = []
        for i in range(npt):
            v = int(points[i])
            if v >= 0 and comp[v] == k and v not in csub:
                csub.append(v)
        if not csub:
            continue
        for v in csub:
            pos = positions[v]
            for a in range(len(pos)):
                for b in range(a + 1, len(pos)):
                    R[pos[a], pos[b]] = R[pos[b], pos[a]] = 0.0
        nsrc = min(1, len(csub)) if shortcut else len(csub)
        jobs = [(csub[si], csub[di]) for si in range(nsrc) for di in range(si + 1, len(csub))
                if any(not excluded[ci, cj] for ci in positions[csub[si]] for cj in positions[csub[di]])]
        if not jobs:
            continue
        ref = members[-1]
        loc, lu = _component_solver(G, members, ref)
        for s, d in jobs:
            b = np.zeros(len(loc))
            if s in loc:
                b[loc[s]] = -1.0
            if d in loc:
                b[loc[d]] = 1.0
            x = lu.solve(b) if lu is not None else b
            v = {u: (x[loc[u]] if u in loc else 0.0) for u in members}
            vs = v[s]
            v = {u: v[u] - vs for u in members}
            resistance = v[d] - v[s]
            vmap = cmap = None
            if maps:
                vnode = np.zeros(G["n_nodes"])
                for u in members:
                    vnode[u] = v[u]
                cn = node_currents(G, members, vnode)
                if opts.get("volt_maps"):
                    vmap = np.zeros(ncell)
                    for c in range(ncell):
                        u = G["nodemap"][c]
                        if u >= 0 and comp[u] == k:
                            vmap[c] = vnode[u]
                        if opts.get("null_voltages") and g[c] == 0:
                            vmap[c] = NODATA
                cmap = np.zeros(ncell)
                for c in range(ncell):
                    u = G["nodemap"][c]
                    if u >= 0 and comp[u] == k:
                        cmap[c] = cn[u]
                        if opts.get("focal_zero") and (u == s or u == d):
                            cmap[c] = 0.0
                    if opts.get("log_transform"):
                        cmap[c] = math.log10(cmap[c]) if cmap[c] > 0 else NODATA
                    if opts.get("null_currents") and g[c] == 0:
                        cmap[c] = NODATA
            for ci in positions[s]:
                for cj in positions[d]:
                    if excluded[ci, cj]:
                        continue
                    R[ci, cj] = R[cj, ci] = resistance
                    if shortcut:
                        for i in range(1, npt):
                            u = int(points[i])
                            if u < 0 or comp[u] != k:
                                continue
                            voltmatrix[i, cj] = 1 - v[u] / resistance
                        continue
                    if not maps:
                        continue
                    if cum is not None:
                        cum += cmap
                    if mx is not None:
                        mx = np.maximum(mx, cmap)
                    if emit is not None and (opts.get("volt_maps") or opts.get("cur_maps")):
                        emit(ci, cj, vmap, cmap.copy() if opts.get("cur_maps") else None)
        if shortcut:
            anchor = positions[csub[0]][0]
            check = [points[i] >= 0 and comp[points[i]] == k for i in range(npt)]
            for x in range(npt):
                if not check[x]:
                    continue
                r1x = R[anchor, x]
                if r1x == -1:
                    continue
                S[x, anchor] = S[anchor, x] = r1x
                for y in range(x, npt):
                    if not check[y]:
                        continue
                    r12 = R[anchor, y]
                    if r12 == -1:
                        continue
                    if r1x != -777:
                        S[anchor, y] = S[y, anchor] = r12
                        r2x = 2 * r12 * voltmatrix[x, y] + r1x - r12
                        if S[y, x] != -777:
                            S[y, x] = S[x, y] = r2x
                    else:
                        S[x, :] = -777
                        S[:, x] = -777
    if shortcut:
        R = S
    np.fill_diagonal(R, 0.0)
    if cum is not None:
        cum = np.maximum(cum, NODATA)
    if mx is not None:
        mx = np.maximum(mx, NODATA)
    return R, cum, mx


def region_polymap(polymap, n, cells, ids, pt1, pt2):
    if polymap is None:
        poly = [0] * n
        for x in range(len(ids)):
            if ids[x] == pt1:
                poly[cells[x]] = pt1
        for x in range(len(ids)):
            if ids[x] == pt2:
                poly[cells[x]] = pt2
        return np.array(poly, dtype=np.int64)
    poly = [int(v) for v in polymap.ravel()]
    k = max(poly)
    for pt in (pt1, pt2):
        idx = [cells[x] for x in range(len(ids)) if ids[x] == pt]
        if len(idx) == 1:
            continue
        k += 1
        vals = sorted(set(poly[c] for c in idx if poly[c] != 0))
        if vals:
            poly = [k if v in vals else v for v in poly]
        for c in idx:
            poly[c] = k
    return np.array(poly, dtype=np.int64)


def pairwise_regions(gmap, polymap, avg, four, cells, ids, excluded, opts, emit=None):
    """raster_pairwise_regions: ids sorted; `excluded` over the distinct ids."""
    pts = sorted(set(int(v) for v in ids))
    npt = len(pts)
    ny, nx = gmap.shape
    ncell = nx * ny
    R = np.full((npt, npt), -1.0)
    cum = np.zeros(ncell) if opts.get("cum") else None
    mx = np.full(ncell, NODATA) if opts.get("max") else None
    for i in range(npt):
        for j in range(i + 1, npt):
            if excluded[i, j] or excluded[j, i]:
                continue
            poly = region_polymap(polymap, ncell, cells, ids, pts[i], pts[j]).reshape(gmap.shape)
            G = raster_graph(gmap, poly, avg, four)
            nodes = []
            for pt in (pts[i], pts[j]):
                x = next(x for x in range(len(ids)) if ids[x] == pt)
                nodes.append(int(G["nodemap"][cells[x]]))
            got = []
            r2, c2, m2 = pairwise(G, gmap, np.array(nodes), np.zeros((2, 2), dtype=bool), opts,
                                  lambda ci, cj, v, c: got.append((ci, cj, v, c)))
            R[i, j] = R[j, i] = r2[0, 1]
            if cum is not None:
                cum += c2
            if mx is not None:
                mx = np.maximum(mx, m2)
            for ci, cj, v, c in got:
                if emit is not None:
                    emit(i if ci == 0 else j, i if cj == 0 else j, v, c)
    np.fill_diagonal(R, 0.0)
    if cum is not None:
        cum = np.maximum(cum, NODATA)
    return np.array(pts), R, cum, mx


def pairwise_ini(path):
    """The pairwise scenario of an INI file: (resistance matrix with ids, cum map, max map, maps by name)."""
    from landschaft_b200 import circuitscape as cs
    path = Path(path)
    base = path.resolve().parent
    cfg = {**cs.DEFAULTS, **cs.parse_config(path)}
    need = lambda key: cs._resolve(cfg[key], base)  # noqa: E731
    cells, meta = cs.read_raster(need("habitat_file"))
    reclass = cs.read_reclass_table(need("reclass_file")) if cs._flag(cfg, "use_reclass_table") else None
    g = cs.habitat_conductance(cells, is_resistance=cs._flag(cfg, "habitat_map_is_resistances"), reclass=reclass)
    poly = None
    if cs._flag(cfg, "use_polygons"):
        poly = cs.read_polymap(need("polygon_file"), meta, integer=True).astype(np.int64)
    if cs._flag(cfg, "use_mask"):
        m = cs.read_polymap(need("mask_file"), meta)
        g = g * np.where(m > 0, 1.0, 0.0)
    points = cs.read_point_map(need("point_file"), meta)
    pairs = cs.read_included_pairs(need("included_pairs_file")) if cs._flag(cfg, "use_included_pairs") else None
    points, excluded_ids = cs._apply_included_pairs(points, pairs)
    cur, cum_only = cs._flag(cfg, "write_cur_maps"), cs._flag(cfg, "write_cum_cur_map_only")
    opts = {"volt_maps": cs._flag(cfg, "write_volt_maps"), "cur_maps": cur and not cum_only, "cum": cur or cum_only,
            "max": cs._flag(cfg, "write_max_cur_maps"), "focal_zero": cs._flag(cfg, "set_focal_node_currents_to_zero"),
            "null_currents": cs._flag(cfg, "set_null_currents_to_nodata"),
            "null_voltages": cs._flag(cfg, "set_null_voltages_to_nodata"),
            "log_transform": cs._flag(cfg, "log_transform_maps")}
    avg, four = cs._flag(cfg, "connect_using_avg_resistances"), cs._flag(cfg, "connect_four_neighbors_only")
    rows, cols = points.cells
    maps = {}
    if points.has_regions:
        cells = [int(r * g.shape[1] + c) for r, c in zip(rows, cols)]
        pts = sorted(set(int(v) for v in points.ids))
        n = len(pts)
        ex = np.array([[(pts[a], pts[b]) in excluded_ids for b in range(n)] for a in range(n)], dtype=bool)

        def emit_r(ci, cj, vmap, cmap):
            name = f"_{pts[ci]}_{pts[cj]}"
            if vmap is not None:
                maps["voltmap" + name] = vmap.reshape(g.shape)
            if cmap is not None:
                maps["curmap" + name] = cmap.reshape(g.shape)

        ids_r, R, cum, mx = pairwise_regions(g, poly, avg, four, cells, [int(v) for v in points.ids], ex, opts,
                                             emit_r)
        res = np.zeros((n + 1, n + 1))
        res[0, 1:] = ids_r
        res[1:, 0] = ids_r
        res[1:, 1:] = R
        return (res, None if cum is None else cum.reshape(g.shape), None if mx is None else mx.reshape(g.shape),
                maps)
    G = raster_graph(g, poly, avg, four)
    nodes = np.array([G["nodemap"][r * g.shape[1] + c] for r, c in zip(rows, cols)], dtype=np.int64)
    ids = points.ids
    n = len(ids)
    ex = np.array([[(int(ids[a]), int(ids[b])) in excluded_ids for b in range(n)] for a in range(n)], dtype=bool)

    def emit(ci, cj, vmap, cmap):
        name = f"_{int(ids[ci])}_{int(ids[cj])}"
        if vmap is not None:
            maps["voltmap" + name] = vmap.reshape(g.shape)
        if cmap is not None:
            maps["curmap" + name] = cmap.reshape(g.shape)

    R, cum, mx = pairwise(G, g, nodes, ex, opts, emit)
    res = np.zeros((n + 1, n + 1))
    res[0, 1:] = ids
    res[1:, 0] = ids
    res[1:, 1:] = R
    return (res, None if cum is None else cum.reshape(g.shape), None if mx is None else mx.reshape(g.shape), maps)
