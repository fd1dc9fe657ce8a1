"""Circuitscape's pairwise mode on rasters (``ls.circuit.circuitscape_pairwise``) with its solves on the GPU.

Mirrors ``src/landschaft/circuit/circuitscape.py`` (the readers :30-330, ``circuitscape_pairwise`` :550-670 and the
pairwise branch of ``circuitscape_ini`` :1039-1213) and the native ``circuit::raster_graph`` /
``circuit::raster_pairwise`` (``src/cpp/circuit/circuitscape.cpp:145-263,474-743``).  The node graph is built on
the host with numpy, as the reference builds it on the host in C++; the solves and the node currents run on the GPU
through ``lsb_graph_pairs`` of the C ABI: one CTA per pair solves the component's grounded Laplacian (CSR) by FP64
Jacobi-preconditioned CG and computes the pair's node currents; the reference factorises each component once
(CHOLMOD-like multifrontal Cholesky) and back-substitutes every pair.

Scope: focal points and focal regions (several cells sharing an id: a graph per pair, the reference's
``raster_pairwise_regions``), raster or text-list point files, short-circuit polygons, masks, include/exclude pair
files, reclass tables, and every pairwise map option.  GeoTIFF inputs and the other scenarios (advanced with
polygons, one-to-all, all-to-one, networks) raise ``NotImplementedError``.
"""

from __future__ import annotations

import ctypes as C
import gzip
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _native as N

NODATA = -9999.0
TRUELIST = ("True", "true", "1")
FALSELIST = ("False", "false", "0")
K_SHIFT = 10 * np.finfo(np.float64).eps  # added to the Laplacian's diagonal, as the reference's factorisation does
SQRT2 = 1.4142135623730951
TWO_SQRT2 = 2 * SQRT2


# --- readers (circuitscape.py:30-330) -----------------------------------------------------------------------------

@dataclass
class RasterMeta:
    nrows: int
    ncols: int
    xllcorner: float
    yllcorner: float
    cellsize: float


def _open(path):
    p = os.fspath(path)
    return gzip.open(p, "rt") if p.lower().endswith("gz") else open(p, encoding="utf-8")


def file_type(path) -> str:
    """``geotiff``, ``npy``, ``aagrid``, ``pairs_aagrid``, ``pairs`` or ``list`` (circuitscape.py:48-70)."""
    p = os.fspath(path)
    with (gzip.open if p.lower().endswith("gz") else open)(p, "rb") as f:
        head = f.read(4)
    if head[2:4] == b"\x2a\x00":
        return "geotiff"
    with _open(p) as f:
        line = f.readline()
    if line.startswith("\x93NUMPY"):
        return "npy"
    if line.lower().startswith("ncols"):
        return "aagrid"
    if line.startswith("min"):
        return "pairs_aagrid"
    if line.startswith("mode"):
        return "pairs"
    return "list"


_ASC_KEYS = ("ncols", "nrows", "xllcorner", "yllcorner", "xllcenter", "yllcenter", "cellsize", "dx", "dy",
             "nodata_value")


def read_raster(path):
    """An ESRI ASCII grid (optionally gzipped) parsed in double, NoData and NaN set to -9999
    (circuitscape.py:73-124).  Returns ``(values, RasterMeta)``."""
    p = os.fspath(path)
    if not os.path.isfile(p):
        raise FileNotFoundError(f'the file "{p}" does not exist')
    if file_type(p) == "geotiff":
        return _read_tiff(p)
    if not p.lower().removesuffix(".gz").endswith(".asc"):
        raise NotImplementedError(f"{p}: only ESRI ASCII grids and uncompressed GeoTIFFs are read")
    header: dict[str, float] = {}
    rows = []
    with _open(p) as f:
        for line in f:
            toks = line.split()
            if not toks:
                continue
            if not rows and len(toks) == 2 and toks[0].lower() in _ASC_KEYS:
                header[toks[0].lower()] = float(toks[1])
                continue
            rows.append([float(t) for t in toks])
    nrows, ncols = int(header["nrows"]), int(header["ncols"])
    a = np.array(rows, dtype=np.float64)
    if a.shape != (nrows, ncols):
        raise ValueError(f"{p}: the ASCII grid does not hold {nrows} rows of {ncols} values")
    dx = header.get("dx", header.get("cellsize", math.nan))
    dy = header.get("dy", dx)
    xll = header["xllcorner"] if "xllcorner" in header else header["xllcenter"] - dx / 2
    yll = header["yllcorner"] if "yllcorner" in header else header["yllcenter"] - dy / 2
    nodata = header.get("nodata_value", NODATA)
    a[(a == nodata) | np.isnan(a)] = NODATA
    return a, RasterMeta(nrows, ncols, xll, yll, dx)


_TIFF_SIZES = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 10: 8, 11: 4, 12: 8, 16: 8}


def _read_tiff(path):
    """A single-band, uncompressed, strip-organised GeoTIFF (the baseline layout GDAL writes by default): values as
    double with GDAL's nodata value (tag 42113) and NaN set to -9999; the grid from the pixel-scale and tiepoint
    tags.  Other layouts raise NotImplementedError."""
    import struct
    with (gzip.open if os.fspath(path).lower().endswith("gz") else open)(path, "rb") as f:
        b = f.read()
    end = {b"II": "<", b"MM": ">"}.get(b[:2])
    if end is None or struct.unpack_from(end + "H", b, 2)[0] != 42:
        raise NotImplementedError(f"{path}: not a classic TIFF")
    off = struct.unpack_from(end + "I", b, 4)[0]
    tags = {}
    for k in range(struct.unpack_from(end + "H", b, off)[0]):
        tag, typ, cnt, _ = struct.unpack_from(end + "HHII", b, off + 2 + 12 * k)
        size = _TIFF_SIZES.get(typ, 1) * cnt
        pos = off + 2 + 12 * k + 8 if size <= 4 else struct.unpack_from(end + "I", b, off + 2 + 12 * k + 8)[0]
        raw = b[pos:pos + size]
        fmt = {3: "H", 4: "I", 8: "h", 9: "i", 11: "f", 12: "d", 16: "Q"}.get(typ)
        tags[tag] = raw.rstrip(b"\0").decode() if typ == 2 else (struct.unpack(f"{end}{cnt}{fmt}", raw) if fmt
                                                                else raw)
    ncols, nrows = tags[256][0], tags[257][0]
    bits = tags.get(258, (1,))[0]
    fmt_code = tags.get(339, (1,))[0]
    if tags.get(259, (1,))[0] != 1 or tags.get(277, (1,))[0] != 1 or 322 in tags or 273 not in tags:
        raise NotImplementedError(f"{path}: only single-band, uncompressed, strip-organised TIFFs are read")
    kind = {1: "u", 2: "i", 3: "f"}[fmt_code]
    dtype = np.dtype(f"{end}{kind}{bits // 8}")
    data = b"".join(b[o:o + c] for o, c in zip(tags[273], tags[279]))
    a = np.frombuffer(data, dtype=dtype, count=nrows * ncols).reshape(nrows, ncols).astype(np.float64)
    if 42113 in tags and tags[42113]:
        nodata = float(tags[42113])
        if kind != "f":
            nodata = float(np.array(nodata).astype(np.int64))
        a[a == nodata] = NODATA
    a[np.isnan(a)] = NODATA
    sx, sy = (tags[33550][0], tags[33550][1]) if 33550 in tags else (1.0, 1.0)
    ti, tj, _, tx, ty, _ = tags[33922] if 33922 in tags else (0.0, 0.0, 0.0, 0.0, float(nrows), 0.0)
    xll = tx - ti * sx
    yll = ty + tj * sy - nrows * sy
    return a, RasterMeta(nrows, ncols, xll, yll, sx)


def _read_rows(path) -> list:
    with _open(path) as f:
        return [[float(t) for t in line.split()] for line in f if line.split()]


def _list_cells(points: np.ndarray, meta: RasterMeta):
    # 1-based row and column: ceil(nrows - (y - yll) / cellsize), ceil((x - xll) / cellsize)
    i = np.ceil(meta.nrows - (points[:, 2] - meta.yllcorner) / meta.cellsize).astype(np.int64)
    j = np.ceil((points[:, 1] - meta.xllcorner) / meta.cellsize).astype(np.int64)
    return i, j


def read_polymap(path, habitat: RasterMeta, *, integer: bool = False, nodata_as=0.0) -> np.ndarray:
    """A raster on the habitat's grid with NoData set to ``nodata_as`` (circuitscape.py:151-160)."""
    a, meta = read_raster(path)
    if integer and not np.all(a == np.round(a)):
        raise ValueError(f"{path} contains non-integer values")
    if nodata_as is not None:
        a[a == NODATA] = nodata_as
    if (meta.nrows, meta.ncols) != (habitat.nrows, habitat.ncols):
        raise ValueError(f"{path} is not on the habitat's grid")
    return a


@dataclass
class FocalPoints:
    """Focal points: 1-based rows, columns and ids, sorted by id; cells sharing an id form a focal region."""

    rows: np.ndarray
    cols: np.ndarray
    ids: np.ndarray

    @property
    def cells(self):
        return np.asarray(self.rows) - 1, np.asarray(self.cols) - 1

    @property
    def has_regions(self) -> bool:
        return len(self.ids) != len(np.unique(self.ids))


def _sorted_points(i, j, v) -> FocalPoints:
    keep = v >= 0
    i, j, v = i[keep], j[keep], v[keep]
    order = np.argsort(v, kind="stable")
    return FocalPoints(i[order].astype(np.int64), j[order].astype(np.int64), v[order].astype(np.int64))


def read_point_map(path, habitat: RasterMeta) -> FocalPoints:
    """A raster of ids or a text list of ``id x y``; negative ids dropped, sorted by id (circuitscape.py:209-229)."""
    if file_type(path) == "list":
        pts = np.array(_read_rows(path), dtype=np.float64).reshape(-1, 3)
        i, j = _list_cells(pts, habitat)
        fp = _sorted_points(i, j, pts[:, 0])
    else:
        a = read_polymap(path, habitat, integer=True)
        jj, ii = np.nonzero(a.T)  # column-major order
        fp = _sorted_points(ii + 1, jj + 1, a[ii, jj])
    i, j, v = fp.rows, fp.cols, fp.ids
    if len(v) and (i.min() < 0 or j.min() < 0 or i.max() > habitat.nrows or j.max() > habitat.ncols):
        raise ValueError("At least one focal node location falls outside of habitat map")
    if len(np.unique(v)) < 2:
        raise ValueError("Less than two valid focal nodes found. Please check focal node location file.")
    return fp


@dataclass
class IncludedPairs:
    """Include / exclude pairs: ``mode`` ("include" or "exclude"), the ids and a 0/1 matrix over them."""

    mode: str
    ids: np.ndarray
    matrix: np.ndarray

    def excluded(self) -> set:
        target = 0 if self.mode == "include" else 1
        m, n = self.matrix, len(self.ids)
        return {(int(self.ids[i]), int(self.ids[j])) for j in range(n) for i in range(n)
                if m[i, j] == target and m[j, i] == target}


def read_included_pairs(path) -> IncludedPairs:
    """A ``min``/``max`` matrix or a ``mode`` list of pairs (circuitscape.py:283-311)."""
    kind = file_type(path)
    with _open(path) as f:
        lines = f.read().splitlines()
    if kind == "pairs_aagrid":
        minval, maxval = float(lines[0].split()[1]), float(lines[1].split()[1])
        a = np.array([[float(t) for t in ln.split()] for ln in lines[2:] if ln.split()])
        ids = a[0, 1:].astype(np.int64)
        m = a[1:, 1:]
        m = np.where(m > maxval, 0, m)
        return IncludedPairs("include", ids, (m >= minval).astype(np.int64))
    if kind == "pairs":
        mode = lines[0].split()[1]
        pairs = np.array([[float(t) for t in ln.split()] for ln in lines[1:] if ln.split()]).reshape(-1, 2)
        ids = np.unique(pairs).astype(np.int64)
        ids = ids[ids != 0]
        pos = {int(v): k for k, v in enumerate(ids)}
        m = np.zeros((len(ids), len(ids)), dtype=np.int64)
        for a, b in pairs.astype(np.int64):
            if a in pos and b in pos:
                m[pos[a], pos[b]] = m[pos[b], pos[a]] = 1
        return IncludedPairs(mode, ids, m)
    raise ValueError("Error reading focal node include/exclude pairs file.")


def read_reclass_table(path) -> dict:
    t = np.array(_read_rows(path), dtype=np.float64)
    if t.ndim != 2 or t.shape[1] != 2:
        raise ValueError(f"{path} must have exactly 2 columns")
    return {float(a): float(b) for a, b in t}


def habitat_conductance(cells, *, is_resistance: bool = True, reclass: dict | None = None) -> np.ndarray:
    """Optionally reclassified, then 1 / resistance (or the conductance), -9999 cells at 0
    (circuitscape.py:329-348)."""
    c = np.array(cells, dtype=np.float64)
    if reclass:
        flat = c.ravel()
        for k, v in enumerate(flat):
            if v in reclass:
                flat[k] = reclass[v]
        c = flat.reshape(c.shape)
    nodata = c == NODATA
    if is_resistance:
        if np.any(c == 0):
            raise ValueError("zero resistance values are not supported for habitat maps; use a short-circuit "
                             "region file instead")
        g = 1 / c
    else:
        g = c.copy()
    g[nodata] = 0.0
    return g


# --- the node graph (circuitscape.cpp:145-263) ----------------------------------------------------------------------

@dataclass
class RasterGraph:
    """Nodes: habitat cells numbered column-major, the cells of a short-circuit region with habitat merged into
    the node of its first habitat cell.  CSR adjacency (neighbours ascending) with the summed edge conductances,
    the Laplacian's diagonal and the connected components (numbered by their smallest node)."""

    nx: int
    ny: int
    n_nodes: int
    nodemap: np.ndarray   # cell (row-major) -> node, -1: none
    ptr: np.ndarray       # int64, n_nodes + 1
    adj: np.ndarray       # int32
    w: np.ndarray         # float64
    degree: np.ndarray    # float64
    comp: np.ndarray      # node -> component
    n_comp: int
    four_neighbors: bool = False
    avg_resistances: bool = False
    merged: bool = False  # a node covers several cells, or a cell without habitat


def _average(x, y, diagonal: bool, resistances: bool):
    if resistances:
        with np.errstate(divide="ignore"):
            s = (1 / x + 1 / y) / 2
            return 1 / (SQRT2 * s) if diagonal else 1 / s
    return (x + y) / TWO_SQRT2 if diagonal else (x + y) / 2


def raster_graph(gmap: np.ndarray, polymap: np.ndarray | None, avg_resistances: bool,
                 four_neighbors: bool, *, lite: bool = False) -> RasterGraph:
    """The node graph.  With ``lite``, a plain grid graph (no node merging cells, average-conductance weights) comes
    without its CSR arrays (ptr, adj, w and degree are None): its components are the 8- or 4-connected regions of
    habitat cells, numbered by their smallest node; the raster solvers need nothing more.  Other graphs are built in
    full either way."""
    ny, nx = gmap.shape
    n = nx * ny
    g = np.ascontiguousarray(gmap, dtype=np.float64).ravel()
    cm = np.arange(n).reshape(ny, nx).T.ravel()  # cells in column-major order
    hab_cm = cm[g[cm] > 0]
    label = np.zeros(n, dtype=np.int64)
    label[hab_cm] = np.arange(1, len(hab_cm) + 1)
    if polymap is not None:
        pm = np.ascontiguousarray(polymap, dtype=np.int64).ravel()
        sel = hab_cm[pm[hab_cm] != 0]
        ids, first = np.unique(pm[sel], return_index=True)  # first habitat cell of each region, column-major
        first_label = label[sel[first]]
        cells = np.flatnonzero(pm != 0)
        k = np.searchsorted(ids, pm[cells])
        k_ok = k < len(ids)
        hit = np.zeros(len(cells), dtype=bool)
        hit[k_ok] = ids[k[k_ok]] == pm[cells[k_ok]]
        label[cells[hit]] = first_label[k[hit]]
    on = label != 0
    uniq, inv = np.unique(label[on], return_inverse=True)
    nodemap = np.full(n, -1, dtype=np.int64)
    nodemap[on] = inv
    n_nodes = len(uniq)
    if lite and not avg_resistances and np.count_nonzero(on) == n_nodes and not np.any(on & ~(g > 0)):
        from scipy import ndimage
        structure = np.ones((3, 3), dtype=bool) if not four_neighbors else ndimage.generate_binary_structure(2, 1)
        lab, k = ndimage.label(nodemap.reshape(ny, nx) >= 0, structure=structure)
        node_lab = np.empty(n_nodes, dtype=np.int64)
        node_lab[nodemap[on]] = lab.ravel()[on] - 1
        _, first = np.unique(node_lab, return_index=True)
        rank = np.empty(k, dtype=np.int64)
        rank[np.argsort(first)] = np.arange(k)
        return RasterGraph(nx, ny, n_nodes, nodemap, None, None, None, None, rank[node_lab] if k else node_lab, int(k),
                           bool(four_neighbors), bool(avg_resistances), False)

    # edges in column-major cell order: right, below, below right, above right; both orientations
    ys, xs = np.divmod(cm, nx)
    dirs = [(xs + 1 < nx, 1, False), (ys + 1 < ny, nx, False)]
    if not four_neighbors:
        dirs += [((ys + 1 < ny) & (xs + 1 < nx), nx + 1, True), ((ys > 0) & (xs + 1 < nx), 1 - nx, True)]
    rank_of = np.empty(n, dtype=np.int64)
    rank_of[cm] = np.arange(n)  # position of each cell in column-major order
    A, B, W, order = [], [], [], []
    for d, (ok, off, diag) in enumerate(dirs):
        c = cm[ok & (nodemap[cm] >= 0)]
        e = c + off
        a, b = nodemap[c], nodemap[e]
        keep = b >= 0
        c, e, a, b = c[keep], e[keep], a[keep], b[keep]
        w = _average(g[c], g[e], diag, avg_resistances)
        keep = a != b  # within a merged node: nothing in the Laplacian
        c, a, b, w = c[keep], a[keep], b[keep], w[keep]
        rank = rank_of[c]
        for first, (p, q) in enumerate(((a, b), (b, a))):
            A.append(p)
            B.append(q)
            W.append(w)
            order.append((rank * 4 + d) * 2 + first)
    A, B, W, order = (np.concatenate(x) if x else np.zeros(0) for x in (A, B, W, order))
    # back to the order met (the emission keys are distinct integers below 8 x cells: a counting scatter), then a
    # stable sort by (row, column): duplicates keep the order met
    slot = np.full(len(cm) * 8, -1, dtype=np.int64)  # keys (rank x 4 + direction) x 2 + orientation
    slot[order.astype(np.int64)] = np.arange(len(order))
    o = slot[slot >= 0]
    A, B, W = A[o].astype(np.int64), B[o].astype(np.int64), W[o]
    s = np.argsort(A * max(n_nodes, 1) + B, kind="stable")
    A, B, W = A[s], B[s], W[s]
    if len(A):
        start = np.flatnonzero(np.r_[True, (A[1:] != A[:-1]) | (B[1:] != B[:-1])])
        wsum = W[start].copy()
        dup = np.diff(np.r_[start, len(A)]) > 1
        for k in np.flatnonzero(dup):  # duplicates (merged nodes) summed in the order met
            acc = W[start[k]]
            for t in range(start[k] + 1, start[k + 1] if k + 1 < len(start) else len(A)):
                acc = acc + W[t]
            wsum[k] = acc
        A, B = A[start], B[start]
    else:
        wsum = W
    ptr = np.zeros(n_nodes + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(A, minlength=n_nodes))
    degree = np.zeros(n_nodes)
    # the diagonal sums each row's entries in adjacency order
    for k in range(int(np.diff(ptr).max()) if n_nodes and len(A) else 0):
        rows = np.flatnonzero(ptr[:-1] + k < ptr[1:])
        degree[rows] += wsum[ptr[:-1][rows] + k]
    comp, n_comp = _components(n_nodes, ptr, B, wsum)
    merged = bool(np.count_nonzero(nodemap >= 0) != n_nodes or np.any((nodemap >= 0) & ~(g > 0)))
    return RasterGraph(nx, ny, n_nodes, nodemap, ptr, B.astype(np.int32), wsum.astype(np.float64), degree, comp,
                       n_comp, bool(four_neighbors), bool(avg_resistances), merged)


def _components(n_nodes, ptr, adj, w):
    """Connected components over the edges of nonzero weight, numbered by their smallest node."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    if n_nodes == 0:
        return np.zeros(0, dtype=np.int64), 0
    rows = np.repeat(np.arange(n_nodes), np.diff(ptr))
    nz = w != 0  # edges of weight 0 do not connect (stored zeros would count as edges)
    m = csr_matrix((np.ones(int(nz.sum()), dtype=np.int8), (rows[nz], np.asarray(adj)[nz])),
                   shape=(n_nodes, n_nodes))
    k, lab = connected_components(m, directed=False)
    _, first = np.unique(lab, return_index=True)
    rank = np.empty(k, dtype=np.int64)
    rank[np.argsort(first)] = np.arange(k)
    return rank[lab], int(k)


# --- the GPU solves -------------------------------------------------------------------------------------------------

@dataclass
class GraphSolveStats:
    jobs: int = 0
    iters_max: int = 0
    iters_mean: float = 0.0
    failures: int = 0


@dataclass
class ComponentSystem:
    """One component's grounded Laplacian in the form lsb_graph_pairs takes: its nodes (ascending), the
    graph-node -> local-index table, and the CSR rows (edges leaving the component dropped; they weigh 0) with the
    diagonal plus the reference factorisation's shift."""

    members: np.ndarray
    local: np.ndarray
    ptr: np.ndarray
    adj: np.ndarray
    w: np.ndarray
    diag: np.ndarray


def component_system(graph: RasterGraph, members: np.ndarray) -> ComponentSystem:
    m = len(members)
    local = np.full(graph.n_nodes, -1, dtype=np.int64)
    local[members] = np.arange(m)
    lens = graph.ptr[members + 1] - graph.ptr[members]
    idx = np.repeat(graph.ptr[members], lens) + (np.arange(lens.sum()) - np.repeat(np.cumsum(lens) - lens, lens))
    la = local[graph.adj[idx]]
    keep = la >= 0
    rowid = np.repeat(np.arange(m), lens)[keep]
    ptr = np.zeros(m + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(rowid, minlength=m))
    return ComponentSystem(members, local, ptr, la[keep].astype(np.int32), graph.w[idx][keep],
                           graph.degree[members] + K_SHIFT)


def system_to_device(sys_: ComponentSystem, device):
    """(n, ptr, adj, w, diag) as device tensors."""
    import torch
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(device)  # noqa: E731
    return (len(sys_.members), t(sys_.ptr, np.int64), t(sys_.adj, np.int32), t(sys_.w, np.float64),
            t(sys_.diag, np.float64))


def solve_pairs(dsys, ground: int, src, dst, *, currents: bool = True, params=None, stats: bool = True):
    """One lsb_graph_pairs call on the current stream: ``dsys`` from system_to_device, ``ground`` / ``src`` /
    ``dst`` local node indices (src, dst: int32 device tensors).  Returns (volt, cur, GraphStats): jobs x n device
    tensors (cur None without ``currents``) and the statistics (None with ``stats=False``, which does not wait)."""
    import torch
    lib = N.load()
    n, d_ptr, d_adj, d_w, d_diag = dsys
    params = params if params is not None else graph_params()
    nb = int(src.numel())
    dev = d_ptr.device
    volt = torch.empty((nb, n), dtype=torch.float64, device=dev)
    cur = torch.empty((nb, n), dtype=torch.float64, device=dev) if currents else None
    nbytes = C.c_size_t(0)
    rc = lib.lsb_graph_pairs_workspace_size(n, nb, C.byref(params), C.byref(nbytes))
    N.check(rc, C.create_string_buffer(b"invalid graph size or parameters"))
    ws = torch.empty(max(int(nbytes.value), 16), dtype=torch.uint8, device=dev)
    st = N.GraphStats() if stats else None
    err = C.create_string_buffer(1024)
    rc = lib.lsb_graph_pairs(n, d_ptr.data_ptr(), d_adj.data_ptr(), d_w.data_ptr(), d_diag.data_ptr(), int(ground),
                             nb, src.data_ptr(), dst.data_ptr(), C.byref(params), volt.data_ptr(),
                             cur.data_ptr() if cur is not None else None, ws.data_ptr(), ws.numel(),
                             C.byref(st) if st is not None else None, err, len(err),
                             torch.cuda.current_stream(dev).cuda_stream)
    N.check(rc, err)
    return volt, cur, st


def _solve_component(graph: RasterGraph, members: np.ndarray, ground: int, src: np.ndarray, dst: np.ndarray,
                     want_currents: bool, params, stats: GraphSolveStats, device):
    """Every job (src, dst node) on one component: unit current into dst, out of src, the ground node at 0 V.
    Returns (volt, cur) as numpy arrays of jobs x members: the voltages relative to the source node, and the node
    currents (None without ``want_currents``)."""
    import torch
    sys_ = component_system(graph, members)
    dsys = system_to_device(sys_, device)
    m = len(members)
    js, jd = sys_.local[src].astype(np.int32), sys_.local[dst].astype(np.int32)
    nj = len(js)
    volt = np.empty((nj, m))
    cur = np.empty((nj, m)) if want_currents else None
    per = max(1, min(nj, (1 << 27) // max(m * 16, 1)))  # jobs per call: outputs of at most 128 MiB
    for b0 in range(0, nj, per):
        b1 = min(nj, b0 + per)
        nb = b1 - b0
        d_src = torch.from_numpy(js[b0:b1]).to(device)
        d_dst = torch.from_numpy(jd[b0:b1]).to(device)
        try:
            v, c, st = solve_pairs(dsys, int(sys_.local[ground]), d_src, d_dst, currents=want_currents,
                                   params=params)
        except N.NativeError:
            stats.failures += nb
            raise
        volt[b0:b1] = v.cpu().numpy()
        if want_currents:
            cur[b0:b1] = c.cpu().numpy()
        stats.iters_mean = (stats.iters_mean * stats.jobs + st.iters_mean * nb) / (stats.jobs + nb)
        stats.jobs += nb
        stats.iters_max = max(stats.iters_max, int(st.iters_max))
    return volt, cur


MAX_RASTER_SIDE = 1024  # the raster solver's limit


def raster_route(graph: RasterGraph) -> bool:
    """Whether the pair solves can run on the raster solver: a plain grid graph (one habitat cell per node, no
    short-circuit regions), average-conductance weights and sides within the raster solver's limit."""
    return (not graph.merged and not graph.avg_resistances and graph.nx <= MAX_RASTER_SIDE
            and graph.ny <= MAX_RASTER_SIDE)


def _solve_component_rasters(graph: RasterGraph, gmap: np.ndarray, members: np.ndarray, src: np.ndarray,
                             dst: np.ndarray, want_currents: bool, tol: float, stats: GraphSolveStats, device,
                             focal: np.ndarray | None = None):
    """The jobs of one component on the raster solver (lsb_rasters: FP32 CG with a multigrid preconditioner inside
    FP64 refinement): job j is the raster with a unit source at dst[j]'s cell and a direct ground at src[j]'s, whose
    voltages are the pair's voltages relative to its source and whose node currents are the pair's.  Same contract
    as _solve_component; with ``focal`` (member indices) it returns instead (the voltages at those members, jobs x
    focal; the currents summed over the jobs; their maximum over the jobs), reduced on the device."""
    import torch

    from . import raster as R
    ny, nx = graph.ny, graph.nx
    ncell = nx * ny
    on = np.flatnonzero(graph.nodemap >= 0)
    node_cell = np.empty(graph.n_nodes, dtype=np.int64)
    node_cell[graph.nodemap[on]] = on
    mcell = torch.from_numpy(node_cell[members]).to(device)
    nj = len(src)
    if focal is not None:
        fcell = torch.from_numpy(node_cell[members[focal]]).to(device)
        volt = np.empty((nj, len(focal)))
        c_sum = torch.zeros(len(members), dtype=torch.float64, device=device)
        c_max = torch.full((len(members),), -np.inf, dtype=torch.float64, device=device)
    else:
        volt = np.empty((nj, len(members)))
        cur = np.empty((nj, len(members))) if want_currents else None
    p = R.raster_params(four_neighbors=graph.four_neighbors, tol=tol)
    g_dev = torch.from_numpy(np.ascontiguousarray(gmap, dtype=np.float64).ravel()).to(device)
    per = max(1, min(nj, (1 << 31) // (40 * ncell)))  # inputs and outputs of a batch within 2 GiB
    for b0 in range(0, nj, per):
        b1 = min(nj, b0 + per)
        nb = b1 - b0
        base = torch.arange(nb, device=device, dtype=torch.int64) * ncell
        S = torch.zeros(nb * ncell, dtype=torch.float64, device=device)
        GR = torch.zeros_like(S)
        S[base + torch.from_numpy(node_cell[dst[b0:b1]]).to(device)] = 1.0
        GR[base + torch.from_numpy(node_cell[src[b0:b1]]).to(device)] = np.inf
        c, v, st = R.run_rasters(g_dev.repeat(nb), S, GR, [(ny, nx)] * nb, p)
        if focal is not None:
            volt[b0:b1] = v.view(nb, ncell)[:, fcell].cpu().numpy()
            cm = c.view(nb, ncell)[:, mcell]
            c_sum += cm.sum(dim=0)
            c_max = torch.maximum(c_max, cm.max(dim=0).values)
        else:
            volt[b0:b1] = v.view(nb, ncell)[:, mcell].cpu().numpy()
            if want_currents:
                cur[b0:b1] = c.view(nb, ncell)[:, mcell].cpu().numpy()
        mean = st.iters_total / max(st.n_solved, 1)
        stats.iters_mean = (stats.iters_mean * stats.jobs + mean * nb) / (stats.jobs + nb)
        stats.jobs += nb
        stats.iters_max = max(stats.iters_max, int(st.iters_max))
    if focal is not None:
        return volt, c_sum.cpu().numpy(), c_max.cpu().numpy()
    return volt, cur


def graph_params(tol=1e-13, max_iter=0):
    p = N.default_graph_params()
    p.tol = float(tol)
    if max_iter:
        p.max_iter = int(max_iter)
    return p


# --- pairwise (circuitscape.cpp:474-743) ----------------------------------------------------------------------------

@dataclass
class PairOptions:
    volt_maps: bool = False
    cur_maps: bool = False
    cum: bool = False
    max: bool = False
    focal_zero: bool = False
    null_currents: bool = False
    null_voltages: bool = False
    log_transform: bool = False

    def maps(self) -> bool:
        return self.volt_maps or self.cur_maps or self.cum or self.max


def raster_pairwise(graph: RasterGraph, gmap: np.ndarray, points: np.ndarray, excluded: np.ndarray,
                    o: PairOptions, emit=None, *, tol=1e-13, device=None, stats: GraphSolveStats | None = None,
                    pair_solver: str = "auto"):
    """Effective resistances between the focal points' nodes ``points`` (-1: off the graph), with the pair maps.

    Returns ``(resistances n x n, cum, max)``; ``emit(ci, cj, voltage_map, current_map)`` receives each pair's maps
    (None where not asked for).  Follows circuitscape.cpp:474-743: components in order, distinct focal nodes in
    first-appearance order, the component's last node grounded, jobs (source, destination) solved with a unit
    current, and without maps or exclusions the shortcut (only the first focal node's pairs, the others from the
    voltages).  ``pair_solver``: "graph" (lsb_graph_pairs, any graph), "raster" (lsb_rasters, plain grid graphs) or
    "auto" (the raster solver where the graph allows it)."""
    import torch
    if pair_solver not in ("auto", "graph", "raster"):
        raise ValueError('pair_solver must be "auto", "graph" or "raster"')
    if pair_solver == "raster" and not raster_route(graph):
        raise ValueError("the raster pair solver needs a plain grid graph (no short-circuit regions, average "
                         f"conductances, sides up to {MAX_RASTER_SIDE})")
    on_rasters = pair_solver == "raster" or (pair_solver == "auto" and raster_route(graph))
    if not on_rasters and graph.ptr is None:
        # a lite graph (no node merging cells): its node map does not depend on the polygons, so the full graph
        # without them is the same graph
        graph = raster_graph(gmap, None, graph.avg_resistances, graph.four_neighbors)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    params = graph_params(tol)
    stats = stats if stats is not None else GraphSolveStats()
    npt = len(points)
    ncell = graph.nx * graph.ny
    gflat = np.ascontiguousarray(gmap, dtype=np.float64).ravel()
    R = np.full((npt, npt), -1.0)
    shortcut = not o.maps() and not excluded.any()
    voltmatrix = np.zeros((npt, npt)) if shortcut else None
    short_res = np.full((npt, npt), -1.0) if shortcut else None
    cum = np.zeros(ncell) if o.cum else None
    mx = np.full(ncell, NODATA) if o.max else None
    order = np.argsort(graph.comp, kind="stable")
    bounds = np.searchsorted(graph.comp[order], np.arange(graph.n_comp + 1))
    positions: dict[int, list] = {}
    for i, v in enumerate(points):
        if v >= 0:
            positions.setdefault(int(v), []).append(i)
    comp_of = np.append(graph.comp, -1)  # index -1 (no node) gives component -1
    pcomp = comp_of[np.asarray(points, dtype=np.int64)]
    cell_comp = comp_of[graph.nodemap]
    for k in range(graph.n_comp):
        csub = []
        for i in range(npt):
            v = int(points[i])
            if v >= 0 and pcomp[i] == k and v not in csub:
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
        members = order[bounds[k]:bounds[k + 1]]  # ascending (stable sort of ascending nodes)
        ground = int(members[-1])
        src = np.array([j[0] for j in jobs], dtype=np.int64)
        dst = np.array([j[1] for j in jobs], dtype=np.int64)
        # only the cum / max maps, one focal point per node: each job adds its current map once, so the maps follow
        # from the jobs' currents at once (on the host the sum runs over the jobs in order, as the per-pair additions
        # do; the raster route reduces on the device)
        summed = (o.maps() and not (o.volt_maps or o.cur_maps or o.focal_zero or o.log_transform or o.null_currents)
                  and all(len(positions[v]) == 1 for v in csub))
        mindex = {int(v): q for q, v in enumerate(members)}
        c_sum = c_max = None
        if on_rasters and summed:
            fq = np.array([mindex[v] for v in csub], dtype=np.int64)
            volt, c_sum, c_max = _solve_component_rasters(graph, gmap, members, src, dst, True, min(tol, 1e-12),
                                                          stats, dev, focal=fq)
            mindex = {v: i for i, v in enumerate(csub)}  # the loop below reads the focal voltages only
            cur = None
        elif on_rasters:
            volt, cur = _solve_component_rasters(graph, gmap, members, src, dst, o.maps(), min(tol, 1e-12), stats,
                                                 dev)
        else:
            volt, cur = _solve_component(graph, members, ground, src, dst, o.maps(), params, stats, dev)
        in_k = cell_comp == k
        cells_k = np.flatnonzero(in_k)
        node_q = np.searchsorted(members, graph.nodemap[cells_k])
        if summed:
            if c_sum is None:
                c_sum, c_max = np.add.reduce(cur, axis=0), cur.max(axis=0)
            if o.cum:
                cum[cells_k] += c_sum[node_q]
            if o.max:
                np.maximum(mx, 0.0, out=mx)
                mx[cells_k] = np.maximum(mx[cells_k], c_max[node_q])
        for jn, (s, d) in enumerate(jobs):
            vcol = volt[jn]
            resistance = vcol[mindex[d]] - vcol[mindex[s]]
            vmap = cmap = None
            if o.maps() and not summed:
                if o.volt_maps:
                    vmap = np.zeros(ncell)
                    vmap[cells_k] = vcol[node_q]
                    if o.null_voltages:
                        vmap[gflat == 0] = NODATA
                cmap = np.zeros(ncell)
                cmap[cells_k] = cur[jn][node_q]
                if o.focal_zero:
                    nodes_k = graph.nodemap[cells_k]
                    cmap[cells_k[(nodes_k == s) | (nodes_k == d)]] = 0.0
                if o.log_transform:
                    with np.errstate(divide="ignore", invalid="ignore"):
                        cmap = np.where(cmap > 0, np.log10(np.where(cmap > 0, cmap, 1.0)), NODATA)
                if o.null_currents:
                    cmap[gflat == 0] = NODATA
            for ci in positions[s]:
                for cj in positions[d]:
                    if excluded[ci, cj]:
                        continue
                    R[ci, cj] = R[cj, ci] = resistance
                    if shortcut:
                        for i in range(1, npt):
                            v = int(points[i])
                            if v < 0 or pcomp[i] != k:
                                continue
                            voltmatrix[i, cj] = 1 - vcol[mindex[v]] / resistance
                        continue
                    if not o.maps() or summed:
                        continue
                    if o.cum:
                        cum += cmap
                    if o.max:
                        np.maximum(mx, cmap, out=mx)
                    if emit is not None and (o.volt_maps or o.cur_maps):
                        emit(ci, cj, vmap.reshape(graph.ny, graph.nx) if vmap is not None else None,
                             cmap.reshape(graph.ny, graph.nx).copy() if o.cur_maps else None)
        if shortcut:
            _shortcut(R, short_res, voltmatrix, points, pcomp, k, positions[csub[0]][0])
    if shortcut:
        R = short_res
    np.fill_diagonal(R, 0.0)
    if cum is not None:
        cum = np.maximum(cum, NODATA).reshape(graph.ny, graph.nx)
    if mx is not None:
        mx = np.maximum(mx, NODATA).reshape(graph.ny, graph.nx)
    return R, cum, mx


def _shortcut(R, S, voltmatrix, points, pcomp, k, anchor):
    """The resistances of every pair of the component from those of its anchor's pairs and the voltages
    (circuitscape.cpp:705-731)."""
    invalid = -777.0
    npt = len(points)
    check = [points[i] >= 0 and pcomp[i] == k for i in range(npt)]
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
            if r1x != invalid:
                S[anchor, y] = S[y, anchor] = r12
                r2x = 2 * r12 * voltmatrix[x, y] + r1x - r12
                if S[y, x] != invalid:
                    S[y, x] = S[x, y] = r2x
            else:
                S[x, :] = invalid
                S[:, x] = invalid


# --- the public calls ------------------------------------------------------------------------------------------------

@dataclass
class CircuitscapeResult:
    """``resistances``: ids in the first row and column (-1: not connected); ``cum_current``, ``max_current``:
    sum and maximum of the pairs' current maps; ``maps``: per-pair maps."""

    resistances: np.ndarray | None = None
    cum_current: np.ndarray | None = None
    max_current: np.ndarray | None = None
    maps: dict = field(default_factory=dict)
    stats: GraphSolveStats | None = None
    voltage: np.ndarray | None = None   # advanced mode: per-cell maps (0 on cells without a node)
    current: np.ndarray | None = None
    nodemap: np.ndarray | None = None


def _grid(value, name) -> np.ndarray:
    a = np.array(value, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError(f"{name} must be a 2-D raster")
    return np.where(np.isnan(a), NODATA, a)


def _points_from_map(pm: np.ndarray) -> FocalPoints:
    pm = pm.copy()
    pm[pm == NODATA] = 0
    jj, ii = np.nonzero(pm.T)
    return _sorted_points(ii + 1, jj + 1, pm[ii, jj])


def _apply_included_pairs(points: FocalPoints, pairs: IncludedPairs | None):
    if pairs is None:
        return points, set()
    if pairs.mode == "include":
        keep = np.isin(points.ids, pairs.ids)
        points = FocalPoints(points.rows[keep], points.cols[keep], points.ids[keep])
    return points, pairs.excluded()


def region_polymap(polymap, n: int, cells: np.ndarray, ids: np.ndarray, pt1: int, pt2: int) -> np.ndarray:
    """The short-circuit regions of one pair of focal regions (circuitscape.cpp:749-779): without polygons the two
    regions' cells; with polygons, each region of several cells becomes one new region together with every polygon
    it overlaps."""
    if polymap is None:
        poly = np.zeros(n, dtype=np.int64)
        poly[cells[ids == pt1]] = pt1
        poly[cells[ids == pt2]] = pt2
        return poly
    poly = np.ascontiguousarray(polymap, dtype=np.int64).ravel().copy()
    k = int(poly.max())
    for pt in (pt1, pt2):
        idx = cells[ids == pt]
        if len(idx) == 1:
            continue
        k += 1
        vals = np.unique(poly[idx][poly[idx] != 0])
        if len(vals):
            poly[np.isin(poly, vals)] = k
        poly[idx] = k
    return poly


def _run_regions(g, poly, points: FocalPoints, excluded_ids: set, four, avg, o: PairOptions, emit, tol, device,
                 pair_solver="auto"):
    """pairwise_regions (circuitscape.cpp:781-866): every pair of distinct ids gets its own graph, its two regions
    made short-circuit regions, and one solve between the nodes of their first cells."""
    rows, cols = points.cells
    cells = (rows * g.shape[1] + cols).astype(np.int64)
    ids = points.ids
    pts = np.unique(ids)
    n = len(pts)
    ex = np.zeros((n, n), dtype=bool)
    if excluded_ids:
        for a in range(n):
            for b in range(n):
                ex[a, b] = (int(pts[a]), int(pts[b])) in excluded_ids
    R = np.full((n, n), -1.0)
    ncell = g.size
    cum = np.zeros(g.shape) if o.cum else None
    mx = np.full(g.shape, NODATA) if o.max else None
    stats = GraphSolveStats()
    shape = poly.shape if poly is not None else g.shape
    for i in range(n):
        for j in range(i + 1, n):
            if ex[i, j] or ex[j, i]:
                continue
            pm = region_polymap(poly, ncell, cells, ids, int(pts[i]), int(pts[j])).reshape(shape)
            graph = raster_graph(g, pm, avg, four, lite=pair_solver != "graph")
            nodes = np.array([graph.nodemap[cells[np.flatnonzero(ids == pts[e])[0]]] for e in (i, j)])
            got = []
            r2, c2, m2 = raster_pairwise(graph, g, nodes, np.zeros((2, 2), dtype=bool), o,
                                         lambda ci, cj, v, c: got.append((ci, cj, v, c)), tol=tol, device=device,
                                         stats=stats, pair_solver=pair_solver)
            R[i, j] = R[j, i] = r2[0, 1]
            if cum is not None:
                cum += c2
            if mx is not None:
                np.maximum(mx, m2, out=mx)
            for ci, cj, v, c in got:
                if emit is not None:
                    emit(i if ci == 0 else j, i if cj == 0 else j, v, c)
    np.fill_diagonal(R, 0.0)
    if cum is not None:
        cum = np.maximum(cum, NODATA)
    res = np.zeros((n + 1, n + 1))
    res[0, 1:] = pts
    res[1:, 0] = pts
    res[1:, 1:] = R
    return res, cum, mx, stats


def _run_pairwise(g, poly, points: FocalPoints, excluded_ids: set, four, avg, o: PairOptions, emit, tol, device,
                  pair_solver="auto"):
    if points.has_regions:
        return _run_regions(g, poly, points, excluded_ids, four, avg, o, emit, tol, device, pair_solver)
    graph = raster_graph(g, poly, avg, four, lite=pair_solver != "graph")
    rows, cols = points.cells
    cells = rows * g.shape[1] + cols
    ok = (cells >= 0) & (cells < g.size)
    nodes = np.where(ok, graph.nodemap[np.where(ok, cells, 0)], -1)
    ids = points.ids
    n = len(ids)
    ex = np.zeros((n, n), dtype=bool)
    if excluded_ids:
        for a in range(n):
            for b in range(n):
                ex[a, b] = (int(ids[a]), int(ids[b])) in excluded_ids
    stats = GraphSolveStats()
    R, cum, mx = raster_pairwise(graph, g, nodes, ex, o, emit, tol=tol, device=device, stats=stats,
                                 pair_solver=pair_solver)
    res = np.zeros((n + 1, n + 1))
    res[0, 1:] = ids
    res[1:, 0] = ids
    res[1:, 1:] = R
    return res, cum, mx, stats


def circuitscape_pairwise(habitat, points, *, habitat_is_resistance: bool = True, polygons=None, mask=None,
                          four_neighbors: bool = False, avg_resistances: bool = False, included_pairs=None,
                          voltage_maps: bool = False, current_maps: bool = False, cum_map: bool = False,
                          max_map: bool = False, set_focal_node_currents_to_zero: bool = False,
                          set_null_currents_to_nodata: bool = False, set_null_voltages_to_nodata: bool = False,
                          log_transform_maps: bool = False, reclass: dict | None = None, n_threads: int = 0,
                          tol: float = 1e-13, device=None, pair_solver: str = "auto") -> CircuitscapeResult:
    """Effective resistances between every pair of focal points on a raster (drop-in for
    ``ls.circuit.circuitscape_pairwise``, circuitscape.py:550-670), solved on the GPU.

    ``habitat``: resistances (or conductances), NaN / -9999 = NoData.  ``points``: a raster of focal ids (0 / NoData
    elsewhere) or :class:`FocalPoints`.  ``polygons``: short-circuit region ids; ``mask``: cells where it is not
    positive are removed; ``included_pairs``: :class:`IncludedPairs` or a path.  The map options keep each pair's
    voltage / current map in ``result.maps`` (keys ``("voltage", id1, id2)`` / ``("current", id1, id2)``) and the
    sum / maximum of the current maps.  ``n_threads`` is accepted for compatibility; ``tol`` is the CG's relative
    residual target; ``pair_solver`` chooses the GPU solve of the pairs: "raster" (the multigrid raster solver, for
    plain grid graphs), "graph" (Jacobi CG on the node graph, any graph) or "auto".
    """
    del n_threads
    cells = _grid(habitat, "habitat")
    g = habitat_conductance(cells, is_resistance=habitat_is_resistance, reclass=reclass)
    poly = None
    if polygons is not None:
        pm = _grid(polygons, "polygons")
        if pm.shape != g.shape:
            raise ValueError("the polygons must have the habitat's shape")
        pm[pm == NODATA] = 0
        if not np.all(pm == np.round(pm)):
            raise ValueError("the polygon raster must hold integer ids")
        poly = pm.astype(np.int64)
    if mask is not None:
        m = _grid(mask, "mask")
        if m.shape != g.shape:
            raise ValueError("the mask must have the habitat's shape")
        m[m == NODATA] = 0
        g = g * np.where(m > 0, 1.0, 0.0)
        if g.sum() == 0:
            raise ValueError("Mask file deleted everything!")
    if not isinstance(points, FocalPoints):
        pm = _grid(points, "points")
        if pm.shape != g.shape:
            raise ValueError("the points must have the habitat's shape")
        points = _points_from_map(pm)
    if included_pairs is not None and not isinstance(included_pairs, IncludedPairs):
        included_pairs = read_included_pairs(included_pairs)
    points, excluded = _apply_included_pairs(points, included_pairs)
    o = PairOptions(volt_maps=voltage_maps, cur_maps=current_maps, cum=current_maps or cum_map, max=max_map, focal_zero=set_focal_node_currents_to_zero,
                    null_currents=set_null_currents_to_nodata, null_voltages=set_null_voltages_to_nodata,
                    log_transform=log_transform_maps)
    maps: dict = {}
    ids = np.unique(points.ids) if points.has_regions else points.ids

    def emit(ci, cj, volt, cur):
        key = (int(ids[ci]), int(ids[cj]))
        if volt is not None:
            maps[("voltage", *key)] = volt
        if cur is not None:
            maps[("current", *key)] = cur

    res, cum, mx, stats = _run_pairwise(g, poly, points, excluded, four_neighbors, avg_resistances, o, emit, tol,
                                        device, pair_solver)
    return CircuitscapeResult(resistances=res, cum_current=cum, max_current=mx, maps=maps, stats=stats)


# --- advanced mode, one-to-all, all-to-one (circuitscape.cpp:382-470,870-1083; circuitscape.py:406-516,704-955) ----

POLICIES = ("keepall", "rmvsrc", "rmvgnd", "rmvall")


def node_sums(graph: RasterGraph, cells: np.ndarray, vals: np.ndarray) -> np.ndarray:
    """Per-node sums of cell values, cells taken in column-major order (stable), zeros skipped."""
    cells = np.asarray(cells, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    s = np.zeros(graph.n_nodes)
    if len(cells) == 0:
        return s
    order = np.lexsort((cells // graph.nx, cells % graph.nx))
    c, v = cells[order], vals[order]
    node = graph.nodemap[c]
    keep = (node >= 0) & (v != 0)
    np.add.at(s, node[keep], v[keep])  # unbuffered: repeated nodes add in the order given
    return s


def resolve_conflicts(src: np.ndarray, gnd: np.ndarray, policy: str):
    """Finite grounds (taken before the policy), then the policy on nodes with both a source and a ground, then no
    direct ground under a positive source (circuitscape.cpp:881-900).  Returns (src, gnd, finite)."""
    finite = np.where(gnd < np.inf, gnd, 0.0)
    both = (src != 0) & (gnd != 0)
    if policy in ("rmvsrc", "rmvall"):
        src = np.where(both, 0.0, src)
    elif policy == "rmvgnd":
        gnd = np.where(both, 0.0, gnd)
    gnd = np.where((gnd == np.inf) & (src > 0), 0.0, gnd)
    return src, gnd, finite


def solve_problems(dsys, jobs, *, currents: bool = True, params=None, stats: bool = True):
    """One lsb_graph_solve call: ``jobs`` lists (src_nodes, src_vals, direct_nodes, finite_nodes, finite_vals) in
    local node indices.  Returns (volt, cur, GraphStats) as in solve_pairs."""
    import torch
    lib = N.load()
    n, d_ptr, d_adj, d_w, d_diag = dsys
    params = params if params is not None else graph_params()
    dev = d_ptr.device
    nb = len(jobs)

    def csr(k):
        lens = [len(j[k]) for j in jobs]
        ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        nodes = np.concatenate([np.asarray(j[k], dtype=np.int32) for j in jobs]) if sum(lens) else np.zeros(1, np.int32)
        return ptr, nodes

    s_ptr, s_node = csr(0)
    s_val = np.concatenate([np.asarray(j[1], dtype=np.float64) for j in jobs] + [np.zeros(1)])
    d_ptr2, d_node = csr(2)
    f_ptr, f_node = csr(3)
    f_val = np.concatenate([np.asarray(j[4], dtype=np.float64) for j in jobs] + [np.zeros(1)])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    T = [t(a) for a in (s_ptr, s_node, s_val, d_ptr2, d_node, f_ptr, f_node, f_val)]
    volt = torch.empty((nb, n), dtype=torch.float64, device=dev)
    cur = torch.empty((nb, n), dtype=torch.float64, device=dev) if currents else None
    nbytes = C.c_size_t(0)
    rc = lib.lsb_graph_solve_workspace_size(n, nb, C.byref(params), C.byref(nbytes))
    N.check(rc, C.create_string_buffer(b"invalid graph size or parameters"))
    ws = torch.empty(max(int(nbytes.value), 16), dtype=torch.uint8, device=dev)
    st = N.GraphStats() if stats else None
    err = C.create_string_buffer(1024)
    rc = lib.lsb_graph_solve(n, d_ptr.data_ptr(), d_adj.data_ptr(), d_w.data_ptr(), d_diag.data_ptr(), nb,
                             *(x.data_ptr() for x in T), C.byref(params), volt.data_ptr(),
                             cur.data_ptr() if cur is not None else None, ws.data_ptr(), ws.numel(),
                             C.byref(st) if st is not None else None, err, len(err),
                             torch.cuda.current_stream(dev).cuda_stream)
    N.check(rc, err)
    return volt, cur, st


def advanced_many(graph: RasterGraph, srcs, gnds, only_nodes, policy: str, *, tol=1e-13, device=None,
                  stats: GraphSolveStats | None = None):
    """raster_advanced_many (circuitscape.cpp:904-1083) on the GPU: every problem (per-node sources and grounds,
    +inf a direct ground) is solved in each component that holds a nonzero source sum and a nonzero ground sum
    (only the component of its check node when only_nodes[p] >= 0; none when it is -2).  Returns per problem a dict
    with the node voltages and currents, the active nodes and whether anything was solved."""
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    params = graph_params(tol)
    stats = stats if stats is not None else GraphSolveStats()
    n = graph.n_nodes
    res = [resolve_conflicts(np.asarray(s, dtype=np.float64), np.asarray(g_, dtype=np.float64), policy)
           for s, g_ in zip(srcs, gnds)]
    out = [{"voltage": np.zeros(n), "current": np.zeros(n), "solved": False,
            "active": np.flatnonzero((r[0] != 0) | (r[1] != 0)).astype(np.int32)} for r in res]
    order = np.argsort(graph.comp, kind="stable")
    bounds = np.searchsorted(graph.comp[order], np.arange(graph.n_comp + 1))
    for k in range(graph.n_comp):
        members = order[bounds[k]:bounds[k + 1]]
        probs = []
        for p, (s, g_, _) in enumerate(res):
            only = int(only_nodes[p])
            if only == -2 or (only >= 0 and graph.comp[only] != k):
                continue
            if np.cumsum(s[members])[-1] != 0 and np.cumsum(g_[members])[-1] != 0:
                probs.append(p)
                out[p]["solved"] = True
        if not probs:
            continue
        sys_ = component_system(graph, members)
        dsys = system_to_device(sys_, dev)
        jobs = []
        for p in probs:
            s, g_, fin = res[p]
            sm, gm, fm = s[members], g_[members], fin[members]
            nz = np.flatnonzero(sm != 0)
            fz = np.flatnonzero(fm != 0)
            jobs.append((nz, sm[nz], np.flatnonzero(gm == np.inf), fz, fm[fz]))
        v, c, st = solve_problems(dsys, jobs, params=params)
        v, c = v.cpu().numpy(), c.cpu().numpy()
        for q, p in enumerate(probs):
            out[p]["voltage"][members] = v[q]
            out[p]["current"][members] = c[q]
        stats.iters_mean = (stats.iters_mean * stats.jobs + st.iters_mean * len(probs)) / (stats.jobs + len(probs))
        stats.jobs += len(probs)
        stats.iters_max = max(stats.iters_max, int(st.iters_max))
    return out


def _advanced_rasters(graph: RasterGraph, gmap, srcs, gnds, only_nodes, policy: str, tol: float, device):
    """advanced_many on the raster solver (lsb_rasters, multigrid), for a plain grid graph and problems on which the
    conflict policy decides nothing (no node with both a source and a ground): each problem becomes one raster with
    its sources and grounds on the components Circuitscape solves (a nonzero source sum and a nonzero ground sum,
    the check node's component only when there is one), zero elsewhere; the raster solver then solves exactly those
    components, with finite grounds on the diagonal and in the node currents.  Returns None when a problem does not
    qualify."""
    import torch

    from . import raster as R
    n = graph.n_nodes
    for s, g_ in zip(srcs, gnds):
        if np.any((np.asarray(s) != 0) & (np.asarray(g_) != 0)):
            return None
    ny, nx = graph.ny, graph.nx
    ncell = nx * ny
    on = np.flatnonzero(graph.nodemap >= 0)
    node_cell = np.empty(n, dtype=np.int64)
    node_cell[graph.nodemap[on]] = on
    out, cells_s, vals_s, cells_g, vals_g = [], [], [], [], []
    for p, (s, g_) in enumerate(zip(srcs, gnds)):
        s, g_, _ = resolve_conflicts(np.asarray(s, dtype=np.float64), np.asarray(g_, dtype=np.float64), policy)
        sum_s = np.bincount(graph.comp, weights=s, minlength=graph.n_comp)  # in node order, as the reference sums
        direct = np.bincount(graph.comp, weights=(g_ == np.inf).astype(np.float64), minlength=graph.n_comp) > 0
        sum_g = np.bincount(graph.comp, weights=np.where(g_ == np.inf, 0.0, g_), minlength=graph.n_comp)
        ok = (sum_s != 0) & (direct | (sum_g != 0))  # a direct ground makes the reference's sum infinite
        only = int(only_nodes[p])
        if only == -2:
            ok[:] = False
        elif only >= 0:
            keep = np.zeros_like(ok)
            keep[graph.comp[only]] = ok[graph.comp[only]]
            ok = keep
        node_ok = ok[graph.comp]
        ns = np.flatnonzero(node_ok & (s != 0))
        ng = np.flatnonzero(node_ok & (g_ != 0))
        cells_s.append(node_cell[ns])
        vals_s.append(s[ns])
        cells_g.append(node_cell[ng])
        vals_g.append(g_[ng])
        out.append({"voltage": np.zeros(n), "current": np.zeros(n), "solved": bool(ok.any()),
                    "active": np.flatnonzero((s != 0) | (g_ != 0)).astype(np.int32)})
    g_dev = torch.from_numpy(np.ascontiguousarray(gmap, dtype=np.float64).ravel()).to(device)
    nc = torch.from_numpy(node_cell).to(device)
    rp = R.raster_params(four_neighbors=graph.four_neighbors, tol=tol)
    todo = [p for p in range(len(out)) if out[p]["solved"]]
    per = max(1, (1 << 31) // (40 * ncell))  # inputs and outputs of a batch within 2 GiB
    for b0 in range(0, len(todo), per):
        batch = todo[b0:b0 + per]
        nb = len(batch)
        S = torch.zeros(nb * ncell, dtype=torch.float64, device=device)
        GR = torch.zeros_like(S)
        for q, p in enumerate(batch):
            S[torch.from_numpy(q * ncell + cells_s[p]).to(device)] = torch.from_numpy(vals_s[p]).to(device)
            GR[torch.from_numpy(q * ncell + cells_g[p]).to(device)] = torch.from_numpy(vals_g[p]).to(device)
        c, v, _ = R.run_rasters(g_dev.repeat(nb), S, GR, [(ny, nx)] * nb, rp)
        v = v.view(nb, ncell)[:, nc].cpu().numpy()
        c = c.view(nb, ncell)[:, nc].cpu().numpy()
        for q, p in enumerate(batch):
            out[p]["voltage"] = v[q]  # 0 on the components not solved
            out[p]["current"] = c[q]
    return out


def multi_advanced(g, poly, avg: bool, four: bool, problems, policy: str, *, tol=1e-13, device=None, stats=None,
                   problem_solver: str = "auto"):
    """The reference's native circuitscape_multi_advanced on the GPU: one graph, many problems given by cells
    (src_cells / src_vals / gnd_cells / gnd_vals, check_cell -1 or a cell whose component alone is solved).
    Returns (nodemap, results).  ``problem_solver``: "graph" (lsb_graph_solve, any problem), "raster" (lsb_rasters;
    plain grid graphs and problems without a node that has both a source and a ground) or "auto" (the raster solver
    where it applies)."""
    if problem_solver not in ("auto", "graph", "raster"):
        raise ValueError('problem_solver must be "auto", "graph" or "raster"')
    graph = raster_graph(g, poly, avg, four, lite=problem_solver != "graph")
    srcs, gnds, only = [], [], []
    for q in problems:
        srcs.append(node_sums(graph, q["src_cells"], q["src_vals"]))
        gnds.append(node_sums(graph, q["gnd_cells"], q["gnd_vals"]))
        o = -1
        if q["check_cell"] >= 0:
            o = int(graph.nodemap[q["check_cell"]])
            if o < 0:
                o = -2
        only.append(o)
    if problem_solver != "graph" and raster_route(graph):
        import torch
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        routed = _advanced_rasters(graph, g, srcs, gnds, only, policy, min(tol, 1e-12), dev)
        if routed is not None:
            return graph.nodemap.reshape(g.shape), routed
    if problem_solver == "raster":
        raise ValueError("the raster problem solver needs a plain grid graph and problems without a node that has "
                         "both a source and a ground")
    if graph.ptr is None:  # a lite graph: the full one (without the polygons, which do not change it)
        graph = raster_graph(g, None, avg, four)
    return graph.nodemap.reshape(g.shape), advanced_many(graph, srcs, gnds, only, policy, tol=tol, device=device,
                                                         stats=stats)


def _advanced(g, poly, src, gnd, four, avg, policy, unit, direct, solver) -> CircuitscapeResult:
    """circuitscape.py:499-516: one problem over the whole raster."""
    if unit:
        src = np.where(src != 0, 1.0, src)
    if direct:
        gnd = np.where(gnd != 0, np.inf, gnd)
    sc, gc = np.flatnonzero(src.ravel() != 0), np.flatnonzero(gnd.ravel() != 0)
    prob = {"src_cells": sc, "src_vals": src.ravel()[sc], "gnd_cells": gc, "gnd_vals": gnd.ravel()[gc],
            "check_cell": -1}
    nm, (r,) = solver(g, poly, avg, four, [prob], policy)
    on = nm >= 0
    volt = np.zeros(nm.shape)
    cur = np.zeros(nm.shape)
    volt[on] = r["voltage"][nm[on]]
    cur[on] = r["current"][nm[on]]
    res = CircuitscapeResult(voltage=volt, current=cur, nodemap=nm)
    res.maps["solved"] = bool(r["solved"])
    return res


def circuitscape_advanced(habitat, source, ground, *, habitat_is_resistance: bool = True,
                          ground_is_resistance: bool = True, polygons=None, mask=None, four_neighbors: bool = False,
                          avg_resistances: bool = False, remove_src_or_gnd: str = "keepall",
                          unit_currents: bool = False, direct_grounds: bool = False, reclass: dict | None = None,
                          n_threads: int = 0, tol: float = 1e-13, device=None,
                          problem_solver: str = "auto") -> CircuitscapeResult:
    """Circuitscape's advanced mode on a node graph (drop-in for ``ls.circuit.circuitscape_advanced``,
    circuitscape.py:406-497): sources and grounds per cell (grounds as resistances unless ``ground_is_resistance``
    is False; 0 / inf = direct), short-circuit polygons, a mask, the conflict policy, unit currents and direct
    grounds.  Returns ``voltage`` and ``current`` maps (0 on cells without a node) and the ``nodemap``."""
    del n_threads
    if remove_src_or_gnd not in POLICIES:
        raise ValueError(f"remove_src_or_gnd must be one of {POLICIES}")
    g, poly = _habitat_and_polygons(habitat, habitat_is_resistance, reclass, polygons, mask)
    src = _grid(source, "source")
    gnd = _grid(ground, "ground")
    if src.shape != g.shape or gnd.shape != g.shape:
        raise ValueError("the source and ground must have the habitat's shape")
    src[src == NODATA] = 0.0
    nod = gnd == NODATA
    if ground_is_resistance:
        with np.errstate(divide="ignore"):
            gnd = 1 / gnd
    gnd[nod] = 0.0
    solver = lambda *a: multi_advanced(*a, tol=tol, device=device, problem_solver=problem_solver)  # noqa: E731
    return _advanced(g, poly, src, gnd, four_neighbors, avg_resistances, remove_src_or_gnd, unit_currents,
                     direct_grounds, solver)


def _point_polymap(polymap, point_map: np.ndarray, ids: np.ndarray) -> np.ndarray:
    """create_new_polymap with a point map (circuitscape.py:712-735): focal points and regions become polygons."""
    if polymap is None:
        return point_map.astype(np.int64)
    newpoly = polymap.copy()
    no_regions = len(ids) == len(np.unique(ids))
    jj, ii = np.nonzero(point_map.T)  # column-major
    if no_regions:
        k = polymap.max()
        for r, c in zip(ii, jj):
            if polymap[r, c] == 0:
                newpoly[r, c] = point_map[r, c] + k
        return newpoly
    k = max(polymap.max(), point_map.max())
    for r, c in zip(ii, jj):
        v1, v2 = point_map[r, c], newpoly[r, c]
        if v2 == 0:
            newpoly[r, c] = k + v1
            continue
        if v1 != v2:
            newpoly[newpoly == v2] = v1
    return newpoly


def read_point_strengths(path) -> np.ndarray:
    """Two columns, id and strength (ids from 0 shifted to 1)."""
    t = np.array(_read_rows(path), dtype=np.float64)
    if t.ndim != 2 or t.shape[1] != 2:
        raise ValueError(f"{path} must have exactly 2 columns")
    if t[:, 0].min() == 0:
        t[:, 0] += 1
    return t


def _one_to_all(g, poly, points: FocalPoints, strengths, pairs, one_to_all: bool, four, avg, opts: dict, emit,
                solver) -> CircuitscapeResult:
    """run_onetoall (circuitscape.py:737-851): one advanced-mode problem per focal id; one-to-all injects the id's
    strength at its point with every other point a direct ground, all-to-one the reverse."""
    ny, nx = g.shape
    if pairs is not None:
        keep = np.isin(points.ids, pairs.ids)
        points = FocalPoints(points.rows[keep], points.cols[keep], points.ids[keep])
        if strengths is not None:
            strengths = strengths[np.isin(strengths[:, 0], pairs.ids)]
    rows, cols = points.cells
    cells = rows * nx + cols
    ids = points.ids
    point_map = np.zeros((ny, nx), dtype=np.int64)
    point_map[rows, cols] = ids
    unique_ids, first = np.unique(ids, return_index=True)
    unique_map = np.zeros((ny, nx), dtype=np.int64)
    unique_map[rows[first], cols[first]] = unique_ids
    no_regions = len(ids) == len(unique_ids)
    mode = 0 if pairs is not None and pairs.mode == "include" else 1
    base_poly = _point_polymap(poly, point_map, ids)
    res = np.zeros(len(unique_ids))
    cum = np.zeros((ny, nx)) if opts["cum"] else None
    mx = np.full((ny, nx), NODATA) if opts["max"] else None
    policy = "rmvgnd" if one_to_all else "rmvsrc"

    def problem(i):
        n = int(unique_ids[i])
        pm = point_map.copy()
        newpoly = base_poly
        strength = float(strengths[i, 1]) if strengths is not None else 1.0
        if pairs is not None:
            row = int(np.nonzero(pairs.ids == n)[0][0])
            for j in range(len(pairs.ids)):
                if j != row and pairs.matrix[row, j] == mode:
                    pm[pm == pairs.ids[j]] = 0
            if not no_regions:
                newpoly = _point_polymap(poly, pm, ids)
        smap = None
        if strengths is not None:
            st = strengths[:, 1].copy()
            st[pm[rows, cols] == 0] = 1.0
            smap = np.zeros((ny, nx))
            smap[rows, cols] = st[: len(rows)]
        if pm.sum() == n:
            return None
        if one_to_all:
            src = np.where(unique_map == n, strength, 0.0)
            gnd = np.where(pm == n, 0, pm).astype(np.float64)
            gnd[gnd > 0] = np.inf
        else:
            if smap is not None:
                src = np.where(unique_map == n, 0.0, smap)
            else:
                src = np.where(unique_map != 0, 1.0, 0.0)
                src = np.where(pm == n, 0.0, src)
            gnd = np.where(pm == n, np.inf, 0.0)
        sc, gc = np.flatnonzero(src), np.flatnonzero(gnd)
        return {"n": n, "strength": strength, "poly": newpoly, "src_cells": sc.astype(np.int64),
                "src_vals": src.ravel()[sc], "gnd_cells": gc.astype(np.int64), "gnd_vals": gnd.ravel()[gc],
                "check_cell": int(cells[np.nonzero(ids == n)[0][0]])}

    probs = [(i, problem(i)) for i in range(len(unique_ids))]
    for i, q in probs:
        if q is None:
            res[i] = -1
    todo = [(i, q) for i, q in probs if q is not None]
    # one solve call per graph (focal regions with included pairs rebuild it per point)
    groups: list = []
    for i, q in todo:
        if groups and groups[-1][0] is q["poly"]:
            groups[-1][1].append((i, q))
        else:
            groups.append((q["poly"], [(i, q)]))
    solved = {}
    for pm_, items in groups:
        nm, results = solver(g, np.ascontiguousarray(pm_, dtype=np.int64), avg, four, [q for _, q in items], policy)
        for (i, _), r in zip(items, results):
            solved[i] = (nm, r)
    for i, q in todo:
        nm, r = solved[i]
        n = q["n"]
        if not r["solved"]:
            res[i] = -1
        elif not one_to_all:
            res[i] = 0
        else:
            node = nm[unique_map == n][0]
            val = 0.0 if node < 0 else r["voltage"][node] / q["strength"]
            res[i] = -1 if val == 0 else val
        on = nm >= 0
        volt = np.zeros((ny, nx))
        volt[on] = r["voltage"][nm[on]]
        cur = np.zeros((ny, nx))
        cur[on] = r["current"][nm[on]]
        if opts["focal_zero"]:
            cur[np.isin(nm, r["active"])] = 0.0
        if cum is not None:
            cum += cur
        if mx is not None:
            np.maximum(mx, cur, out=mx)
        emit(n, volt if opts["volt_maps"] else None, cur if opts["cur_maps"] else None)
    if cum is not None:
        cum[cum < NODATA] = NODATA
    if mx is not None:
        mx[mx < NODATA] = NODATA
    return CircuitscapeResult(resistances=np.column_stack([unique_ids.astype(np.float64), res]), cum_current=cum,
                              max_current=mx)


def _habitat_and_polygons(habitat, habitat_is_resistance, reclass, polygons, mask):
    g = habitat_conductance(_grid(habitat, "habitat"), is_resistance=habitat_is_resistance, reclass=reclass)
    poly = None
    if polygons is not None:
        pm = _grid(polygons, "polygons")
        if pm.shape != g.shape:
            raise ValueError("the polygons must have the habitat's shape")
        pm[pm == NODATA] = 0
        if not np.all(pm == np.round(pm)):
            raise ValueError("the polygon raster must hold integer ids")
        poly = pm.astype(np.int64)
    if mask is not None:
        m = _grid(mask, "mask")
        if m.shape != g.shape:
            raise ValueError("the mask must have the habitat's shape")
        m[m == NODATA] = 0
        g = g * np.where(m > 0, 1.0, 0.0)
        if g.sum() == 0:
            raise ValueError("Mask file deleted everything!")
    return g, poly


def circuitscape_one_to_all(habitat, points, *, all_to_one: bool = False, habitat_is_resistance: bool = True,
                            polygons=None, mask=None, four_neighbors: bool = False, avg_resistances: bool = False,
                            included_pairs=None, strengths=None, voltage_maps: bool = False,
                            current_maps: bool = False, cum_map: bool = False, max_map: bool = False,
                            set_focal_node_currents_to_zero: bool = False, reclass: dict | None = None,
                            n_threads: int = 0, tol: float = 1e-13, device=None,
                            problem_solver: str = "auto") -> CircuitscapeResult:
    """Circuitscape's one-to-all (or, with ``all_to_one``, all-to-one) mode on rasters (drop-in for
    ``ls.circuit.circuitscape_one_to_all``, circuitscape.py:854-953).  ``resistances`` has the ids in its first
    column and each point's result in the second (one-to-all: the voltage at the point per unit strength, -1 when
    nothing was solved); ``maps`` keys ``("voltage", id)`` / ``("current", id)``."""
    del n_threads
    g, poly = _habitat_and_polygons(habitat, habitat_is_resistance, reclass, polygons, mask)
    if not isinstance(points, FocalPoints):
        pm = _grid(points, "points")
        if pm.shape != g.shape:
            raise ValueError("the points must have the habitat's shape")
        points = _points_from_map(pm)
    if included_pairs is not None and not isinstance(included_pairs, IncludedPairs):
        included_pairs = read_included_pairs(included_pairs)
    if strengths is not None and isinstance(strengths, (str, os.PathLike)):
        strengths = read_point_strengths(strengths)
    maps: dict = {}

    def emit(n, volt, cur):
        if volt is not None:
            maps[("voltage", n)] = volt
        if cur is not None:
            maps[("current", n)] = cur

    opts = {"volt_maps": voltage_maps, "cur_maps": current_maps, "cum": current_maps or cum_map, "max": max_map,
            "focal_zero": set_focal_node_currents_to_zero}
    solver = lambda *a: multi_advanced(*a, tol=tol, device=device, problem_solver=problem_solver)  # noqa: E731
    r = _one_to_all(g, poly, points, None if strengths is None else np.asarray(strengths, dtype=np.float64),
                    included_pairs, not all_to_one, four_neighbors, avg_resistances, opts, emit, solver)
    r.maps = maps
    return r


def _read_list3(path) -> np.ndarray:
    return np.array(_read_rows(path), dtype=np.float64).reshape(-1, 3)


def _source_and_ground(source_path, ground_path, meta: RasterMeta, ground_is_res: bool):
    """read_source_and_ground_maps (circuitscape.py:1230-1258)."""
    kind = file_type(ground_path)
    if kind in ("aagrid", "geotiff"):
        gnd = read_polymap(ground_path, meta, nodata_as=None)
    elif kind == "list":
        pts = _read_list3(ground_path)
        gnd = np.full((meta.nrows, meta.ncols), NODATA)
        i, j = _list_cells(pts, meta)
        gnd[i - 1, j - 1] = pts[:, 0]
    else:
        raise ValueError("Cannot recognise file type.")
    kind = file_type(source_path)
    if kind in ("aagrid", "geotiff"):
        src = read_polymap(source_path, meta)
        src[src == NODATA] = 0.0
    elif kind == "list":
        pts = _read_list3(source_path)
        src = np.zeros((meta.nrows, meta.ncols))
        i, j = _list_cells(pts, meta)
        src[i - 1, j - 1] = pts[:, 0]
    else:
        raise ValueError("Cannot recognize file type.")
    nod = gnd == NODATA
    if ground_is_res:
        with np.errstate(divide="ignore"):
            gnd = 1 / gnd
    gnd[nod] = 0.0
    return src, gnd


# --- INI files (circuitscape.py:977-1213) -------------------------------------------------------------------------

DEFAULTS = {
    "data_type": "raster", "scenario": "not entered", "connect_four_neighbors_only": "False",
    "connect_using_avg_resistances": "False", "use_polygons": "False", "use_mask": "False", "mask_file": "None",
    "habitat_file": "(Browse for a resistance file)", "habitat_map_is_resistances": "True",
    "use_included_pairs": "False", "included_pairs_file": "(Browse for a file with pairs to include or exclude)",
    "point_file": "(Browse for file with locations of focal points or regions)", "use_reclass_table": "False",
    "reclass_file": "(Browse for file with reclassification data)", "write_cur_maps": "False",
    "write_volt_maps": "False", "write_cum_cur_map_only": "False", "write_max_cur_maps": "False",
    "set_null_currents_to_nodata": "False", "set_null_voltages_to_nodata": "False",
    "set_focal_node_currents_to_zero": "False", "log_transform_maps": "False",
    "polygon_file": "(Browse for a short-circuit region file)",
    "source_file": "(Browse for a current source file)", "ground_file": "(Browse for a ground point file)",
    "ground_file_is_resistances": "True", "use_unit_currents": "False", "use_direct_grounds": "False",
    "remove_src_or_gnd": "keepall", "use_variable_source_strengths": "False", "variable_source_file": "None",
    "output_file": "(Choose a base name for output files)", "write_as_tif": "False",
}
SCENARIOS = {"pairwise": "pairwise", "Pairwise": "pairwise", "advanced": "advanced", "Advanced": "advanced",
             "one-to-all": "one-to-all", "one_to_all": "one-to-all", "all-to-one": "all-to-one",
             "all_to_one": "all-to-one"}


def parse_config(path) -> dict:
    """Every line but ``[section]`` ones split at its first ``=`` (key right-stripped, value stripped)."""
    cfg = {}
    with open(path, encoding="utf-8") as f:
        for line in f:
            if line.startswith("["):
                continue
            key, sep, value = line.partition("=")
            if sep:
                cfg[key.rstrip()] = value.strip()
    return cfg


def _unset(path: str) -> bool:
    return path == "" or path == "None" or path.startswith("(")


def _flag(cfg, key) -> bool:
    v = cfg[key]
    if v in TRUELIST:
        return True
    if v in FALSELIST:
        return False
    raise ValueError(f'{key} = "{v}": expected True or False')


def _resolve(name: str, base: Path) -> Path:
    p = Path(name)
    if p.is_absolute() or p.exists():
        return p
    q = base / p
    return q if q.exists() else p


def _write_grid(prefix: str, values: np.ndarray, meta: RasterMeta) -> None:
    """An ESRI ASCII grid (Circuitscape's header, NoData -9999, NaN written as NoData); values as Python writes
    floats (repr), so that reading the file back gives the same doubles."""
    out = np.where(np.isnan(values), NODATA, values)
    with open(prefix + ".asc", "w", encoding="utf-8") as f:
        f.write(f"ncols         {meta.ncols}\nnrows         {meta.nrows}\n")
        f.write(f"xllcorner     {meta.xllcorner!r}\nyllcorner     {meta.yllcorner!r}\n")
        f.write(f"cellsize      {meta.cellsize!r}\nNODATA_value  -9999\n")
        for row in out:
            f.write(" ".join(repr(float(v)) for v in row) + "\n")


def _write_matrix(path: str, a: np.ndarray) -> None:
    with open(path, "w", encoding="utf-8") as f:
        for row in np.atleast_2d(a):
            f.write(" ".join(repr(float(v)) for v in row) + "\n")


def _output_prefix(cfg) -> str:
    out = cfg["output_file"]
    if _unset(out):
        raise ValueError("output_file is not set")
    if _flag(cfg, "write_as_tif"):
        raise NotImplementedError("write_as_tif: only ESRI ASCII grids are written")
    Path(out).parent.mkdir(parents=True, exist_ok=True)
    return out.split(".out")[0]


def _write_outputs(cfg, scenario: str, result: CircuitscapeResult, meta: RasterMeta) -> None:
    """Circuitscape's output files (circuitscape.py:1261-1286): the configuration in output_file, the maps next
    to it (the per-pair and per-point maps are written as they are computed), the resistance matrices."""
    prefix = _output_prefix(cfg)
    with open(cfg["output_file"], "w", encoding="utf-8") as f:
        for k, v in cfg.items():
            f.write(f"{k} = {v}\n")
    if scenario == "advanced":
        if _flag(cfg, "write_volt_maps"):
            _write_grid(prefix + "_voltmap", result.voltage, meta)
        if _flag(cfg, "write_cur_maps") or _flag(cfg, "write_cum_cur_map_only"):
            _write_grid(prefix + "_curmap", result.current, meta)
        return
    if result.cum_current is not None:
        _write_grid(prefix + "_cum_curmap", result.cum_current, meta)
    if result.max_current is not None:
        _write_grid(prefix + "_max_curmap", result.max_current, meta)
    if scenario == "pairwise":
        r = result.resistances
        _write_matrix(prefix + "_resistances.out", r)
        fp = r[1:, 0]
        three = [(fp[i], fp[j], r[j + 1, i + 1]) for i in range(len(fp)) for j in range(i + 1, len(fp))]
        _write_matrix(prefix + "_resistances_3columns.out", np.array(three).reshape(-1, 3))


def circuitscape_ini(path, *, write_outputs: bool = True, tol: float = 1e-13, device=None,
                     pair_solver: str = "auto", problem_solver: str = "auto", _solver=None) -> CircuitscapeResult:
    """Run a Circuitscape INI file on rasters (scenarios pairwise, advanced, one-to-all and all-to-one), as the
    reference's ``circuitscape_ini`` does (circuitscape.py:1039-1213); paths are read from the working directory, or
    else next to the INI file.  ``maps`` are keyed as Circuitscape names its files (``voltmap_<id1>_<id2>``,
    ``curmap_<id>``...).  With ``write_outputs`` the maps go next to ``output_file`` as Circuitscape names them
    (``<base>_voltmap``, ``<base>_curmap``..., ESRI ASCII grids; the per-pair and per-point maps are then written
    instead of kept in ``maps``), the resistances to ``<base>_resistances.out`` and the configuration to
    ``output_file``.  ``_solver``
    replaces the GPU solve of the advanced-mode scenarios (a callable with the signature of multi_advanced without
    its keywords)."""
    path = Path(path)
    base = path.resolve().parent
    cfg = {**DEFAULTS, **parse_config(path)}
    if cfg["data_type"] not in ("raster", "Raster"):
        raise NotImplementedError(f'data_type = "{cfg["data_type"]}": only rasters are supported')
    scenario = SCENARIOS.get(cfg["scenario"])
    if scenario is None:
        raise ValueError(f'scenario = "{cfg["scenario"]}" is not one of {sorted(set(SCENARIOS.values()))}')
    for key in ("low_memory_mode", "preemptive_memory_release"):
        if cfg.get(key, "False") in TRUELIST:
            raise ValueError(f"{key} is not implemented in Circuitscape.jl; remove it or set it to False")

    def need(key):
        if _unset(cfg[key]):
            raise ValueError(f"{key} is not set")
        p = _resolve(cfg[key], base)
        if not p.is_file():
            raise FileNotFoundError(f'{key} = "{cfg[key]}" does not exist')
        return p

    cells, meta = read_raster(need("habitat_file"))
    reclass = read_reclass_table(need("reclass_file")) if _flag(cfg, "use_reclass_table") else None
    g = habitat_conductance(cells, is_resistance=_flag(cfg, "habitat_map_is_resistances"), reclass=reclass)
    poly = None
    if _flag(cfg, "use_polygons"):
        poly = read_polymap(need("polygon_file"), meta, integer=True).astype(np.int64)
    if _flag(cfg, "use_mask"):
        m = read_polymap(need("mask_file"), meta)
        g = g * np.where(m > 0, 1.0, 0.0)
        if g.sum() == 0:
            raise ValueError("Mask file deleted everything!")
    four = _flag(cfg, "connect_four_neighbors_only")
    avg = _flag(cfg, "connect_using_avg_resistances")
    policy = cfg["remove_src_or_gnd"]
    if policy == "not entered":  # Circuitscape 4's default
        policy = "keepall"
    if policy not in POLICIES:
        raise ValueError(f"remove_src_or_gnd must be one of {POLICIES}")
    solver = _solver if _solver is not None else (
        lambda *a: multi_advanced(*a, tol=tol, device=device, problem_solver=problem_solver))

    prefix = _output_prefix(cfg) if write_outputs else None
    if scenario == "advanced":
        src, gnd = _source_and_ground(need("source_file"), need("ground_file"), meta,
                                      _flag(cfg, "ground_file_is_resistances"))
        result = _advanced(g, poly, src, gnd, four, avg, policy, _flag(cfg, "use_unit_currents"),
                           _flag(cfg, "use_direct_grounds"), solver)
        if write_outputs:
            _write_outputs(cfg, scenario, result, meta)
        return result

    points = read_point_map(need("point_file"), meta)
    pairs = read_included_pairs(need("included_pairs_file")) if _flag(cfg, "use_included_pairs") else None
    maps: dict = {}
    if scenario != "pairwise":
        strengths = (read_point_strengths(need("variable_source_file"))
                     if _flag(cfg, "use_variable_source_strengths") else None)
        cum_only = _flag(cfg, "write_cum_cur_map_only")
        opts = {"volt_maps": _flag(cfg, "write_volt_maps"),
                # the advanced-mode kernel writes every point's current map with write_cum_cur_map_only too
                "cur_maps": _flag(cfg, "write_cur_maps") or cum_only,
                "cum": _flag(cfg, "write_cur_maps") or cum_only, "max": _flag(cfg, "write_max_cur_maps"),
                "focal_zero": _flag(cfg, "set_focal_node_currents_to_zero")}

        def emit_point(n, volt, curmap):
            for kind, grid in (("voltmap", volt), ("curmap", curmap)):
                if grid is None:
                    continue
                if write_outputs:
                    _write_grid(f"{prefix}_{kind}_{n}", grid, meta)
                else:
                    maps[f"{kind}_{n}"] = grid

        result = _one_to_all(g, poly, points, strengths, pairs, scenario == "one-to-all", four, avg, opts,
                             emit_point, solver)
        result.maps = maps
        if write_outputs:
            _write_outputs(cfg, scenario, result, meta)
        return result

    points, excluded = _apply_included_pairs(points, pairs)
    cur, cum_only = _flag(cfg, "write_cur_maps"), _flag(cfg, "write_cum_cur_map_only")
    o = PairOptions(volt_maps=_flag(cfg, "write_volt_maps"), cur_maps=cur and not cum_only, cum=cur or cum_only,
                    max=_flag(cfg, "write_max_cur_maps"), focal_zero=_flag(cfg, "set_focal_node_currents_to_zero"),
                    null_currents=_flag(cfg, "set_null_currents_to_nodata"),
                    null_voltages=_flag(cfg, "set_null_voltages_to_nodata"),
                    log_transform=_flag(cfg, "log_transform_maps"))
    ids = np.unique(points.ids) if points.has_regions else points.ids

    def emit(ci, cj, volt, curmap):
        name = f"_{int(ids[ci])}_{int(ids[cj])}"
        for kind, grid in (("voltmap", volt), ("curmap", curmap)):
            if grid is None:
                continue
            if write_outputs:
                _write_grid(f"{prefix}_{kind}{name}", grid, meta)
            else:
                maps[kind + name] = grid

    res, cum, mx, stats = _run_pairwise(g, poly, points, excluded, four, avg, o, emit, tol, device, pair_solver)
    result = CircuitscapeResult(resistances=res, cum_current=cum, max_current=mx, maps=maps, stats=stats)
    if write_outputs:
        _write_outputs(cfg, scenario, result, meta)
    return result
