"""Oracle (test infrastructure only): numpy restatement of the reference's
quadtree mesh and quadtree global step.  Used by tests/ to check the
library's quadtree path; never part of the product.

  * generate_quadtree_mesh  func_quadtree/GenerateQuadtreeMesh.m:17-115 with
    funMarkEdge.m, funMarkInside.m, refinement/QrefineR.m and
    refinement/provideGeometricData.m (red refinement, 1-irregular rule,
    hanging nodes in element slots 5-8);
  * subpb2_quadtree         func_quadtree/Subpb2Quadtree.m:41-347 (2x2 Gauss
    points, hanging-node shape functions, Dirichlet nodes fixed to U, the
    duals multiplied by zero as the reference does) with scipy's sparse
    direct solve in place of MATLAB's backslash;
  * nodal_strain_quadtree   func_quadtree/funGlobalNodalStrainQuadtree.m:33-203
    Gauss-point strains (slots 5-8 ignored, as the reference zeroes them);
    the reference then interpolates them to the nodes with
    scatteredInterpolant('linear') -- parity unpinned -- this restatement
    extrapolates each element's 2x2 Gauss values to its corners and averages
    over the elements at a node (the rule of funGlobal_NodalStrainAvg.m);
  * graph_fill              refill of flagged nodes; the reference uses
    scatteredInterpolant('natural') (LocalICGN.m:144-161,
    Subpb1Quadtree.m:194-199) -- parity unpinned -- this restatement solves
    the graph Laplacian of the mesh edges with the good nodes fixed.
Node and element indices are 1-based like the reference; 0 = empty slot.
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------- marking
def mark_edge(coords, elems, mask, min_size):
    """funMarkEdge.m: elements whose bounding box spans both mask values and
    whose smaller side exceeds min_size.  mask is (H, W), Img(x, y) =
    mask[y-1, x-1]."""
    out = np.zeros(len(elems), bool)
    for e, el in enumerate(elems):
        xs = coords[el[:4] - 1, 0]
        ys = coords[el[:4] - 1, 1]
        x0, x1, y0, y1 = int(xs.min()), int(xs.max()), int(ys.min()), int(ys.max())
        blk = mask[y0 - 1:y1, x0 - 1:x1]
        rng = blk.max() - blk.min()
        size = min(abs(x1 - x0), abs(y1 - y0))
        out[e] = rng > 0 and size > min_size
    return out


def mark_inside(coords, elems, mask):
    """funMarkInside.m: elements with less than half their box in the mask
    (threshold 0.5 * dx * dy, as written)."""
    inside = np.zeros(len(elems), bool)
    for e, el in enumerate(elems):
        xs = coords[el[:4] - 1, 0]
        ys = coords[el[:4] - 1, 1]
        x0, x1, y0, y1 = int(xs.min()), int(xs.max()), int(ys.min()), int(ys.max())
        if mask[y0 - 1:y1, x0 - 1:x1].sum() < 0.5 * (x1 - x0) * (y1 - y0):
            inside[e] = True
    return inside


# ---------------------------------------------------------------- QrefineR
def _geometric_data(irregular, elems):
    """provideGeometricData.m: sorted unique edges; the three edges of each
    irregular triple (parent, half 1, half 2) and the four of each element."""
    # reshape(elements(:,[1:3,2:3,1]),[],2): column-major stacking of columns
    ed3 = np.stack([irregular[:, [0, 1, 2]].T.reshape(-1), irregular[:, [1, 2, 0]].T.reshape(-1)],
                   axis=1) if len(irregular) else np.zeros((0, 2), np.int64)
    ed4 = np.stack([elems[:, [0, 1, 2, 3]].T.reshape(-1), elems[:, [1, 2, 3, 0]].T.reshape(-1)], axis=1)
    edges = np.concatenate([ed3, ed4])
    edge2nodes, ie = np.unique(np.sort(edges, axis=1), axis=0, return_inverse=True)
    ie = ie.reshape(-1)
    n3 = len(ed3)
    irr2edges = ie[:n3].reshape(3, -1).T if n3 else np.zeros((0, 3), np.int64)
    el2edges = ie[n3:].reshape(4, -1).T
    return edge2nodes, irr2edges, el2edges


def qrefine_r(coords, elems, irregular, marked):
    """QrefineR.m (no boundary lists): returns coords, elements (n x 4),
    irregular (n x 3: sorted parent edge, hanging node)."""
    nE = len(elems)
    edge2nodes, irr2edges, el2edges = _geometric_data(irregular, elems)
    e2n = np.zeros(len(edge2nodes), np.int64)
    e2n[el2edges[marked].reshape(-1)] = 1
    if len(irregular):
        e2n[irr2edges[:, 0]] = 1
    first = True
    swap = np.zeros(0, np.int64)
    kdx = np.ones(1)
    while first or len(kdx) or len(swap):
        first = False
        me = e2n[el2edges]
        s = np.abs(me).sum(axis=1)
        kdx = np.nonzero((s < 4) & ((s > 2) | (me.min(axis=1) < 0)))[0]
        sub = el2edges[kdx]
        e2n[sub[me[kdx] == 0]] = 1
        if len(irregular):
            me3 = e2n[irr2edges]
            flag = irr2edges[np.any(me3[:, 1:] != 0, axis=1), 0]
            swap = flag[e2n[flag] != -1]
            e2n[swap] = -1
        else:
            swap = np.zeros(0, np.int64)
    if len(irregular):
        e2n[irr2edges[:, 0]] = -1
    idx = e2n > 0
    nn0 = len(coords)
    e2n[idx] = nn0 + 1 + np.arange(int(idx.sum()))
    coords = np.concatenate([coords, (coords[edge2nodes[idx, 0] - 1] + coords[edge2nodes[idx, 1] - 1]) / 2])
    if len(irregular):
        e2n[irr2edges[:, 0]] = irregular[:, 2]
    newNodes = e2n[el2edges]                                   # nE x 4
    reftyp = (newNodes != 0).astype(np.int64) @ (2 ** np.arange(4))
    none = reftyp < 15
    red = reftyp == 15
    ridx = np.nonzero(red)[0]
    mid = np.zeros(nE, np.int64)
    mid[ridx] = len(coords) + 1 + np.arange(len(ridx))
    coords = np.concatenate([coords, (coords[elems[ridx, 0] - 1] + coords[elems[ridx, 1] - 1] +
                                      coords[elems[ridx, 2] - 1] + coords[elems[ridx, 3] - 1]) / 4])
    cnt = np.where(none, 1, 4)
    start = np.concatenate([[0], np.cumsum(cnt)])
    new = np.zeros((start[-1], 4), np.int64)
    new[start[:-1][none]] = elems[none]
    e, nn, m = elems[ridx], newNodes[ridx], mid[ridx]
    s0 = start[:-1][red]
    new[s0 + 0] = np.stack([e[:, 0], nn[:, 0], m, nn[:, 3]], axis=1)
    new[s0 + 1] = np.stack([e[:, 1], nn[:, 1], m, nn[:, 0]], axis=1)
    new[s0 + 2] = np.stack([e[:, 2], nn[:, 2], m, nn[:, 1]], axis=1)
    new[s0 + 3] = np.stack([e[:, 3], nn[:, 3], m, nn[:, 2]], axis=1)
    # irregularity data: partially refined elements, in MATLAB find() order
    kdx = np.nonzero((reftyp > 0) & (reftyp < 15))[0]
    sub = newNodes[kdx]
    jj, ii = np.nonzero(sub.T)                                 # column-major
    edx = el2edges[kdx[ii], jj]
    irr = [np.concatenate([edge2nodes[edx], sub[ii, jj][:, None]], axis=1)]
    if len(irregular):
        nn2 = e2n[irr2edges[:, 1:3]]
        k2 = np.nonzero(nn2.sum(axis=1) != 0)[0]
        sub2 = nn2[k2]
        jj, ii = np.nonzero(sub2.T)
        edx = irr2edges[k2[ii], jj + 1]
        irr.append(np.concatenate([edge2nodes[edx], sub2[ii, jj][:, None]], axis=1))
    newIrr = np.concatenate(irr).astype(np.int64) if irr else np.zeros((0, 3), np.int64)
    return coords, new, newIrr


def generate_quadtree_mesh(coords, elems, mask, step, min_size=2):
    """GenerateQuadtreeMesh.m:17-115.  coords (n x 2), elems (ne x 4, 1-based)
    of the uniform mesh; mask (H, W) ImgRefMask.  Returns coords, elements
    (ne x 8; slots 5-8 hanging nodes on edges 2-3, 3-4, 4-1, 1-2), dirichlet
    (sorted node numbers)."""
    c = np.asarray(coords, np.float64).copy()
    el = np.asarray(elems, np.int64).copy()
    irr = np.zeros((0, 3), np.int64)
    while True:
        mk = np.nonzero(mark_edge(c, el, mask, 2 * min_size))[0]
        c, el, irr = qrefine_r(c, el, irr, mk)
        if len(mk) == 0:
            break
    E = np.zeros((len(el), 8), np.int64)
    E[:, :4] = el
    pairs = [((0, 1), 7), ((1, 2), 4), ((2, 3), 5), ((3, 0), 6),
             ((1, 0), 7), ((2, 1), 4), ((3, 2), 5), ((0, 3), 6)]
    lut = {}
    for (a, b), slot in pairs:
        for k in range(len(el) - 1, -1, -1):   # first match wins
            lut[((int(el[k, a]), int(el[k, b])), slot)] = k
    for a, b, h in irr.tolist():
        for (pa, pb), slot in pairs:
            k = lut.get(((a, b), slot))
            if k is not None:
                E[k, slot] = h
    keep = ~mark_inside(c, E, mask)
    E = E[keep]
    # Dirichlet nodes: refined elements, elements at the ROI border, 2 rings
    d13 = np.hypot(c[E[:, 0] - 1, 0] - c[E[:, 2] - 1, 0], c[E[:, 0] - 1, 1] - c[E[:, 2] - 1, 1])
    refined = d13 < 0.99 * np.sqrt(2) * step
    xmin, xmax = coords[:, 0].min(), coords[:, 0].max()
    ymin, ymax = coords[:, 1].min(), coords[:, 1].max()
    border = ((c[E[:, 0] - 1, 0] < xmin + 1.01 * step) | (c[E[:, 2] - 1, 0] > xmax - 1.01 * step) |
              (c[E[:, 0] - 1, 1] < ymin + 1.01 * step) | (c[E[:, 2] - 1, 1] > ymax - 1.01 * step))
    mark = np.unique(E[refined | border])
    mark = mark[mark != 0]
    for _ in range(2):
        hit = np.isin(E, mark) & (E != 0)
        sel = hit.any(axis=1)
        mark = np.unique(E[sel])
        mark = mark[mark != 0]
    return c, E, mark


def uniform_mesh(x0, y0, M, N):
    """MeshSetUp.m:23-39 node list (x fastest) and elements."""
    coords = np.stack([np.asarray(x0, np.float64).reshape(-1), np.asarray(y0, np.float64).reshape(-1)], 1)
    el = []
    for j in range(1, N):
        for i in range(1, M):
            el.append([(j - 1) * M + i, (j - 1) * M + i + 1, j * M + i + 1, j * M + i])
    return coords, np.asarray(el, np.int64)


# ------------------------------------------------------- shape functions
def _shape(ksi, eta, d):
    """N1..N8 and their ksi/eta derivatives (Subpb2Quadtree.m:152-160 and the
    funDN* helpers); d = presence of slots 5-8."""
    d5, d6, d7, d8 = d
    N5 = d5 * 0.5 * (1 + ksi) * (1 - abs(eta))
    N6 = d6 * 0.5 * (1 + eta) * (1 - abs(ksi))
    N7 = d7 * 0.5 * (1 - ksi) * (1 - abs(eta))
    N8 = d8 * 0.5 * (1 - eta) * (1 - abs(ksi))
    N1 = (1 - ksi) * (1 - eta) * 0.25 - 0.5 * (N7 + N8)
    N2 = (1 + ksi) * (1 - eta) * 0.25 - 0.5 * (N8 + N5)
    N3 = (1 + ksi) * (1 + eta) * 0.25 - 0.5 * (N5 + N6)
    N4 = (1 - ksi) * (1 + eta) * 0.25 - 0.5 * (N6 + N7)
    sg = np.sign
    d5k, d5e = d5 * 0.5 * (1 - abs(eta)), d5 * 0.5 * (1 + ksi) * sg(-eta)
    d6k, d6e = d6 * 0.5 * (1 + eta) * sg(-ksi), d6 * 0.5 * (1 - abs(ksi))
    d7k, d7e = d7 * 0.5 * (-1) * (1 - abs(eta)), d7 * 0.5 * (1 - ksi) * sg(-eta)
    d8k, d8e = d8 * 0.5 * (1 - eta) * sg(-ksi), d8 * 0.5 * (-1) * (1 - abs(ksi))
    dk = [-0.25 * (1 - eta) - 0.5 * (d7k + d8k), 0.25 * (1 - eta) - 0.5 * (d8k + d5k),
          0.25 * (1 + eta) - 0.5 * (d5k + d6k), -0.25 * (1 + eta) - 0.5 * (d6k + d7k),
          d5k, d6k, d7k, d8k]
    de = [-0.25 * (1 - ksi) - 0.5 * (d7e + d8e), -0.25 * (1 + ksi) - 0.5 * (d8e + d5e),
          0.25 * (1 + ksi) - 0.5 * (d5e + d6e), 0.25 * (1 - ksi) - 0.5 * (d6e + d7e),
          d5e, d6e, d7e, d8e]
    return np.array([N1, N2, N3, N4, N5, N6, N7, N8]), np.array(dk), np.array(de)


_G2 = (-1 / np.sqrt(3), 1 / np.sqrt(3))


def _element_gp(c, el):
    """(N, dN/dx, dN/dy, J*w) at the 2x2 Gauss points of one element
    (ndgrid order: ksi fastest)."""
    d = [1.0 if el[s] else 0.0 for s in range(4, 8)]
    pts = np.array([c[n - 1] if n else (0.0, 0.0) for n in el])
    out = []
    for eta in _G2:
        for ksi in _G2:
            N, dk, de = _shape(ksi, eta, d)
            J11, J12 = dk @ pts[:, 0], dk @ pts[:, 1]
            J21, J22 = de @ pts[:, 0], de @ pts[:, 1]
            det = J11 * J22 - J12 * J21
            dx = (J22 * dk - J12 * de) / det
            dy = (-J21 * dk + J11 * de) / det
            out.append((N, dx, dy, det))
    return out


def subpb2_quadtree(coords, elems, dirichlet, beta, mu, U, F):
    """Subpb2Quadtree.m with alpha = 0 and GaussPtOrder 2.  U (2n), F (4n);
    the reference multiplies udual and vdual by zero (W = 0*udual,
    v = 0*vdual), so they are not arguments.  Returns Uhat (2n): Dirichlet
    nodes keep U, nodes in no element get 0."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    n = len(coords)
    rows, cols, vals = [], [], []
    b = np.zeros(2 * n)
    for el in elems:
        slots = [s for s in range(8) if el[s]]
        Ke = np.zeros((8, 8))
        bu = np.zeros(8)
        bv = np.zeros(8)
        for N, dx, dy, J in _element_gp(coords, el):
            Ke += J * (beta * (np.outer(dx, dx) + np.outer(dy, dy)) + mu * np.outer(N, N))
            uu = sum(N[s] * U[2 * (el[s] - 1)] for s in slots)
            vv = sum(N[s] * U[2 * (el[s] - 1) + 1] for s in slots)
            for s in slots:
                k = el[s] - 1
                bu[s] += J * (beta * (dx[s] * F[4 * k] + dy[s] * F[4 * k + 2]) + mu * N[s] * uu)
                bv[s] += J * (beta * (dx[s] * F[4 * k + 1] + dy[s] * F[4 * k + 3]) + mu * N[s] * vv)
        for a in slots:
            b[2 * (el[a] - 1)] += bu[a]
            b[2 * (el[a] - 1) + 1] += bv[a]
            for c2 in slots:
                rows.append(el[a] - 1)
                cols.append(el[c2] - 1)
                vals.append(Ke[a, c2])
    K = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    involved = np.zeros(n, bool)
    involved[elems[elems != 0] - 1] = True
    dmask = np.zeros(n, bool)
    dmask[np.asarray(dirichlet, np.int64) - 1] = True
    free = involved & ~dmask
    Uh = np.zeros(2 * n)
    for f in range(2):
        x = np.zeros(n)
        x[dmask] = U[f::2][dmask]
        rhs = b[f::2] - K @ x
        fi = np.nonzero(free)[0]
        x[fi] = spl.spsolve(K[fi][:, fi].tocsc(), rhs[fi])
        Uh[f::2] = x
    return Uh


def nodal_strain_quadtree(coords, elems, U):
    """Gauss-point strains of funGlobalNodalStrainQuadtree.m (Q4 corners
    only) extrapolated to each element's corners and averaged per node;
    output per node [du/dx du/dy dv/dx dv/dy] in the [F11 F21 F12 F22]
    slots as the reference writes them.  Nodes in no element get 0."""
    n = len(coords)
    acc = np.zeros((n, 4))
    cnt = np.zeros(n)
    # corner (ksi, eta) of local nodes 1..4 and the Gauss points' positions
    cks = np.array([(-1, -1), (1, -1), (1, 1), (-1, 1)], np.float64)
    g = 1 / np.sqrt(3)
    for el in elems:
        e4 = np.array([el[0], el[1], el[2], el[3], 0, 0, 0, 0])
        gps = []
        vals = []
        for N, dx, dy, J in _element_gp(coords, e4):
            u = np.array([U[2 * (e4[s] - 1)] for s in range(4)])
            v = np.array([U[2 * (e4[s] - 1) + 1] for s in range(4)])
            vals.append([dx[:4] @ u, dy[:4] @ u, dx[:4] @ v, dy[:4] @ v])
        vals = np.array(vals)                                   # 4 GPs x 4
        # bilinear in (ksi, eta) through the 4 Gauss values, evaluated at the
        # corners: GP order ksi fastest: (-g,-g), (g,-g), (-g,g), (g,g)
        for a in range(4):
            k, e = cks[a] / g
            w = np.array([(1 - k) * (1 - e), (1 + k) * (1 - e), (1 - k) * (1 + e), (1 + k) * (1 + e)]) / 4
            acc[el[a] - 1] += w @ vals
            cnt[el[a] - 1] += 1
    out = np.zeros((n, 4))
    nz = cnt > 0
    out[nz] = acc[nz] / cnt[nz, None]
    return out.reshape(-1)


def mesh_edges(elems):
    """Node pairs along each element's boundary (corners and hanging nodes in
    order 1-8-2-5-3-6-4-7), unique, 1-based."""
    order = [0, 7, 1, 4, 2, 5, 3, 6]
    ed = set()
    for el in elems:
        ring = [el[s] for s in order if el[s]]
        for a, b in zip(ring, ring[1:] + ring[:1]):
            ed.add((min(a, b), max(a, b)))
    return np.array(sorted(ed), np.int64)


FILL_TETHER = 1e-6


def graph_fill(n, edges, vals, bad):
    """Harmonic refill: values at bad nodes solve (L + t I) x = (adjacency x)
    over the mesh-edge graph L with the good nodes fixed; the tether
    t = 1e-6 ties bad nodes without a path to a good node (hole nodes in no
    element) to 0.  vals (n x nf)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    vals = np.array(vals, np.float64, copy=True).reshape(n, -1)
    bad = np.asarray(bad, bool)
    a, b = edges[:, 0] - 1, edges[:, 1] - 1
    L = sp.coo_matrix((np.ones(2 * len(a)), (np.r_[a, b], np.r_[b, a])), shape=(n, n)).tocsr()
    deg = np.asarray(L.sum(axis=1)).reshape(-1)
    bi = np.nonzero(bad)[0]
    if len(bi) == 0:
        return vals
    A = (sp.diags(deg) - L)[bi][:, bi].tocsc()
    good = ~bad
    for f in range(vals.shape[1]):
        x = np.where(good, vals[:, f], 0.0)
        rhs = (L @ x)[bi]
        vals[bi, f] = spl.spsolve(A + FILL_TETHER * sp.identity(len(bi), format="csc"), rhs)
    return vals


# ------------------------------------------------------------- frame
def icgn_flags(it, floor=np.nan):
    """LocalICGN.m:117-131 (floor NaN) / Subpb1Quadtree.m:172-181 (floor 20):
    returns the bad mask and the reference's bad-point count."""
    it = np.asarray(it)
    b1 = (it < 0) | (it > 99)
    g = it[~b1].astype(np.float64)
    m = g.mean() if len(g) else np.nan
    sd = g.std(ddof=1) if len(g) > 1 else (0.0 if len(g) == 1 else np.nan)
    thr = m + 0.15 * sd
    if not np.isnan(floor):
        thr = np.fmax(thr, floor)
    bad = b1 | (it > thr)
    return bad, int(b1.sum() - (it == 102).sum())


def interp_uniform(xs, ys, fields, pts):
    """Bilinear interpolation of fields (nf x ny x nx on the uniform node grid
    xs, ys) at pts (n x 2) -- stands in for scatteredInterpolant('linear'),
    GenerateQuadtreeMesh.m:124-130 (parity unpinned)."""
    x, y = pts[:, 0], pts[:, 1]
    i = np.clip(np.searchsorted(xs, x, side="right") - 1, 0, len(xs) - 2)
    j = np.clip(np.searchsorted(ys, y, side="right") - 1, 0, len(ys) - 2)
    tx = (x - xs[i]) / (xs[i + 1] - xs[i])
    ty = (y - ys[j]) / (ys[j + 1] - ys[j])
    out = []
    for f in fields:
        out.append((1 - ty) * ((1 - tx) * f[j, i] + tx * f[j, i + 1]) +
                   ty * ((1 - tx) * f[j + 1, i] + tx * f[j + 1, i + 1]))
    return np.stack(out, 1)


def subset_sizes(coords, elems, winsize, mode="uniform", lo=16, hi=64):
    """Per-node subset size: the reference's uniform winsize
    (Subpb1Quadtree.m:50), or twice the smallest side of the elements at the
    node clipped to [lo, hi] (even)."""
    n = len(coords)
    if mode == "uniform":
        return np.full(n, int(winsize), np.int32)
    side = np.full(n, np.inf)
    s = np.abs(coords[elems[:, 2] - 1, 0] - coords[elems[:, 0] - 1, 0])
    for k in range(8):
        nz = elems[:, k] > 0
        np.minimum.at(side, elems[nz, k] - 1, s[nz])
    side[~np.isfinite(side)] = winsize / 2
    w = np.clip(2 * side, lo, hi)
    return (2 * np.round(w / 2)).astype(np.int32)


def select_beta(betas, e1, e2):
    """main_ALDIC_Quadtree.m:179-190: normalised error sum, three-point
    parabola vertex in log10(beta) around the minimum when it has two
    neighbours, else the minimising beta."""
    e1, e2 = np.asarray(e1), np.asarray(e2)
    es = (e1 - e1.mean()) / e1.std(ddof=1) + (e2 - e2.mean()) / e2.std(ddof=1)
    k = int(np.nanargmin(es))
    if 1 <= k <= len(betas) - 2:
        p = np.polyfit(np.log10(betas[k - 1:k + 2]), es[k - 1:k + 2], 2)
        return 10 ** (-p[1] / 2 / p[0])
    return betas[k]


def frame(f_raw, g_raw, mask, winsize, step, search, tol=1e-2, mu=1e-3, n_admm=3, tol2=1e-2,
          min_size=2, subsets="uniform", gridx=None, gridy=None):
    """One frame of main_ALDIC_Quadtree.m Sections 3-6 (ImgSeqNum 2) with
    the interactive outlier removal and the strain smoothing
    (DICpara.StrainSmoothness, regularizeNd) left out."""
    import oracle as O
    f_raw, g_raw = np.asarray(f_raw), np.asarray(g_raw)
    H, W = f_raw.shape
    mask = np.asarray(mask, np.float64)
    gx = tuple(gridx) if gridx is not None else (1, W)
    gy = tuple(gridy) if gridy is not None else (1, H)
    roi = (gx[0], gx[1], gy[0], gy[1])
    fn, _, _ = O.normalize(f_raw, roi)                    # funNormalizeImg(Img, gridxyROIRange)
    gn, mg, _ = O.normalize(g_raw, roi)
    dfdx, dfdy = O.gradient(fn, mask)
    x, y, u, v, cc, _ = O.int_search(f_raw, g_raw, mg, gx, gy, winsize, step, (search, search))
    hole = mask[y.astype(int) - 1, x.astype(int) - 1] == 0        # IntegerSearch.m:68-73
    u, v = np.where(hole, np.nan, u), np.where(hole, np.nan, v)
    ny, nx = u.shape
    coords0, el0 = uniform_mesh(x.reshape(-1), y.reshape(-1), nx, ny)
    ug = O.inpaint_springs(nx, ny, u.reshape(-1)).reshape(ny, nx)
    vg = O.inpaint_springs(nx, ny, v.reshape(-1)).reshape(ny, nx)
    c, E, d = generate_quadtree_mesh(coords0, el0, mask, step, min_size)
    n = len(c)
    U0 = interp_uniform(x[0], y[:, 0], [ug, vg], c).reshape(-1)
    wins = subset_sizes(c, E, winsize, subsets)
    edges = mesh_edges(E)
    # Section 4
    U1, F1, it, H21 = O.icgn_batch(fn, gn, dfdx, dfdy, c, U0, wins, tol)
    bad, nbad = icgn_flags(it)
    U1 = graph_fill(n, edges, np.where(bad[:, None], 0.0, U1.reshape(n, 2)), bad).reshape(-1)
    F1 = graph_fill(n, edges, np.where(bad[:, None], 0.0, F1.reshape(n, 4)), bad).reshape(-1)
    U_icgn, F_icgn = U1.copy(), F1.copy()
    # Section 5
    betas = np.array([1e-3, 1e-2, 1e-1]) * step * step * mu
    e1, e2 = [], []
    for b in betas:
        U2 = subpb2_quadtree(c, E, d, b, mu, U1, F1)
        F2 = nodal_strain_quadtree(c, E, U2)
        e1.append(np.linalg.norm(U1 - U2))
        e2.append(np.linalg.norm(F1 - F2))
    beta = select_beta(betas, e1, e2)
    if abs(beta - betas[-1]) > np.finfo(float).eps:
        U2 = subpb2_quadtree(c, E, d, beta, mu, U1, F1)
        F2 = nodal_strain_quadtree(c, E, U2)
    dd = np.repeat(4 * (d - 1), 4) + np.tile(np.arange(4), len(d))
    F2[dd] = F1[dd]
    udual, vdual = F2 - F1, U2 - U1
    # Section 6
    upd, upd2, its = [], [], [it]
    U1old = U1.copy()
    for step_k in range(2, 2 + n_admm):
        U2old = U2.copy()
        U1, it1 = O.subpb1_batch(fn, gn, dfdx, dfdy, c, U2, F2, vdual, H21, wins, mu, tol)
        b1, _ = icgn_flags(it1, 20.0)
        U1 = graph_fill(n, edges, np.where(b1[:, None], 0.0, U1.reshape(n, 2)), b1).reshape(-1)
        F1 = F2.copy()
        U2 = subpb2_quadtree(c, E, d, beta, mu, U1, F1)
        F2 = nodal_strain_quadtree(c, E, U2)
        F2[dd] = F1[dd]
        upd.append(np.linalg.norm(U2old - U2) / np.sqrt(2 * n))
        upd2.append(np.linalg.norm(U1old - U1) / np.sqrt(2 * n))
        U1old = U1.copy()
        its.append(it1)
        udual, vdual = F2 - F1, U2 - U1
        if upd[-1] < tol2 or upd2[-1] < tol2:
            break
    return dict(coords=c, elems=E, dirichlet=d, U=U2, F=F2, U_icgn=U_icgn, F_icgn=F_icgn,
                iters_icgn=it, bad_icgn=nbad, beta=beta, update_y=upd, update_y2=upd2,
                wins=wins, U0=U0)
