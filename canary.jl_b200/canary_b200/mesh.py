"""Mesh generation and connectivity of Canary (src/mesh.jl), single rank.

Host-side mirror of the reference's setup API used by the Euler/NS drivers:
brickmesh -> partition (Hilbert-curve element order) -> connectmesh ->
mappings.  Index arrays keep the reference's 1-based Int64 convention and
column-major (Fortran-ordered) layouts, so they can be handed unchanged to
the device library.  Multi-rank partitioning and ghost exchange are outside
this package's scope (one rank drives one GPU).
"""
from __future__ import annotations

import numpy as np

_U64 = np.uint64


def linearpartition(n: int, p: int, np_: int) -> range:
    """Range of the p-th of np_ nearly equal pieces of 1:n (mesh.jl:13)."""
    return range((p - 1) * n // np_ + 1, p * n // np_ + 1)


def hilbertcode(Y, bits: int = 64) -> np.ndarray:
    """Hilbert integer of integer axes coordinates, Skilling's AxestoTranspose
    followed by the bit transpose (mesh.jl:35-88).  Y is (n,) or (n, m) for m
    points at once; returns the same shape (uint64, H[0] most significant)."""
    X = np.array(Y, dtype=_U64, copy=True)
    single = X.ndim == 1
    if single:
        X = X[:, None]
    n = X.shape[0]
    M = _U64(1) << _U64(bits - 1)
    Q = M
    for _ in range(bits - 1):
        P = Q - _U64(1)
        for i in range(n):
            hit = (X[i] & Q) != 0
            t = (X[0] ^ X[i]) & P
            x0 = np.where(hit, X[0] ^ P, X[0] ^ t)
            xi = np.where(hit, X[i], X[i] ^ t)
            X[0] = x0
            if i != 0:
                X[i] = xi
            else:
                X[0] = np.where(hit, X[0], X[0])
        Q >>= _U64(1)
    for i in range(1, n):
        X[i] ^= X[i - 1]
    t = np.zeros(X.shape[1], dtype=_U64)
    Q = M
    for _ in range(bits - 1):
        t = np.where((X[n - 1] & Q) != 0, t ^ (Q - _U64(1)), t)
        Q >>= _U64(1)
    for i in range(n):
        X[i] ^= t
    H = np.zeros_like(X)
    for i in range(n):
        for j in range(bits):
            k = i * bits + j
            bit = (X[n - 1 - (k % n)] >> _U64(k // n)) & _U64(1)
            H[n - 1 - i] |= bit << _U64(j)
    return H[:, 0] if single else H


def _scaled_floor(c: np.ndarray) -> np.ndarray:
    """floor((2^64-1) * c) exactly for c in [0, 1] (mesh.jl:136 evaluates it in
    128-bit arithmetic, where the product is exact)."""
    out = np.zeros(c.shape, dtype=_U64)
    m, ex = np.frexp(c)  # c = m 2^ex, m in [0.5, 1)
    for idx in np.ndindex(c.shape):
        if c[idx] <= 0.0:
            continue
        mi = int(np.ldexp(m[idx], 53))
        sh = 53 - int(ex[idx])
        prod = ((1 << 64) - 1) * mi
        out[idx] = (1 << 64) - 1 if sh <= 0 else (prod >> sh if sh < 128 else 0)
    return out


def centroidtocode(elemtocoord) -> np.ndarray:
    """Hilbert code of each element centroid (mesh.jl:107-141), (d, nelem)."""
    etc = np.asarray(elemtocoord, dtype=np.float64)
    d, nvert, nelem = etc.shape
    cen = np.zeros((d, nelem))
    for v in range(nvert):  # sequential sum over corners
        cen = cen + etc[:, v, :]
    cen = cen / nvert
    if nelem > 0:
        cmin, cmax = cen.min(axis=1), cen.max(axis=1)
    else:
        cmin, cmax = np.full(d, np.inf), np.full(d, -np.inf)
    size = cmax - cmin
    if np.all(size == 0):
        size = np.ones(d)
    else:
        size = np.where(size == 0, size.max(), size)
    c = (cen - cmin[:, None]) / size[:, None]
    return hilbertcode(_scaled_floor(c), 64)


def _corner_fmask(d: int):
    # corners (0-based, column-major in the 2^d cube) of each face (mesh.jl:281-284)
    return [[v for v in range(2 ** d) if ((v >> (f // 2)) & 1) == f % 2] for f in range(2 * d)]


def brickmesh(x, periodic, part: int = 1, numparts: int = 1, boundary=None):
    """Cartesian brick mesh (mesh.jl:259-317).

    Returns (elemtovert (2^d, nelem), elemtocoord (d, 2^d, nelem),
    elemtobndy (2d, nelem), faceconnections [[e, f, verts...], ...])."""
    d = len(x)
    assert d == len(periodic) and d >= 1 and 1 <= part <= numparts
    if boundary is None:
        boundary = np.ones((2, d), dtype=np.int64)
    boundary = np.asarray(boundary, dtype=np.int64).reshape(2, d, order="F")
    x = [np.asarray(xi, dtype=np.float64) for xi in x]
    nx = [len(xi) for xi in x]
    ned = [n - 1 for n in nx]
    nvert, nface = 2 ** d, 2 * d
    loc = linearpartition(int(np.prod(ned)), part, numparts)
    g = np.arange(loc.start - 1, loc.stop - 1, dtype=np.int64)
    ec = []
    for i in range(d):
        ec.append(g % ned[i] + 1)
        g = g // ned[i]
    nloc = len(loc)
    etv = np.zeros((nvert, nloc), dtype=np.int64, order="F")
    etc = np.zeros((d, nvert, nloc), dtype=np.float64, order="F")
    etb = np.zeros((nface, nloc), dtype=np.int64, order="F")
    strides = np.cumprod([1] + nx[:-1])
    for v in range(nvert):
        vid = np.zeros(nloc, dtype=np.int64)
        for j in range(d):
            vc = ec[j] + ((v >> j) & 1)
            vid += (vc - 1) * strides[j]
            etc[j, v, :] = x[j][vc - 1]
        etv[v, :] = vid + 1
    for i in range(d):
        if not periodic[i]:
            etb[2 * i, ec[i] == 1] = boundary[0, i]
            etb[2 * i + 1, ec[i] == ned[i]] = boundary[1, i]
    fm = _corner_fmask(d)
    fc = []
    for el in range(nloc):
        for i in range(d):
            if periodic[i] and ec[i][el] == ned[i]:
                verts = []
                for v in fm[2 * i]:
                    vid = 0
                    for j in range(d):
                        base = 1 if j == i else int(ec[j][el])
                        vid += (base + ((v >> j) & 1) - 1) * int(strides[j])
                    verts.append(vid + 1)
                fc.append([el + 1, 2 * (i + 1)] + verts)
    return etv, etc, etb, fc


def partition(elemtovert, elemtocoord, elemtobndy, faceconnections):
    """Single-rank Hilbert-curve partition (mesh.jl:499-580): elements are
    reordered by the Hilbert code of their centroids (ties by element
    number) and face connections follow their elements."""
    etc = np.asarray(elemtocoord, dtype=np.float64)
    d, nvert, nelem = etc.shape
    nface, nfv = 2 * d, 2 ** (d - 1)
    code = centroidtocode(etc)
    keys = [np.arange(nelem)] + [code[i] for i in range(d - 1, -1, -1)]
    order = np.lexsort(keys)
    e2fc = np.zeros((nfv, nface, nelem), dtype=np.int64)
    for row in faceconnections:
        e2fc[:, row[1] - 1, row[0] - 1] = row[2:]
    etv = np.asfortranarray(np.asarray(elemtovert)[:, order])
    etc = np.asfortranarray(etc[:, :, order])
    etb = np.asfortranarray(np.asarray(elemtobndy)[:, order])
    e2fc = e2fc[:, :, order]
    fc = [[e + 1, f + 1] + [int(v) for v in e2fc[:, f, e]]
          for e in range(nelem) for f in range(nface) if e2fc[0, f, e] > 0]
    return etv, etc, etb, fc


def _sort_face(v):
    """vertsortandorder for 1, 2 or 4 face vertices (mesh.jl:595-719)."""
    v = list(v)
    if len(v) == 1:
        return tuple(v), 1
    if len(v) == 2:
        return (tuple(v), 1) if v[0] <= v[1] else ((v[1], v[0]), 2)
    if len(v) == 4:
        a, b, c, dd = v
        s = []
        for (p, q) in ((0, 1), (2, 3), (0, 2), (1, 3), (1, 2)):
            if v[q] < v[p]:
                v[p], v[q] = v[q], v[p]
                s.append(True)
            else:
                s.append(False)
        table = {(0, 0, 0, 0, 0): 1, (0, 0, 0, 0, 1): 2, (1, 0, 0, 0, 0): 3,
                 (0, 0, 1, 1, 1): 4, (1, 1, 0, 0, 1): 5, (0, 0, 1, 1, 0): 6,
                 (1, 1, 1, 1, 1): 7, (1, 1, 1, 1, 0): 8}
        key = tuple(int(t) for t in s)
        if key not in table:
            raise ValueError(f"Problem finding vertex ordering {tuple(v)} with flips {tuple(s)}")
        return tuple(v), table[key]
    raise ValueError("unsupported face vertex count")


def connectmesh(elemtovert, elemtocoord, elemtobndy, faceconnections):
    """Single-rank face matching (mesh.jl:751-956): faces with the same sorted
    vertex tuple are connected.  Returns a dict with elemtoelem, elemtoface,
    elemtoordr, elemtobndy (all (nface, nelem), 1-based) and elemtocoord."""
    etv = np.asarray(elemtovert, dtype=np.int64)
    etc = np.asarray(elemtocoord, dtype=np.float64)
    d, nvert, nelem = etc.shape
    nface, nfv = 2 * d, 2 ** (d - 1)
    fm = _corner_fmask(d)
    keys = np.zeros((nface * nelem, nfv), dtype=np.int64)
    orient = np.ones(nface * nelem, dtype=np.int64)
    for f in range(nface):
        fv = etv[fm[f], :]  # (nfv, nelem)
        fv_sorted = np.sort(fv, axis=0)
        keys[f::nface, :] = fv_sorted.T
        if d == 2:
            orient[f::nface] = np.where(fv[0] <= fv[1], 1, 2)
        elif d == 3:
            # Cartesian face vertex order of a brick is already sorted (o = 1);
            # anything else needs the full vertsortandorder table
            ok = np.all(fv == fv_sorted, axis=0)
            if not np.all(ok):
                for e in np.nonzero(~ok)[0]:
                    _, orient[e * nface + f] = _sort_face(fv[:, e])
    for row in faceconnections:
        j = (row[0] - 1) * nface + (row[1] - 1)
        vs, o = _sort_face(row[2:])
        keys[j, :] = vs
        orient[j] = o
    cols = np.lexsort([np.arange(nface * nelem)] + [keys[:, q] for q in range(nfv - 1, -1, -1)])
    ks = keys[cols]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    e2e = np.tile(np.arange(1, nelem + 1, dtype=np.int64), (nface, 1))
    e2f = np.tile(np.arange(1, nface + 1, dtype=np.int64)[:, None], (1, nelem))
    e2o = np.ones((nface, nelem), dtype=np.int64)
    j, n = 0, len(cols)
    while j < n:
        if j + 1 < n and same[j]:
            for m, o in ((cols[j], cols[j + 1]), (cols[j + 1], cols[j])):
                me, mf = divmod(int(m), nface)
                ne, nf = divmod(int(o), nface)
                e2e[mf, me] = ne + 1
                e2f[mf, me] = nf + 1
                if d == 2:
                    e2o[mf, me] = 1 if orient[o] == orient[m] else 2
                elif d == 3:
                    if orient[o] != 1 or orient[m] != 1:
                        raise NotImplementedError("TODO add support for other orientations")
            j += 2
        else:
            j += 1
    return dict(elemtocoord=np.asfortranarray(etc), elemtoelem=np.asfortranarray(e2e),
                elemtoface=np.asfortranarray(e2f), elemtoordr=np.asfortranarray(e2o),
                elemtobndy=np.asfortranarray(np.asarray(elemtobndy, dtype=np.int64)),
                elems=range(1, nelem + 1), realelems=range(1, nelem + 1),
                ghostelems=range(nelem + 1, nelem + 1), sendelems=[], nabrtorank=[],
                nabrtorecv=[], nabrtosend=[])


def face_nodes(N: int, d: int) -> np.ndarray:
    """fmask of mappings (mesh.jl:979-983): 0-based volume node of each face
    node, shape (Nfp, nface)."""
    Nq = N + 1
    p = np.arange(Nq ** d).reshape((Nq,) * d, order="F")
    cols = []
    for f in range(2 * d):
        sl = [slice(None)] * d
        sl[f // 2] = N * (f % 2)
        cols.append(p[tuple(sl)].ravel(order="F"))
    return np.stack(cols, axis=1)


def mappings(N: int, elemtoelem, elemtoface, elemtoordr):
    """vmapM/vmapP, (Nfp, nface, nelem) 1-based linear node ids (mesh.jl:973-1001)."""
    e2e = np.asarray(elemtoelem, dtype=np.int64)
    e2f = np.asarray(elemtoface, dtype=np.int64)
    e2o = np.asarray(elemtoordr, dtype=np.int64)
    nface, nelem = e2e.shape
    d = nface // 2
    Np = (N + 1) ** d
    if np.any(e2o != 1):
        raise NotImplementedError("only face orientation 1 is supported (mesh.jl:993-994)")
    fm = face_nodes(N, d) + 1
    e = np.arange(nelem, dtype=np.int64)
    vmapM = Np * e[None, None, :] + fm[:, :, None]
    vmapP = Np * (e2e[None, :, :] - 1) + fm[:, (e2f - 1)]  # fm[:, f2] for each (f, e)
    return np.asfortranarray(vmapM), np.asfortranarray(vmapP)
