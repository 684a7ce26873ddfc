"""Structured box meshes in the reference's compute-mesh layout (numpy, host side).

Restates, for hexahedral boxes, what the reference's generateBox (src/fvm/mesh/RawMesh.cpp:391-502)
and serial Mesh::build (src/fvm/mesh/Mesh.cpp:112-333 buildGlobal, :600-648 finishLocal) produce:

* point numbering P(i,j,k) = i + (nx+1)(j + (ny+1)k), cells C(i,j,k) = i + nx(j + ny k);
* internal faces in owner-cell order, +x, +y, +z per cell; then the cyclic pairs merged into
  internal faces (owner on the min side, d carrying the periodic shift); then the wall/patch
  faces patch by patch (xMin xMax yMin yMax zMin zMax); empty front/back faces of 2D boxes
  are dropped;
* face geometry by the triangle decomposition about the vertex average, cell geometry by the
  pyramid decomposition about the face-centre average, all sums in the reference's order, so
  the arrays agree with the reference to rounding (bit-for-bit in practice);
* w, deltaCoeffs, nonOrthDeltaCoeffs (1/max(n·d, 0.05|d|)), corrVecs, skewVecs.

Everything is vectorised so a 256x192x128 box builds in seconds.
"""
from __future__ import annotations

import math

import numpy as np

VSMALL = 1.0e-300

PATCH_NAMES = ("xMin", "xMax", "yMin", "yMax", "zMin", "zMax")


def tanh_stretch(beta: float):
    """tanhStretch (RawMesh.cpp:387-389): symmetric two-sided clustering."""
    tb = math.tanh(beta)
    return lambda t: np.array([0.5 * (1.0 + math.tanh(beta * (2.0 * v - 1.0)) / tb) for v in np.atleast_1d(t)])


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _mag(a):
    return np.sqrt(_dot(a, a))


def box_points(n, lo=(0, 0, 0), hi=(1, 1, 1), beta=(0, 0, 0)):
    """Vertex coordinates in generateBox order, shape ((nx+1)(ny+1)(nz+1), 3)."""
    nx, ny, nz = (int(v) for v in n)
    axes = []
    for d, nd in enumerate((nx, ny, nz)):
        t = np.arange(nd + 1, dtype=np.float64) / nd
        if beta[d] and beta[d] > 0:
            t = tanh_stretch(beta[d])(t)
        axes.append(lo[d] + (hi[d] - lo[d]) * t)
    X = np.broadcast_to(axes[0][None, None, :], (nz + 1, ny + 1, nx + 1))
    Y = np.broadcast_to(axes[1][None, :, None], (nz + 1, ny + 1, nx + 1))
    Z = np.broadcast_to(axes[2][:, None, None], (nz + 1, ny + 1, nx + 1))
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).copy()


def jitter_interior(points, n, amplitude, seed):
    """Moves every interior vertex by U(-amplitude*h_d, +amplitude*h_d) in each direction d
    (h_d: the smaller adjacent spacing along d).  Boundary vertices stay, so periodic faces
    keep matching; for a one-cell-thick (2D) box the jitter is the same on both layers."""
    nx, ny, nz = (int(v) for v in n)
    P = np.ascontiguousarray(points, np.float64).reshape(nz + 1, ny + 1, nx + 1, 3).copy()
    rng = np.random.default_rng(seed)
    flat = nz == 1
    kin = slice(None) if flat else slice(1, -1)
    interior = (kin, slice(1, -1), slice(1, -1))
    shape = P[interior + (0,)].shape
    if flat:
        shape = (1,) + shape[1:]
    for d, nd in enumerate((nx, ny, nz)):
        if nd < 2:
            continue
        ax = 2 - d
        coord = P[..., d]
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        mid = [slice(None)] * 3
        lo[ax], mid[ax], hi[ax] = slice(0, -2), slice(1, -1), slice(2, None)
        h = np.minimum(coord[tuple(mid)] - coord[tuple(lo)], coord[tuple(hi)] - coord[tuple(mid)])
        # h is defined on points interior along ax; restrict it to points interior in all directions
        hsl = list(interior)
        hsl[ax] = slice(None)
        hv = h[tuple(hsl)]
        u = rng.uniform(-1.0, 1.0, size=shape)
        coord[interior] += amplitude * (u * hv)
    return P.reshape(-1, 3)


def _face_geometry(pts, fp):
    """faceGeometry (Mesh.cpp:21-48) for quads: fp (nF, 4) point indices."""
    q = pts[fp]  # (nF, 4, 3)
    pavg = ((q[:, 0] + q[:, 1]) + q[:, 2]) + q[:, 3]
    pavg = pavg / 4.0
    sumN = np.zeros_like(pavg)
    sumA = np.zeros(len(fp))
    sumAc = np.zeros_like(pavg)
    for k in range(4):
        p0 = q[:, k]
        p1 = q[:, (k + 1) % 4]
        c = (p0 + p1) + pavg
        nk = _cross(p1 - p0, pavg - p0)
        a = _mag(nk)
        sumN = sumN + nk
        sumA = sumA + a
        sumAc = sumAc + a[:, None] * c
    small = sumA < VSMALL
    Cf = sumAc / (3.0 * sumA)[:, None]
    Cf[small] = pavg[small]
    Sf = 0.5 * sumN
    return Sf, Cf


def box_mesh(n, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(False, False, False), two_d=False, beta=(0, 0, 0),
             points=None, patch_types=None):
    """Builds the compute mesh of a box.  Returns a dict with the cfd::Mesh array names:
    n_cells, n_internal_faces, n_faces, owner, neighbour, V, C, Sf, magSf, Cf, d, w, deltaCoeffs,
    ndc, corrVecs, skewVecs, skewed, patch_start, patch_size, patch_names, two_d, empty_dir."""
    nx, ny, nz = (int(v) for v in n)
    if nx < 1 or ny < 1 or nz < 1:
        raise ValueError("bad resolution")
    if two_d and nz != 1:
        raise ValueError("twoD requires n[2] == 1")
    for d, nd in enumerate((nx, ny, nz)):
        if periodic[d] and nd < 2 and not (d == 2 and two_d):
            raise ValueError("a periodic direction needs at least 2 cells")
    pts = box_points(n, lo, hi, beta) if points is None else np.ascontiguousarray(points, np.float64).reshape(-1, 3)

    def P(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    def Cc(i, j, k):
        return i + nx * (j + ny * k)

    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    nC = nx * ny * nz
    # ---- internal faces in owner order (+x, +y, +z per cell), as generateBox emits them
    cand_own, cand_nei, cand_fp, cand_key = [], [], [], []
    for dirn in range(3):
        if dirn == 0:
            m = I + 1 < nx
            i, j, k = I[m], J[m], K[m]
            fp = np.stack([P(i + 1, j, k), P(i + 1, j + 1, k), P(i + 1, j + 1, k + 1), P(i + 1, j, k + 1)], 1)
            nb = Cc(i + 1, j, k)
        elif dirn == 1:
            m = J + 1 < ny
            i, j, k = I[m], J[m], K[m]
            fp = np.stack([P(i, j + 1, k), P(i, j + 1, k + 1), P(i + 1, j + 1, k + 1), P(i + 1, j + 1, k)], 1)
            nb = Cc(i, j + 1, k)
        else:
            m = K + 1 < nz
            i, j, k = I[m], J[m], K[m]
            fp = np.stack([P(i, j, k + 1), P(i + 1, j, k + 1), P(i + 1, j + 1, k + 1), P(i, j + 1, k + 1)], 1)
            nb = Cc(i, j, k + 1)
        own = Cc(i, j, k)
        cand_own.append(own)
        cand_nei.append(nb)
        cand_fp.append(fp)
        cand_key.append(own * 3 + dirn)
    key = np.concatenate(cand_key)
    order = np.argsort(key, kind="stable")
    r_own = np.concatenate(cand_own)[order]
    r_nei = np.concatenate(cand_nei)[order]
    r_fp = np.concatenate(cand_fp)[order]
    nI_raw = len(r_own)
    # ---- boundary patches of the raw mesh
    patches = []  # (name, type, fp, owner)
    jj, kk = np.meshgrid(np.arange(ny), np.arange(nz), indexing="xy")
    jj, kk = jj.ravel(), kk.ravel()  # k outer, j inner
    for side in range(2):
        i = 0 if side == 0 else nx
        if side == 0:
            fp = np.stack([P(i, jj, kk), P(i, jj, kk + 1), P(i, jj + 1, kk + 1), P(i, jj + 1, kk)], 1)
        else:
            fp = np.stack([P(i, jj, kk), P(i, jj + 1, kk), P(i, jj + 1, kk + 1), P(i, jj, kk + 1)], 1)
        patches.append((PATCH_NAMES[side], "cyclic" if periodic[0] else "patch", fp,
                        Cc(0 if side == 0 else nx - 1, jj, kk)))
    ii, kk = np.meshgrid(np.arange(nx), np.arange(nz), indexing="xy")
    ii, kk = ii.ravel(), kk.ravel()
    for side in range(2):
        j = 0 if side == 0 else ny
        if side == 0:
            fp = np.stack([P(ii, j, kk), P(ii + 1, j, kk), P(ii + 1, j, kk + 1), P(ii, j, kk + 1)], 1)
        else:
            fp = np.stack([P(ii, j, kk), P(ii, j, kk + 1), P(ii + 1, j, kk + 1), P(ii + 1, j, kk)], 1)
        patches.append((PATCH_NAMES[2 + side], "cyclic" if periodic[1] else "patch", fp,
                        Cc(ii, 0 if side == 0 else ny - 1, kk)))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    ii, jj = ii.ravel(), jj.ravel()
    for side in range(2):
        k = 0 if side == 0 else nz
        if side == 0:
            fp = np.stack([P(ii, jj, k), P(ii, jj + 1, k), P(ii + 1, jj + 1, k), P(ii + 1, jj, k)], 1)
        else:
            fp = np.stack([P(ii, jj, k), P(ii + 1, jj, k), P(ii + 1, jj + 1, k), P(ii, jj + 1, k)], 1)
        typ = "empty" if two_d else ("cyclic" if periodic[2] else "patch")
        patches.append((PATCH_NAMES[4 + side], typ, fp, Cc(ii, jj, 0 if side == 0 else nz - 1)))
    if patch_types is not None:
        patches = [(nm, typ if typ in ("cyclic", "empty") else str(patch_types[q]), fp, ow)
                   for q, (nm, typ, fp, ow) in enumerate(patches)]

    # ---- raw face geometry, in raw face order
    all_fp = np.concatenate([r_fp] + [p[2] for p in patches])
    all_own = np.concatenate([r_own] + [p[3] for p in patches])
    Sf_raw, Cf_raw = _face_geometry(pts, all_fp)
    nF_raw = len(all_fp)
    # ---- cell geometry (Mesh.cpp:135-153): faces of each cell in ascending raw face order
    cf = np.concatenate([np.arange(nF_raw), np.arange(nI_raw)])
    cc = np.concatenate([all_own, r_nei])
    o = np.lexsort((cf, cc))
    cell_faces = cf[o].reshape(nC, 6)
    is_own = (all_own[cell_faces] == np.arange(nC)[:, None])
    cEst = np.zeros((nC, 3))
    for q in range(6):
        cEst = cEst + Cf_raw[cell_faces[:, q]]
    cEst = cEst / 6.0
    cSum = np.zeros((nC, 3))
    vSum = np.zeros(nC)
    for q in range(6):
        f = cell_faces[:, q]
        S = np.where(is_own[:, q, None], Sf_raw[f], -Sf_raw[f])
        pv = np.maximum(_dot(S, Cf_raw[f] - cEst), VSMALL)
        cSum = cSum + pv[:, None] * (0.75 * Cf_raw[f] + 0.25 * cEst)
        vSum = vSum + pv
    C = cSum / vSum[:, None]
    V = vSum / 3.0
    # ---- compute faces: internal, then cyclic pairs, then boundary patches (Mesh.cpp:239-320)
    own_l, nei_l, Sf_l, Cf_l, d_l = [r_own], [r_nei], [Sf_raw[:nI_raw]], [Cf_raw[:nI_raw]], [C[r_nei] - C[r_own]]
    starts = np.cumsum([nI_raw] + [len(p[2]) for p in patches])[:-1]
    done = [False] * 6
    for ia in range(6):
        if patches[ia][1] != "cyclic" or done[ia]:
            continue
        ib = ia + 1 if ia % 2 == 0 else ia - 1
        done[ia] = done[ib] = True
        fa = starts[ia] + np.arange(len(patches[ia][2]))
        fb = starts[ib] + np.arange(len(patches[ib][2]))  # faces match index by index on a box
        o_ = all_own[fa]
        n_ = all_own[fb]
        own_l.append(o_)
        nei_l.append(n_)
        Sf_l.append(Sf_raw[fa])
        Cf_l.append(Cf_raw[fa])
        d_l.append(((C[n_] + (Cf_raw[fa] - Cf_raw[fb])) - C[o_]))
    nI = int(sum(len(x) for x in own_l))
    patch_start, patch_size, patch_names, patch_kinds = [], [], [], []
    empty_n = np.zeros(3)
    two = False
    for q, (nm, typ, fp, ow) in enumerate(patches):
        if typ == "cyclic":
            continue
        f = starts[q] + np.arange(len(fp))
        if typ == "empty":
            two = True
            empty_n = empty_n + np.abs(Sf_raw[f]).sum(axis=0)
            continue
        patch_start.append(nI + sum(patch_size))
        patch_size.append(len(fp))
        patch_names.append(nm)
        patch_kinds.append(typ)
        own_l.append(all_own[f])
        Sf_l.append(Sf_raw[f])
        Cf_l.append(Cf_raw[f])
        d_l.append(Cf_raw[f] - C[all_own[f]])
    owner = np.concatenate(own_l).astype(np.int32)
    neighbour = np.concatenate(nei_l).astype(np.int32)
    Sf = np.concatenate(Sf_l)
    Cf = np.concatenate(Cf_l)
    d = np.concatenate(d_l)
    nF = len(owner)
    # ---- finishLocal (Mesh.cpp:600-626)
    magSf = _mag(Sf)
    nrm = Sf / magSf[:, None]
    w = np.ones(nF)
    skew = np.zeros((nF, 3))
    CP = C[owner[:nI]]
    sOwn = np.abs(_dot(Sf[:nI], Cf[:nI] - CP))
    sNei = np.abs(_dot(Sf[:nI], (CP + d[:nI]) - Cf[:nI]))
    w[:nI] = sNei / (sOwn + sNei)
    skew[:nI] = Cf[:nI] - (CP + d[:nI] * (1.0 - w[:nI])[:, None])
    magd = _mag(d)
    skewness = _mag(skew[:nI]) / magd[:nI] if nI else np.zeros(0)
    dc = 1.0 / magd
    ndc = 1.0 / np.maximum(_dot(nrm, d), 0.05 * magd)
    corr = nrm - d * ndc[:, None]
    empty_dir = -1
    if two:
        empty_dir = int(np.argmax(empty_n)) if empty_n.max() > 0 else 0
        # first maximum, as the reference's strict '>' scan
        empty_dir = 0
        for a in (1, 2):
            if empty_n[a] > empty_n[empty_dir]:
                empty_dir = a
    return dict(n_cells=nC, n_internal_faces=nI, n_faces=nF, owner=owner, neighbour=neighbour, V=V, C=C, Sf=Sf,
                magSf=magSf, Cf=Cf, d=d, w=w, deltaCoeffs=dc, ndc=ndc, corrVecs=corr, skewVecs=skew,
                skewed=bool(skewness.size and skewness.max() > 1e-8), patch_start=np.array(patch_start, np.int32),
                patch_size=np.array(patch_size, np.int32), patch_names=patch_names, patch_kinds=patch_kinds,
                two_d=two, empty_dir=empty_dir, shape=(nx, ny, nz), periodic=tuple(bool(p) for p in periodic))


def poisson_matrix(mesh: dict, gamma=1.0, ref_cell: int | None = 0):
    """LDU arrays of fvm::laplacian(gamma, p) with zeroGradient walls and no non-orthogonal
    correction (Fvm.h:149-154: upper = Γ|S|ndc, diag -= on both sides), then
    setReference(ref_cell) (FvMatrix.h:134-141: the reference cell's diagonal doubled).
    Returns (diag, upper)."""
    nI = mesh["n_internal_faces"]
    g = np.broadcast_to(np.asarray(gamma, np.float64), (mesh["n_faces"],))
    upper = g[:nI] * mesh["magSf"][:nI] * mesh["ndc"][:nI]
    diag = np.zeros(mesh["n_cells"])
    # face-ordered accumulation (owner then neighbour per face), as the reference's face loop
    idx = np.stack([mesh["owner"][:nI], mesh["neighbour"]], axis=1).ravel()
    np.subtract.at(diag, idx, np.repeat(upper, 2))
    if ref_cell is not None:
        diag[ref_cell] += diag[ref_cell]
    return diag, upper
