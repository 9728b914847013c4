"""Independent numpy/scipy restatement of the reference's P2/P1 PISO step for small meshes.

Written separately from the C++ oracle (different language, dense element loops, direct sparse
solves instead of Krylov iterations) so that the two restatements cross-check each other.
Citations are to sudo-shaka/Cell-Fluid-Structure-Analysis:
  geometry/gradients  src/Mesh/Mesh.cpp:448-471, 590-614
  P2 edge numbering   src/Mesh/Mesh.cpp:641-677
  assembly            src/FEM/NavierStokes.cpp:70-356
  pisoStep            src/FEM/NavierStokes.cpp:374-771, 804-839
Used by gen_golden.py (fixtures) and by tests.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
WALL, INLET, OUTLET, INTERNAL, UNDEFINED = range(5)


def geometry(xyz, tets):
    P = xyz[tets]  # [nt,4,3]
    a, b, c, d = P[:, 0], P[:, 1], P[:, 2], P[:, 3]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a) / 6.0)
    sixv = np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a))
    inv = (1.0 / sixv)[:, None]
    g = np.empty((len(tets), 4, 3))
    g[:, 0] = inv * np.cross(d - b, c - b)
    g[:, 1] = inv * np.cross(c - a, d - a)
    g[:, 2] = inv * np.cross(d - a, b - a)
    g[:, 3] = inv * np.cross(b - a, c - a)
    return vol, g


def edge_numbering(tets):
    ids = {}
    te = np.empty((len(tets), 6), np.int64)
    for t, v in enumerate(tets):
        for e, (i, j) in enumerate(EDGES):
            k = (min(v[i], v[j]), max(v[i], v[j]))
            if k not in ids:
                ids[k] = len(ids)
            te[t, e] = ids[k]
    return te, ids


def node_grads(g):
    """[nt,10,3]: P1 gradients then centroid P2 gradients grad phi_a + grad phi_b."""
    out = np.empty((g.shape[0], 10, 3))
    out[:, :4] = g
    for e, (i, j) in enumerate(EDGES):
        out[:, 4 + e] = g[:, i] + g[:, j]
    return out


def mass_table():
    m = np.empty((10, 10))
    for i in range(10):
        for j in range(10):
            if i < 4 and j < 4:
                m[i, j] = 1 / 10 if i == j else 1 / 20
            elif i >= 4 and j >= 4:
                m[i, j] = 1 / 15 if i == j else 1 / 60
            else:
                m[i, j] = 1 / 30
    return m


def assemble(xyz, tets, density, viscosity):
    nv = len(xyz)
    vol, g = geometry(xyz, tets)
    te, ids = edge_numbering(tets)
    ne = len(ids)
    N2 = nv + ne
    nodes = np.concatenate([tets, nv + te], axis=1)  # [nt,10]
    G10 = node_grads(g)
    mt = mass_table()
    Me = density * vol[:, None, None] * mt[None]
    Ke = (1.0 / viscosity) * vol[:, None, None] * np.einsum("tia,tja->tij", G10, G10)
    rows = np.repeat(nodes, 10, axis=1).ravel()
    cols = np.tile(nodes, (1, 10)).ravel()
    M = sp.csr_matrix((Me.ravel(), (rows, cols)), shape=(N2, N2))
    K = sp.csr_matrix((Ke.ravel(), (rows, cols)), shape=(N2, N2))
    r4 = np.repeat(tets, 4, axis=1).ravel()
    c4 = np.tile(tets, (1, 4)).ravel()
    Gc = [sp.csr_matrix(((vol[:, None, None] / 4.0 * np.broadcast_to(g[:, None, :, c], (len(tets), 4, 4))).ravel(),
                         (r4, c4)), shape=(nv, nv)) for c in range(3)]
    Le = vol[:, None, None] * np.einsum("tia,tja->tij", g, g)
    L = sp.csr_matrix((Le.ravel(), (r4, c4)), shape=(nv, nv))
    rs = np.asarray(M.sum(axis=1)).ravel()
    invm = np.where(np.abs(rs) > 1e-14, 1.0 / np.where(rs == 0, 1, rs), 1.0)
    return dict(nv=nv, ne=ne, N2=N2, vol=vol, g=g, te=te, ids=ids, nodes=nodes, M=M, K=K,
                G=Gc, L=L, invm=invm)


def p2_tags(p1, ids, ne):
    p2 = np.full(ne, UNDEFINED, np.int64)
    for (a, b), k in ids.items():
        p2[k] = p1[a] if (p1[a] == p1[b] and p1[a] != INTERNAL) else INTERNAL
    return p2


def advection(A, tets, u):
    nv, N2 = A["nv"], A["N2"]
    g, vol = A["g"], A["vol"]
    uv = u[tets]  # [nt,4,3]
    ue = 0.25 * uv.sum(axis=1)
    gu = np.einsum("tja,tjb->tab", uv, g)
    c = np.einsum("tab,tb->ta", gu, ue)
    conv = np.zeros((N2, 3))
    np.add.at(conv, tets.ravel(), -np.repeat((vol / 4.0)[:, None] * c, 4, axis=0))
    np.add.at(conv, (nv + A["te"]).ravel(), -np.repeat((vol / 24.0)[:, None] * c, 6, axis=0))
    return conv


def divergence(A, tets, u):
    g, vol = A["g"], A["vol"]
    d = np.einsum("tja,tja->t", u[tets], g)
    out = np.zeros(A["nv"])
    np.add.at(out, tets.ravel(), np.repeat((vol / 4.0) * d, 4))
    return out


def piso_step(A, tets, bc, inlet, u, p, dt, relax_u=1.0, relax_p=1.0, outlet_type=0,
              outlet_pressure=0.0, ref_node=-1, n_corr=1):
    """One pisoStep with exact (direct) solves. bc: [N2] tags, inlet: [N2,3]."""
    nv, N2 = A["nv"], A["N2"]
    conv = advection(A, tets, u)
    dirich = (bc == INLET) | (bc == WALL)
    lhs = (A["M"] / dt + A["K"]).tolil()
    for i in np.nonzero(dirich)[0]:
        lhs[i, i] += 1e10
    lhs = lhs.tocsc()
    ustar = np.zeros((N2, 3))
    for c in range(3):
        rhs = A["M"] @ u[:, c] / dt
        rhs[:nv] -= A["G"][c] @ p
        rhs += conv[:, c]
        rhs[dirich] += 1e10 * np.where(bc[dirich] == INLET, inlet[dirich, c], 0.0)
        ustar[:, c] = spla.spsolve(lhs, rhs)
    p = p.copy()
    u_new = u.copy()
    pcorr = np.zeros(nv)
    Lbc = A["L"].tolil()
    rhs_base_pen = np.zeros(nv)
    if outlet_type == 1:
        if ref_node >= 0:
            Lbc[ref_node, ref_node] += 1e12
    else:
        for i in np.nonzero(bc[:nv] == OUTLET)[0]:
            Lbc[i, i] += 1e12
            rhs_base_pen[i] += 1e12 * outlet_pressure
    Lbc = Lbc.tocsc()
    for _ in range(n_corr):
        div = divergence(A, tets, ustar)
        rhs = -div / dt + rhs_base_pen
        pcorr = spla.spsolve(Lbc, rhs)
        p = p + relax_p * pcorr
        if outlet_type == 0:
            p[bc[:nv] == OUTLET] = outlet_pressure
        if ref_node >= 0:
            p = p - p[ref_node]
        gp = np.stack([A["G"][c] @ pcorr for c in range(3)], axis=1)
        u_new = ustar.copy()
        f = -dt * A["invm"][:nv]
        ok = A["invm"][:nv] > 1e-14
        u_new[:nv][ok] = ustar[:nv][ok] + relax_u * (f[ok, None] * gp[ok])
        u_new[bc == INLET] = inlet[bc == INLET]
        u_new[bc == WALL] = 0.0
    return u_new, ustar, p, pcorr


LOCAL_FACES = [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)]


def faces(xyz, tets):
    """Faces in sorted-triple order (src/Mesh/Mesh.cpp:494-530): (verts of tet_a's local face,
    tet_a, tet_b or -1), plus normal, area, center (src/Mesh/Mesh.cpp:460-469)."""
    fm = {}
    for t, v in enumerate(tets):
        for f, lf in enumerate(LOCAL_FACES):
            fv = tuple(int(v[k]) for k in lf)
            key = tuple(sorted(fv))
            if key not in fm:
                fm[key] = [fv, t, -1]
            else:
                fm[key][2] = t
    out = []
    for key in sorted(fm):
        fv, ta, tb = fm[key]
        a, b, c = xyz[list(fv)]
        ab, ac = b - a, c - a
        n = np.cross(ac, ab)
        n = n / np.linalg.norm(n)
        out.append((fv, ta, tb, n, 0.5 * np.linalg.norm(np.cross(ab, ac)), (a + b + c) / 3.0))
    return out


def setup_bc(xyz, tets, ids, ne, direction=(1.0, 0.0, 0.0), coverage=1.0):
    """Mesh::setupBoundaryConditions (src/Mesh/Mesh.cpp:325-417) + P2 rule."""
    mn, mx = xyz.min(axis=0), xyz.max(axis=0)
    size = mx - mn
    ax = 0
    if size[1] > size[0] and size[1] > size[2]:
        ax = 1
    elif size[2] > size[0] and size[2] > size[1]:
        ax = 2
    tol = size[ax] * 0.01 * coverage
    inlet_pos = mn[ax] if direction[ax] > 0 else mx[ax]
    outlet_pos = mx[ax] if direction[ax] > 0 else mn[ax]
    p1 = np.full(len(xyz), INTERNAL, np.int64)
    for fv, ta, tb, n, area, center in faces(xyz, tets):
        if tb != -1:
            continue
        p1[list(fv)] = WALL
        if abs(center[ax] - inlet_pos) < tol:
            p1[list(fv)] = INLET
        elif abs(center[ax] - outlet_pos) < tol:
            p1[list(fv)] = OUTLET
    return p1, p2_tags(p1, ids, ne)
