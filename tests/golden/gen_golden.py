"""Generates the golden fixtures in this folder from the independent numpy restatement
(numpy_restatement.py). Run from the repository root:  python tests/golden/gen_golden.py

Fixtures:
  prism6.npz    1x1x1 structured prism (6 tets, src/Mesh/Mesh.cpp:146-225): dense M, K, Gx, Gy,
                Gz, L and 1/rowsum(M) for density 1000, viscosity 0.001 (the reference defaults).
  cyl_piso.npz  small cylinder (L=30, R=2, 2 rings, 4 layers): tags and three pisoStep states
                (exact solves) for rho=1060, nu=0.004, dt=0.01, plug inlet 0.5 set after
                initialize (the reference's CLI order), Dirichlet p=0 outlet.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import numpy_restatement as nr  # noqa: E402


def prism6():
    xyz = np.array([[i, j, k] for k in (0.0, 1.0) for j in (0.0, 1.0) for i in (0.0, 1.0)])
    v = list(range(8))
    tets = np.array([[v[0], v[1], v[3], v[7]], [v[0], v[3], v[2], v[7]], [v[0], v[2], v[6], v[7]],
                     [v[0], v[6], v[4], v[7]], [v[0], v[4], v[5], v[7]], [v[0], v[5], v[1], v[7]]])
    A = nr.assemble(xyz, tets, 1000.0, 0.001)
    np.savez(HERE / "prism6.npz", xyz=xyz, tets=tets, M=A["M"].toarray(), K=A["K"].toarray(),
             Gx=A["G"][0].toarray(), Gy=A["G"][1].toarray(), Gz=A["G"][2].toarray(),
             L=A["L"].toarray(), invm=A["invm"], te=A["te"])


def cylinder_points(length, radius, rings, layers):
    """Same construction as Mesh::generateCylinder (for an independent fixture mesh)."""
    disk = [(0.0, 0.0)]
    starts, sizes = [0], [1]
    for k in range(1, rings + 1):
        starts.append(len(disk))
        m = 6 * k
        sizes.append(m)
        r = radius * k / rings
        for j in range(m):
            th = 2.0 * np.pi * j / m
            disk.append((r * np.cos(th), r * np.sin(th)))
    tris = []
    for k in range(1, rings + 1):
        ma, mb, sa, sb = sizes[k - 1], sizes[k], starts[k - 1], starts[k]
        i = j = 0
        while i < ma or j < mb:
            na = 2.0 if k == 1 else (i + 1) / ma
            nb = (j + 1) / mb
            adv_in = (j >= mb) or (i < ma and k > 1 and na < nb)
            if adv_in:
                tris.append((sa + i % ma, sb + j % mb, sa + (i + 1) % ma))
                i += 1
            else:
                tris.append((sa + i % ma, sb + j % mb, sb + (j + 1) % mb))
                j += 1
            if k == 1 and j >= mb:
                break
    np_ = len(disk)
    xyz = np.array([(length * l / layers, y, z) for l in range(layers + 1) for (y, z) in disk])
    perm = [(0, 1, 2, 3, 4, 5), (1, 2, 0, 4, 5, 3), (2, 0, 1, 5, 3, 4), (3, 5, 4, 0, 2, 1),
            (4, 3, 5, 1, 0, 2), (5, 4, 3, 2, 1, 0)]
    tets = []
    for l in range(layers):
        for tr in tris:
            P = [l * np_ + tr[a] for a in range(3)] + [(l + 1) * np_ + tr[a] for a in range(3)]
            imin = int(np.argmin(P))
            V = [P[perm[imin][a]] for a in range(6)]
            if min(V[1], V[5]) < min(V[2], V[4]):
                out = [(V[0], V[1], V[2], V[5]), (V[0], V[1], V[5], V[4]), (V[0], V[4], V[5], V[3])]
            else:
                out = [(V[0], V[1], V[2], V[4]), (V[0], V[4], V[2], V[5]), (V[0], V[4], V[5], V[3])]
            for c in out:
                a, b, cc, d = xyz[list(c)]
                det = np.dot(np.cross(b - a, cc - a), d - a)
                tets.append((c[0], c[1], c[3], c[2]) if det < 0 else c)
    return xyz, np.array(tets)


def cyl_piso():
    xyz, tets = cylinder_points(30.0, 2.0, 2, 4)
    A = nr.assemble(xyz, tets, 1060.0, 0.004)
    p1, p2 = nr.setup_bc(xyz, tets, A["ids"], A["ne"])
    bc = np.concatenate([p1, p2])
    inlet = np.zeros((A["N2"], 3))
    inlet[:, 0] = 0.5
    u = np.zeros((A["N2"], 3))  # initialize() ran with a zero inlet
    p = np.zeros(A["nv"])
    states = []
    for _ in range(3):
        u, ustar, p, pc = nr.piso_step(A, tets, bc, inlet, u, p, 0.01)
        states.append((u.copy(), ustar.copy(), p.copy(), pc.copy()))
    np.savez(HERE / "cyl_piso.npz", xyz=xyz, tets=tets, p1=p1, p2=p2, te=A["te"],
             u=np.stack([s[0] for s in states]), ustar=np.stack([s[1] for s in states]),
             p=np.stack([s[2] for s in states]), pcorr=np.stack([s[3] for s in states]),
             conv0=nr.advection(A, tets, states[0][0]), div0=nr.divergence(A, tets, states[0][1]))


if __name__ == "__main__":
    prism6()
    cyl_piso()
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))
