"""ctypes wrapper of the CPU oracle (oracle/ns_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker and by
bench.py's CPU-baseline leg. The product path never loads it. Parity is unpinned: the reference
cannot be compiled here (Eigen, yaml-cpp and TetGen are absent) and ships no golden vectors.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle_ns.so"

MAT = {"M": 0, "K": 1, "Gx": 2, "Gy": 3, "Gz": 4, "L": 5}
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    L = C.CDLL(str(LIB))
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    sig = {
        "orc_create": (vp, [i64, vp, i64, vp, i32, vp, dbl]),
        "orc_destroy": (None, [vp]),
        "orc_sizes": (None, [vp, vp]),
        "orc_get_mesh": (None, [vp] + [vp] * 9),
        "orc_set_bc": (None, [vp, vp, vp]),
        "orc_set_fluid": (None, [vp, dbl, dbl]),
        "orc_set_params": (None, [vp, dbl, dbl, dbl, i32, i32, i32, dbl, dbl, i32, dbl, i32, i32, i32]),
        "orc_set_inlet": (None, [vp, vp]),
        "orc_set_coarse_target": (i32, [vp, i32]),
        "orc_set_momentum_solver": (i32, [vp, i32]),
        "orc_coarse_size": (i32, [vp]),
        "orc_initialize": (None, [vp]),
        "orc_reference_node": (i32, [vp]),
        "orc_piso_step": (i32, [vp]),
        "orc_simple_step": (i32, [vp]),
        "orc_momentum": (i32, [vp]),
        "orc_pressure": (i32, [vp]),
        "orc_correct": (i32, [vp]),
        "orc_get_state": (None, [vp, vp, vp, vp, vp, vp]),
        "orc_set_state": (None, [vp, vp, vp]),
        "orc_matrix_nnz": (i64, [vp, i32, vp]),
        "orc_get_matrix": (None, [vp, i32, vp, vp, vp]),
        "orc_get_inv_lumped_mass": (None, [vp, vp]),
        "orc_advection": (None, [vp, vp]),
        "orc_divergence": (None, [vp, vp, vp]),
        "orc_pressure_forces": (None, [vp, vp]),
        "orc_shear_stress": (None, [vp, vp]),
        "orc_stats": (None, [vp, vp, vp, vp]),
        "orc_set_threads": (i32, [i32]),
        "orc_cylinder": (i32, [dbl, dbl, i32, i32, vp, vp]),
        "orc_solve_poisson_raw": (i32, [vp, vp, vp, dbl, i32, vp]),
        "orc_adjoint_forward": (i32, [vp, i32]),
        "orc_objective": (i32, [vp, i32, i32, dbl, dbl, vp, vp, vp, vp]),
        "orc_adjoint_backward": (i32, [vp, vp, vp, dbl, vp, vp, vp]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a
    _lib = L
    return L


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def cylinder(length: float, radius: float, rings: int, layers: int):
    """Synthetic cylinder along x (vertices [nv][3], tets [nt][4]): the same arrays as the
    product's procedural mesher, built here so that CPU runs of the oracle load no product
    library."""
    np_disk = 1 + 3 * rings * (rings + 1)
    xyz = np.empty((np_disk * (layers + 1), 3), np.float64)
    tets = np.empty((18 * rings * rings * layers, 4), np.int32)
    if lib().orc_cylinder(float(length), float(radius), int(rings), int(layers), _p(xyz), _p(tets)) != 0:
        raise ValueError("cylinder: rings, layers >= 1 and positive length/radius required")
    return xyz, tets


def parabolic_inlet(o: "Oracle", peak: float, radius: float, axis: int = 0) -> np.ndarray:
    """u_axis = peak (1 - r^2 / R^2) at every P1 vertex and P2 edge node of the oracle mesh, r the
    distance from the axis through the origin; other components zero. [N2, 3]."""
    nodes = np.concatenate([o.vertices, o.mesh()["edge_xyz"]])
    other = [a for a in range(3) if a != axis]
    r2 = nodes[:, other[0]] ** 2 + nodes[:, other[1]] ** 2
    out = np.zeros_like(nodes)
    out[:, axis] = peak * (1.0 - r2 / (radius * radius))
    return out


class Oracle:
    """FP64 CPU restatement of the reference NavierStokesSolver on a raw (xyz, tets) mesh."""

    def __init__(self, xyz, tets, direction=(1.0, 0.0, 0.0), coverage=1.0, apply_bc=True):
        self.L = lib()
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        tets = np.ascontiguousarray(tets, np.int32).reshape(-1, 4)
        self.vertices = xyz
        d = np.ascontiguousarray(direction, np.float64)
        self.h = C.c_void_p(self.L.orc_create(len(xyz), _p(xyz), len(tets), _p(tets),
                                              1 if apply_bc else 0, _p(d), float(coverage)))
        s = np.zeros(5, np.int64)
        self.L.orc_sizes(self.h, _p(s))
        self.nv, self.nt, self.ne, self.nf, self.nbf = (int(x) for x in s)
        self.N2 = self.nv + self.ne
        self.params = dict(dt=1e-4, tol_mom=1e-6, tol_p=1e-8, maxit_mom=1000, maxit_p=1000,
                           n_corr=1, relax_u=1.0, relax_p=1.0, outlet_type=0,
                           outlet_pressure=0.0, reference_node=-1, pressure_solver=0, conv_norm=0)

    def __del__(self):
        if getattr(self, "h", None) is not None:
            self.L.orc_destroy(self.h)
            self.h = None

    def mesh(self) -> dict:
        nt, nv, ne, nf = self.nt, self.nv, self.ne, self.nf
        out = dict(tet_edges=np.empty((nt, 6), np.int32), p1=np.empty(nv, np.int32),
                   p2=np.empty(ne, np.int32), face_verts=np.empty((nf, 3), np.int32),
                   face_tets=np.empty((nf, 2), np.int32), face_geom=np.empty((nf, 7)),
                   vol=np.empty(nt), grads=np.empty((nt, 4, 3)), edge_xyz=np.empty((ne, 3)))
        self.L.orc_get_mesh(self.h, *(_p(out[k]) for k in (
            "tet_edges", "p1", "p2", "face_verts", "face_tets", "face_geom", "vol", "grads", "edge_xyz")))
        return out

    def set_bc(self, p1, p2):
        a = np.ascontiguousarray(p1, np.int32)
        b = np.ascontiguousarray(p2, np.int32)
        self.L.orc_set_bc(self.h, _p(a), _p(b))

    def set_fluid(self, density, viscosity):
        self.L.orc_set_fluid(self.h, float(density), float(viscosity))

    def set_params(self, **kw):
        self.params.update(kw)
        p = self.params
        self.L.orc_set_params(self.h, float(p["dt"]), float(p["tol_mom"]), float(p["tol_p"]),
                              int(p["maxit_mom"]), int(p["maxit_p"]), int(p["n_corr"]),
                              float(p["relax_u"]), float(p["relax_p"]), int(p["outlet_type"]),
                              float(p["outlet_pressure"]), int(p["reference_node"]),
                              int(p["pressure_solver"]), int(p["conv_norm"]))

    def set_momentum_solver(self, solver: int):
        """0: BiCGSTAB (the reference's), 1: Jacobi CG on the same system (as the device's
        CFSA_KRYLOV_CG momentum method)."""
        if self.L.orc_set_momentum_solver(self.h, int(solver)) != 0:
            raise ValueError(f"unknown momentum solver {solver}")

    def set_coarse_target(self, target: int):
        """Aggregate count the two-level pressure preconditioner (pressure_solver 3) aims for,
        1..1024 as on the device."""
        if self.L.orc_set_coarse_target(self.h, int(target)) != 0:
            raise ValueError(f"coarse target {target} outside [1, 1024]")

    def solve_poisson_raw(self, rhs, tol=1e-8, maxit=1000):
        """solvePressureBiCGSTAB: (converged, x, iterations) of Jacobi BiCGSTAB on the raw Poisson
        matrix (no boundary penalty) from a zero guess."""
        b = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros(self.nv)
        it = C.c_int(0)
        code = self.L.orc_solve_poisson_raw(self.h, _p(b), _p(x), float(tol), int(maxit), C.byref(it))
        return code == 0, x, it.value

    def coarse_size(self) -> int:
        return self.L.orc_coarse_size(self.h)

    def set_inlet(self, per_node):
        v = np.ascontiguousarray(per_node, np.float64).reshape(self.N2, 3)
        self.L.orc_set_inlet(self.h, _p(v))

    def initialize(self):
        self.L.orc_initialize(self.h)

    def reference_node(self) -> int:
        return self.L.orc_reference_node(self.h)

    def piso_step(self) -> int:
        return self.L.orc_piso_step(self.h)

    def simple_step(self) -> int:
        return self.L.orc_simple_step(self.h)

    def momentum(self) -> int:
        return self.L.orc_momentum(self.h)

    def pressure(self) -> int:
        return self.L.orc_pressure(self.h)

    def correct(self) -> int:
        return self.L.orc_correct(self.h)

    def state(self) -> dict:
        u = np.empty((self.N2, 3))
        us = np.empty((self.N2, 3))
        p = np.empty(self.nv)
        pc = np.empty(self.nv)
        t = C.c_double()
        self.L.orc_get_state(self.h, _p(u), _p(us), _p(p), _p(pc), C.addressof(t))
        return dict(u=u, ustar=us, p=p, pcorr=pc, time=t.value)

    def set_state(self, u, p):
        u = np.ascontiguousarray(u, np.float64).reshape(self.N2, 3)
        p = np.ascontiguousarray(p, np.float64).reshape(self.nv)
        self.L.orc_set_state(self.h, _p(u), _p(p))

    def matrix(self, name: str):
        which = MAT[name]
        nr = C.c_int64()
        nnz = self.L.orc_matrix_nnz(self.h, which, C.addressof(nr))
        rp = np.empty(nr.value + 1, np.int64)
        ci = np.empty(nnz, np.int32)
        va = np.empty(nnz)
        self.L.orc_get_matrix(self.h, which, _p(rp), _p(ci), _p(va))
        return rp, ci, va

    def inv_lumped_mass(self):
        out = np.empty(self.N2)
        self.L.orc_get_inv_lumped_mass(self.h, _p(out))
        return out

    def advection(self):
        out = np.empty((self.N2, 3))
        self.L.orc_advection(self.h, _p(out))
        return out

    def divergence(self, u):
        u = np.ascontiguousarray(u, np.float64).reshape(self.N2, 3)
        out = np.empty(self.nv)
        self.L.orc_divergence(self.h, _p(u), _p(out))
        return out

    def pressure_forces(self):
        out = np.empty((self.nv, 3))
        self.L.orc_pressure_forces(self.h, _p(out))
        return out

    def shear_stress(self):
        out = np.empty((self.nv, 3))
        self.L.orc_shear_stress(self.h, _p(out))
        return out

    # ---- discrete adjoint
    def adjoint_forward(self, nsteps: int) -> int:
        return self.L.orc_adjoint_forward(self.h, int(nsteps))

    def objective(self, kind=0, axis=0, lo=0.0, hi=0.0):
        """(J, dJ/du [N2,3], dJ/dp [nv], explicit dJ/dviscosity) on the current state."""
        J = C.c_double()
        dnu = C.c_double()
        su = np.zeros((self.N2, 3))
        sp = np.zeros(self.nv)
        rc = self.L.orc_objective(self.h, int(kind), int(axis), float(lo), float(hi),
                                  C.addressof(J), _p(su), _p(sp), C.addressof(dnu))
        if rc:
            raise ValueError("objective vertex set is empty")
        return J.value, su, sp, dnu.value

    def adjoint_backward(self, seed_u, seed_p, dnu_explicit=0.0) -> dict:
        lu = np.ascontiguousarray(seed_u, np.float64).reshape(self.N2, 3).copy()
        lp = np.ascontiguousarray(seed_p, np.float64).reshape(self.nv).copy()
        gin = np.zeros((self.N2, 3))
        gnu = C.c_double()
        it = np.zeros(2, np.int32)
        rc = self.L.orc_adjoint_backward(self.h, _p(lu), _p(lp), float(dnu_explicit), _p(gin),
                                         C.addressof(gnu), _p(it))
        return dict(rc=rc, grad_inlet=gin, grad_viscosity=gnu.value, grad_u0=lu, grad_p0=lp,
                    iters=it.tolist())

    def stats(self) -> dict:
        it = np.zeros(4, np.int32)
        res = np.zeros(4)
        times = np.zeros(5)
        self.L.orc_stats(self.h, _p(it), _p(res), _p(times))
        return dict(momentum_iters=it[:3].tolist(), pressure_iters=int(it[3]),
                    momentum_residual=res[:3].tolist(), pressure_residual=float(res[3]),
                    t_assembly=times[0], t_conv=times[1], t_momentum=times[2],
                    t_pressure=times[3], t_correct=times[4])
