"""Python binding of the B200 P2/P1 PISO Navier-Stokes solver (ctypes over include/cfsa_ns.h
and include/cfsa_mesh.h).

The classes mirror the reference's C++ API so that scripts read like uses of
``NavierStokesSolver`` (include/FEM/NavierStokes.hpp:53-193) and ``Mesh``
(include/Mesh/Mesh.hpp:35-220): same method names, same argument meaning, ``bool`` results for
the step calls. All numerics run in lib/libcfsa.so on the GPU; there is no CPU fallback — a
missing library or a missing CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libcfsa.so"

# status codes (include/cfsa_ns.h)
OK, NOT_CONVERGED, BREAKDOWN, NAN, CUDA_ERROR, BAD_ARG, NOT_INITIALIZED, UNSUPPORTED = range(8)

MAT_MASS, MAT_STIFFNESS, MAT_GRAD_X, MAT_GRAD_Y, MAT_GRAD_Z, MAT_POISSON, MAT_MOMENTUM, MAT_POISSON_BC = range(8)
KERNEL_MOMENTUM_SPMV, KERNEL_PRESSURE_SPMV, KERNEL_PRESSURE_SOLVE, KERNEL_MOMENTUM_SPMV_F32 = 0, 1, 2, 3
KRYLOV_CG, KRYLOV_BICGSTAB, KRYLOV_CG1, KRYLOV_CG2L = 0, 1, 2, 3
PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED_FULL = 0, 1, 2
NORM_REFERENCE, NORM_JACOBI = 0, 1
OBJECTIVE_WALL_SHEAR, OBJECTIVE_PRESSURE_DROP = 0, 1
VTK_SHEAR_STRESS, VTK_PRESSURE_FORCES = 1, 2


class FluidBCType(enum.IntEnum):
    Wall = 0
    Inlet = 1
    Outlet = 2
    Internal = 3
    Undefined = 4


class OutletType(enum.IntEnum):
    DirichletPressure = 0
    Neumann = 1
    Undefined = 2


class InletType(enum.IntEnum):
    Uniform = 0
    Pulsitile = 1
    Undefined = 2


@dataclass
class Fluid:
    """include/FEM/NavierStokes.hpp:45-51"""

    density: float = 1000.0
    viscosity: float = 0.001
    effective_viscosity: list = field(default_factory=list)


class CfsaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[cfsa status {code}] {msg}")
        self.code = code


class _MeshView(C.Structure):
    _fields_ = [
        ("nv", C.c_int64), ("nt", C.c_int64), ("ne", C.c_int64),
        ("vertices", C.c_void_p), ("tets", C.c_void_p), ("tet_edges", C.c_void_p),
        ("p1_bc", C.c_void_p), ("p2_bc", C.c_void_p),
        ("nbf", C.c_int64), ("bface_verts", C.c_void_p), ("bface_tet", C.c_void_p),
        ("bface_normal", C.c_void_p), ("bface_area", C.c_void_p),
    ]


class _Fluid(C.Structure):
    _fields_ = [("density", C.c_double), ("viscosity", C.c_double)]


class Stats(C.Structure):
    _fields_ = [
        ("momentum_iters", C.c_int32 * 3), ("pressure_iters", C.c_int32),
        ("momentum_residual", C.c_double * 3), ("pressure_residual", C.c_double),
        ("momentum_outer", C.c_int32 * 3), ("pressure_outer", C.c_int32),
        ("steps", C.c_int64), ("time", C.c_double), ("last_step_ms", C.c_double),
        ("nnz_p2", C.c_int64), ("nnz_p1", C.c_int64),
        ("kernel_launches", C.c_int64), ("krylov_iters", C.c_int64 * 2),
        ("phase_ms", C.c_double * 3),
    ]

    def as_dict(self) -> dict:
        return {
            "momentum_iters": list(self.momentum_iters),
            "pressure_iters": int(self.pressure_iters),
            "momentum_residual": list(self.momentum_residual),
            "pressure_residual": float(self.pressure_residual),
            "momentum_outer": list(self.momentum_outer),
            "pressure_outer": int(self.pressure_outer),
            "steps": int(self.steps), "time": float(self.time),
            "last_step_ms": float(self.last_step_ms),
            "nnz_p2": int(self.nnz_p2), "nnz_p1": int(self.nnz_p1),
            "kernel_launches": int(self.kernel_launches),
            "krylov_iters": [int(x) for x in self.krylov_iters],
            "phase_ms": [float(x) for x in self.phase_ms],
        }


class Objective(C.Structure):
    """cfsa_objective: kind (OBJECTIVE_*), axis and [lo, hi] of a wall-shear patch."""

    _fields_ = [("kind", C.c_int32), ("axis", C.c_int32), ("lo", C.c_double), ("hi", C.c_double)]


class AdjointStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64), ("checkpoint_every", C.c_int32), ("checkpoints", C.c_int32),
        ("recomputed_steps", C.c_int64), ("momentum_iters", C.c_int64), ("pressure_iters", C.c_int64),
        ("forward_ms", C.c_double), ("backward_ms", C.c_double), ("record_bytes", C.c_int64),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: (float(getattr(self, k)) if t is C.c_double else int(getattr(self, k)))
                for k, t in self._fields_}


_LIB = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load lib/libcfsa.so (built by __graft_entry__.build() or `make` in this folder)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"CUDA extension not built: {p} is missing (run __graft_entry__.build())")
    lib = C.CDLL(str(p))
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    pp = C.POINTER(C.c_void_p)
    sig = {
        # mesh
        "cfsa_mesh_from_msh": (i32, [C.c_char_p, pp]),
        "cfsa_mesh_from_arrays": (i32, [i64, vp, i64, vp, pp]),
        "cfsa_mesh_structured_prism": (i32, [dbl, dbl, dbl, i32, i32, i32, pp]),
        "cfsa_mesh_cylinder": (i32, [dbl, dbl, i32, i32, pp]),
        "cfsa_mesh_y_bifurcation": (i32, [vp, pp]),
        "cfsa_mesh_setup_boundary_conditions": (i32, [vp, vp, dbl]),
        "cfsa_mesh_set_fluid_bc": (i32, [vp, vp, vp]),
        "cfsa_mesh_write_msh": (i32, [vp, C.c_char_p]),
        "cfsa_mesh_sizes": (i32, [vp, vp]),
        "cfsa_mesh_get_vertices": (i32, [vp, vp]),
        "cfsa_mesh_get_tets": (i32, [vp, vp]),
        "cfsa_mesh_get_tet_edges": (i32, [vp, vp]),
        "cfsa_mesh_get_edge_nodes": (i32, [vp, vp]),
        "cfsa_mesh_get_fluid_bc": (i32, [vp, vp, vp]),
        "cfsa_mesh_get_faces": (i32, [vp, vp, vp, vp]),
        "cfsa_mesh_get_tet_geometry": (i32, [vp, vp, vp]),
        "cfsa_mesh_destroy": (None, [vp]),
        "cfsa_mesh_last_error": (C.c_char_p, []),
        # solver
        "cfsa_ns_create": (i32, [vp, vp, pp]),
        "cfsa_ns_destroy": (None, [vp]),
        "cfsa_ns_last_error": (C.c_char_p, [vp]),
        "cfsa_ns_sizes": (i32, [vp, vp]),
        "cfsa_ns_set_dt": (i32, [vp, dbl]),
        "cfsa_ns_set_tolerances": (i32, [vp, dbl, dbl]),
        "cfsa_ns_set_max_iterations": (i32, [vp, i32, i32]),
        "cfsa_ns_set_num_corrections": (i32, [vp, i32]),
        "cfsa_ns_set_relaxation": (i32, [vp, dbl, dbl]),
        "cfsa_ns_set_outlet": (i32, [vp, i32, dbl]),
        "cfsa_ns_set_reference_node": (i32, [vp, i32]),
        "cfsa_ns_set_inlet_uniform": (i32, [vp, vp]),
        "cfsa_ns_set_inlet_profile": (i32, [vp, vp]),
        "cfsa_ns_set_pressure_solver": (i32, [vp, i32]),
        "cfsa_ns_set_momentum_solver": (i32, [vp, i32]),
        "cfsa_ns_get_velocity_async": (i32, [vp, vp]),
        "cfsa_ns_get_pressure_async": (i32, [vp, vp]),
        "cfsa_ns_wait_outputs": (i32, [vp]),
        "cfsa_ns_set_coarse_target": (i32, [vp, i32]),
        "cfsa_ns_save_state": (i32, [vp, C.c_char_p]),
        "cfsa_ns_load_state": (i32, [vp, C.c_char_p]),
        "cfsa_ns_get_coarse_size": (i32, [vp, vp]),
        "cfsa_ns_set_precision": (i32, [vp, i32]),
        "cfsa_ns_set_convergence_norm": (i32, [vp, i32]),
        "cfsa_ns_set_viscosity": (i32, [vp, dbl]),
        "cfsa_ns_initialize_fields": (i32, [vp]),
        "cfsa_ns_assemble": (i32, [vp]),
        "cfsa_ns_update_vertices": (i32, [vp, vp]),
        "cfsa_ns_update_boundary_tags": (i32, [vp, vp, vp]),
        "cfsa_ns_piso_step": (i32, [vp]),
        "cfsa_ns_piso_steps": (i32, [vp, i32, vp]),
        "cfsa_ns_simple_step": (i32, [vp]),
        "cfsa_ns_momentum_predictor": (i32, [vp]),
        "cfsa_ns_pressure_poisson": (i32, [vp]),
        "cfsa_ns_correct_velocity": (i32, [vp]),
        "cfsa_ns_get_velocity": (i32, [vp, vp]),
        "cfsa_ns_get_velocity_star": (i32, [vp, vp]),
        "cfsa_ns_get_pressure": (i32, [vp, vp]),
        "cfsa_ns_get_pressure_correction": (i32, [vp, vp]),
        "cfsa_ns_set_fields": (i32, [vp, vp, vp]),
        "cfsa_ns_get_time": (i32, [vp, vp]),
        "cfsa_ns_get_stats": (i32, [vp, vp]),
        "cfsa_ns_compute_divergence": (i32, [vp, vp, vp]),
        "cfsa_ns_compute_advection": (i32, [vp, vp]),
        "cfsa_ns_compute_shear_stress": (i32, [vp, vp]),
        "cfsa_ns_compute_pressure_forces": (i32, [vp, vp]),
        "cfsa_ns_compute_total_fluid_forces": (i32, [vp, vp]),
        "cfsa_ns_get_matrix_size": (i32, [vp, i32, vp, vp]),
        "cfsa_ns_get_matrix": (i32, [vp, i32, vp, vp, vp]),
        "cfsa_ns_get_inv_lumped_mass": (i32, [vp, vp]),
        "cfsa_ns_profile_kernel": (i32, [vp, i32, i32, vp, vp]),
        "cfsa_ns_set_barrier_spin_limit": (i32, [vp, C.c_int64]),
        "cfsa_ns_solve_pressure_bicgstab": (i32, [vp, vp, vp, dbl, i32]),
        "cfsa_ns_compute_divergence_noalloc": (i32, [vp, vp, vp]),
        "cfsa_ns_objective": (i32, [vp, vp, vp]),
        "cfsa_ns_write_vtk": (i32, [vp, C.c_char_p, C.c_double, i32]),
        "cfsa_ns_adjoint_forward": (i32, [vp, i32, i32, vp]),
        "cfsa_ns_adjoint_backward": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "cfsa_ns_adjoint_backward_seed": (i32, [vp, vp, vp, C.c_double, vp, vp, vp, vp]),
        "cfsa_ns_get_adjoint_stats": (i32, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


class Mesh:
    """Host mesh (include/Mesh/Mesh.hpp). Owns a cfsa_mesh handle."""

    def __init__(self, handle: int):
        self._lib = load_library()
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.cfsa_mesh_destroy(h)
            self._h = None

    def _check(self, code: int):
        if code != OK:
            raise CfsaError(code, self._lib.cfsa_mesh_last_error().decode())

    @classmethod
    def _make(cls, fn, *args) -> "Mesh":
        lib = load_library()
        out = C.c_void_p()
        code = getattr(lib, fn)(*args, C.byref(out))
        if code != OK:
            raise CfsaError(code, lib.cfsa_mesh_last_error().decode())
        return cls(out.value)

    @classmethod
    def cylinder(cls, length: float, radius: float, rings: int, layers: int) -> "Mesh":
        return cls._make("cfsa_mesh_cylinder", float(length), float(radius), int(rings), int(layers))

    @classmethod
    def yBifurcation(cls, parent_radius=2.0, parent_length=15.0, daughter_radius=1.5,
                     daughter_length=12.0, angle_deg=35.0, blend=0.5, cell=0.0813) -> "Mesh":
        """Y-bifurcation meshed on a Kuhn lattice of edge `cell`, tagged by the generator
        (inlet at x = 0, both daughter caps outlet, wall elsewhere)."""
        spec = np.array([parent_radius, parent_length, daughter_radius, daughter_length, angle_deg,
                         blend, cell], np.float64)
        return cls._make("cfsa_mesh_y_bifurcation", _ptr(spec))

    @classmethod
    def fromMshFile(cls, path) -> "Mesh":
        return cls._make("cfsa_mesh_from_msh", str(path).encode())

    @classmethod
    def fromArrays(cls, xyz, tets) -> "Mesh":
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        tets = _c(tets, np.int32).reshape(-1, 4)
        return cls._make("cfsa_mesh_from_arrays", len(xyz), _ptr(xyz), len(tets), _ptr(tets))

    @classmethod
    def structuredRectangularPrism(cls, length, width, height, nx=1, ny=1, nz=1) -> "Mesh":
        return cls._make("cfsa_mesh_structured_prism", float(length), float(width), float(height),
                         int(nx), int(ny), int(nz))

    def setupBoundaryConditions(self, direction=(1.0, 0.0, 0.0), coverage: float = 1.0):
        d = _c(direction, np.float64)
        self._check(self._lib.cfsa_mesh_setup_boundary_conditions(self._h, _ptr(d), float(coverage)))

    def setFluidBC(self, p1=None, p2=None):
        a = None if p1 is None else _c(p1, np.int8)
        b = None if p2 is None else _c(p2, np.int8)
        self._check(self._lib.cfsa_mesh_set_fluid_bc(self._h, None if a is None else _ptr(a),
                                                     None if b is None else _ptr(b)))

    def writeMshFile(self, path):
        self._check(self._lib.cfsa_mesh_write_msh(self._h, str(path).encode()))

    @property
    def sizes(self) -> tuple:
        s = np.zeros(5, np.int64)
        self._check(self._lib.cfsa_mesh_sizes(self._h, _ptr(s)))
        return tuple(int(x) for x in s)

    def nVertices(self):
        return self.sizes[0]

    def nTets(self):
        return self.sizes[1]

    def getNumberOfEdgeNodes(self):
        return self.sizes[2]

    def nFaces(self):
        return self.sizes[3]

    def vertices(self) -> np.ndarray:
        out = np.empty((self.sizes[0], 3))
        self._check(self._lib.cfsa_mesh_get_vertices(self._h, _ptr(out)))
        return out

    def tets(self) -> np.ndarray:
        out = np.empty((self.sizes[1], 4), np.int32)
        self._check(self._lib.cfsa_mesh_get_tets(self._h, _ptr(out)))
        return out

    def tetEdges(self) -> np.ndarray:
        out = np.empty((self.sizes[1], 6), np.int32)
        self._check(self._lib.cfsa_mesh_get_tet_edges(self._h, _ptr(out)))
        return out

    def edgeNodes(self) -> np.ndarray:
        out = np.empty((self.sizes[2], 3))
        self._check(self._lib.cfsa_mesh_get_edge_nodes(self._h, _ptr(out)))
        return out

    def fluidBC(self):
        s = self.sizes
        p1 = np.empty(s[0], np.int8)
        p2 = np.empty(s[2], np.int8)
        self._check(self._lib.cfsa_mesh_get_fluid_bc(self._h, _ptr(p1), _ptr(p2)))
        return p1, p2

    def faces(self):
        nf = self.sizes[3]
        v = np.empty((nf, 3), np.int32)
        t = np.empty((nf, 2), np.int32)
        g = np.empty((nf, 7))
        self._check(self._lib.cfsa_mesh_get_faces(self._h, _ptr(v), _ptr(t), _ptr(g)))
        return v, t, g

    def tetGeometry(self):
        nt = self.sizes[1]
        vol = np.empty(nt)
        grads = np.empty((nt, 4, 3))
        self._check(self._lib.cfsa_mesh_get_tet_geometry(self._h, _ptr(vol), _ptr(grads)))
        return vol, grads

    def nodePositions(self) -> np.ndarray:
        """P1 vertices followed by P2 edge nodes, [N2, 3]."""
        return np.concatenate([self.vertices(), self.edgeNodes()])


class NavierStokesSolver:
    """Mirror of the reference NavierStokesSolver class on the GPU C ABI.

    As in the reference, setters may be called before ``initialize``; the inlet velocity in
    effect at ``initialize`` seeds the inlet nodes of the initial field
    (src/FEM/NavierStokes.cpp:33-46) and a Neumann outlet picks the first Internal vertex as
    pressure reference when none was set (:51-67).
    """

    def __init__(self):
        self._lib = load_library()
        self._h = None
        self._mesh = None
        self.fluid = Fluid()
        self.dt = 1e-4
        self.tolerance = 1e-12  # reference default (NavierStokes.hpp:57)
        self.momentum_tol = 1e-6  # NavierStokes.cpp:500
        self.pressure_tol = 1e-8  # NavierStokes.cpp:635
        self.maxit = (1000, 1000)
        self.n_corrections = 1
        self.relax_u = 1.0
        self.relax_p = 1.0
        self.outlet_type = OutletType.DirichletPressure
        self.outlet_pressure = 0.0
        self.inlet_type = InletType.Uniform
        self.reference_node = -1
        self.mean_inlet_velocity = np.zeros(3)
        self.inlet_profile = None
        self.krylov = KRYLOV_BICGSTAB  # the reference's pressure method; CG variants opt-in
        self.momentum_krylov = KRYLOV_BICGSTAB  # the reference's momentum method; CG opt-in
        self.coarse_target = 256
        self.precision = PRECISION_FP64
        self.conv_norm = NORM_REFERENCE
        self.N2 = self.nv = self.ne = self.nt = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.cfsa_ns_destroy(h)
            self._h = None

    # ------------------------------------------------------------------ plumbing
    def _check(self, code: int):
        if code != OK:
            raise CfsaError(code, self._lib.cfsa_ns_last_error(self._h).decode())

    def _status(self, code: int) -> bool:
        if code in (CUDA_ERROR, BAD_ARG, UNSUPPORTED):
            raise CfsaError(code, self._lib.cfsa_ns_last_error(self._h).decode())
        return code == OK

    def _push_params(self):
        L, h = self._lib, self._h
        self._check(L.cfsa_ns_set_dt(h, float(self.dt)))
        self._check(L.cfsa_ns_set_tolerances(h, float(self.momentum_tol), float(self.pressure_tol)))
        self._check(L.cfsa_ns_set_max_iterations(h, int(self.maxit[0]), int(self.maxit[1])))
        self._check(L.cfsa_ns_set_num_corrections(h, int(self.n_corrections)))
        self._check(L.cfsa_ns_set_relaxation(h, float(self.relax_u), float(self.relax_p)))
        self._check(L.cfsa_ns_set_outlet(h, int(self.outlet_type), float(self.outlet_pressure)))
        self._check(L.cfsa_ns_set_reference_node(h, int(self.reference_node)))
        self._check(L.cfsa_ns_set_pressure_solver(h, int(self.krylov)))
        self._check(L.cfsa_ns_set_coarse_target(h, int(self.coarse_target)))
        self._check(L.cfsa_ns_set_precision(h, int(self.precision)))
        self._check(L.cfsa_ns_set_momentum_solver(h, int(self.momentum_krylov)))
        self._check(L.cfsa_ns_set_convergence_norm(h, int(self.conv_norm)))
        self._push_inlet()

    def _push_inlet(self):
        if self._h is None:
            return
        if self.inlet_profile is not None:
            prof = _c(self.inlet_profile, np.float64).reshape(self.N2, 3)
            self._check(self._lib.cfsa_ns_set_inlet_profile(self._h, _ptr(prof)))
        else:
            v = _c(self.mean_inlet_velocity, np.float64)
            self._check(self._lib.cfsa_ns_set_inlet_uniform(self._h, _ptr(v)))

    # ------------------------------------------------------------------ reference API
    def initialize(self, mesh: Mesh, fluid: Fluid):
        """NavierStokesSolver::initialize (src/FEM/NavierStokes.cpp:10-68)."""
        self._mesh = mesh
        self.fluid = fluid
        nv, nt, ne, nf, nb = mesh.sizes
        self.nv, self.nt, self.ne, self.N2 = nv, nt, ne, nv + ne
        self._arrays = {}
        xyz = mesh.vertices()
        tets = mesh.tets()
        edges = mesh.tetEdges()
        p1, p2 = mesh.fluidBC()
        fv, ft, fg = mesh.faces()
        bmask = ft[:, 1] == -1
        bverts = _c(fv[bmask], np.int32)
        btet = _c(ft[bmask, 0], np.int32)
        bnorm = _c(fg[bmask, 0:3], np.float64)
        barea = _c(fg[bmask, 3], np.float64)
        self._arrays = dict(xyz=xyz, tets=tets, edges=edges, p1=p1, p2=p2, bverts=bverts,
                            btet=btet, bnorm=bnorm, barea=barea)
        view = _MeshView(nv, nt, ne, _ptr(xyz), _ptr(tets), _ptr(edges), _ptr(p1), _ptr(p2),
                         len(bverts), _ptr(bverts), _ptr(btet), _ptr(bnorm), _ptr(barea))
        fl = _Fluid(float(fluid.density), float(fluid.viscosity))
        out = C.c_void_p()
        code = self._lib.cfsa_ns_create(C.byref(view), C.byref(fl), C.byref(out))
        if code != OK:
            raise CfsaError(code, self._lib.cfsa_ns_last_error(None).decode())
        self._h = out
        if self.reference_node < 0 and self.outlet_type == OutletType.Neumann:
            internal = np.nonzero(p1 == FluidBCType.Internal)[0]
            self.reference_node = int(internal[0]) if len(internal) else 0
        self._push_params()
        self._check(self._lib.cfsa_ns_initialize_fields(self._h))

    def build_sparse_matrices(self):
        self._check(self._lib.cfsa_ns_assemble(self._h))

    def pisoStep(self) -> bool:
        return self._status(self._lib.cfsa_ns_piso_step(self._h))

    def pisoSteps(self, n: int) -> tuple[bool, int]:
        done = C.c_int(0)
        ok = self._status(self._lib.cfsa_ns_piso_steps(self._h, int(n), C.byref(done)))
        return ok, done.value

    def simpleStep(self) -> bool:
        return self._status(self._lib.cfsa_ns_simple_step(self._h))

    def solveMomentumPredictor(self) -> bool:
        return self._status(self._lib.cfsa_ns_momentum_predictor(self._h))

    def solvePressurePoisson(self) -> bool:
        return self._status(self._lib.cfsa_ns_pressure_poisson(self._h))

    def correctVelocity(self) -> bool:
        return self._status(self._lib.cfsa_ns_correct_velocity(self._h))

    def solvePressureBiCGSTAB(self, rhs, x=None, tol: float = 1e-8, maxit: int = 1000):
        """solvePressureBiCGSTAB (NavierStokes.cpp:773-802): Jacobi BiCGSTAB on the raw Poisson
        matrix from a zero guess; returns (ok, x) with x the [nv] iterate."""
        b = np.ascontiguousarray(rhs, np.float64)
        if b.shape != (self.nv,):
            raise ValueError(f"rhs must have {self.nv} entries")
        out = np.empty(self.nv) if x is None else x
        ok = self._status(self._lib.cfsa_ns_solve_pressure_bicgstab(self._h, _ptr(b), _ptr(out), float(tol), int(maxit)))
        return ok, out

    def computeDivergence(self, u) -> np.ndarray:
        u = _c(u, np.float64).reshape(self.N2, 3)
        out = np.empty(self.nv)
        self._check(self._lib.cfsa_ns_compute_divergence(self._h, _ptr(u), _ptr(out)))
        return out

    def computeDivergenceNoAlloc(self, u_dev_ptr: int, div_dev_ptr: int) -> int:
        """Divergence on caller-owned device arrays (u [3][N2] component-major, div [nv]) with
        no device allocation; returns the C status code."""
        return self._lib.cfsa_ns_compute_divergence_noalloc(self._h, C.c_void_p(u_dev_ptr), C.c_void_p(div_dev_ptr))

    def computeAdvectionRHS(self) -> np.ndarray:
        out = np.empty((self.N2, 3))
        self._check(self._lib.cfsa_ns_compute_advection(self._h, _ptr(out)))
        return out

    def computeShearStress(self) -> np.ndarray:
        out = np.empty((self.nv, 3))
        self._check(self._lib.cfsa_ns_compute_shear_stress(self._h, _ptr(out)))
        return out

    def computePressureForces(self) -> np.ndarray:
        out = np.empty((self.nv, 3))
        self._check(self._lib.cfsa_ns_compute_pressure_forces(self._h, _ptr(out)))
        return out

    def computeTotalFluidForces(self) -> np.ndarray:
        out = np.empty((self.nv, 3))
        self._check(self._lib.cfsa_ns_compute_total_fluid_forces(self._h, _ptr(out)))
        return out

    # getters (NavierStokes.hpp:146-189)
    def getVelocity(self, out: np.ndarray | None = None) -> np.ndarray:
        """Velocity [N2, 3] (P1 vertices first). `out`: a C-contiguous float64 [N2, 3] array to
        fill instead of a new one (e.g. a pinned buffer for fast repeated reads)."""
        out = self._out((self.N2, 3), out)
        self._check(self._lib.cfsa_ns_get_velocity(self._h, _ptr(out)))
        return out

    def getVelocityAsync(self, out: np.ndarray) -> np.ndarray:
        """Stream-ordered read-back of u into `out` (C-contiguous float64 [N2, 3], ideally pinned):
        returns at once, the copy overlaps later steps; `out` is complete after waitOutputs()."""
        if out is None:
            raise ValueError("getVelocityAsync needs a caller-owned output array")
        out = self._out((self.N2, 3), out)
        self._check(self._lib.cfsa_ns_get_velocity_async(self._h, _ptr(out)))
        return out

    def getPressureAsync(self, out: np.ndarray) -> np.ndarray:
        """As getVelocityAsync for p ([nv])."""
        if out is None:
            raise ValueError("getPressureAsync needs a caller-owned output array")
        out = self._out((self.nv,), out)
        self._check(self._lib.cfsa_ns_get_pressure_async(self._h, _ptr(out)))
        return out

    def waitOutputs(self):
        """Wait for every stream-ordered read-back issued so far."""
        self._check(self._lib.cfsa_ns_wait_outputs(self._h))

    @staticmethod
    def _out(shape, out):
        if out is None:
            return np.empty(shape)
        if out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape {shape}")
        return out

    def getVelocityStar(self) -> np.ndarray:
        out = np.empty((self.N2, 3))
        self._check(self._lib.cfsa_ns_get_velocity_star(self._h, _ptr(out)))
        return out

    def getPressure(self, out: np.ndarray | None = None) -> np.ndarray:
        out = self._out((self.nv,), out)
        self._check(self._lib.cfsa_ns_get_pressure(self._h, _ptr(out)))
        return out

    def getPressureCorrection(self) -> np.ndarray:
        out = np.empty(self.nv)
        self._check(self._lib.cfsa_ns_get_pressure_correction(self._h, _ptr(out)))
        return out

    def getVelocityAtNode(self, i: int) -> np.ndarray:
        return self.getVelocity()[i]

    def getPressureAtNode(self, i: int) -> float:
        return float(self.getPressure()[i])

    def getTime(self) -> float:
        t = C.c_double()
        self._check(self._lib.cfsa_ns_get_time(self._h, C.byref(t)))
        return t.value

    def getDt(self):
        return self.dt

    def getViscosity(self):
        return self.fluid.viscosity

    def getDensity(self):
        return self.fluid.density

    def getTolerance(self):
        return self.tolerance

    def getMesh(self):
        return self._mesh

    def setFields(self, u=None, p=None):
        a = None if u is None else _c(u, np.float64).reshape(self.N2, 3)
        b = None if p is None else _c(p, np.float64).reshape(self.nv)
        self._check(self._lib.cfsa_ns_set_fields(self._h, None if a is None else _ptr(a),
                                                 None if b is None else _ptr(b)))

    def saveState(self, path: str):
        """Write u, p, time and step count to a binary restart file (new: the reference's VTK
        output cannot be read back)."""
        self._check(self._lib.cfsa_ns_save_state(self._h, os.fsencode(path)))

    def loadState(self, path: str):
        """Restore u, p, time and step count from saveState's file (same mesh sizes)."""
        self._check(self._lib.cfsa_ns_load_state(self._h, os.fsencode(path)))

    def stats(self) -> dict:
        s = Stats()
        self._check(self._lib.cfsa_ns_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def matrix(self, which: int):
        """CSR arrays (rowptr, cols, vals) of one assembled operator."""
        nr, nnz = C.c_int64(), C.c_int64()
        self._check(self._lib.cfsa_ns_get_matrix_size(self._h, int(which), C.byref(nr), C.byref(nnz)))
        rp = np.empty(nr.value + 1, np.int64)
        ci = np.empty(nnz.value, np.int32)
        va = np.empty(nnz.value)
        self._check(self._lib.cfsa_ns_get_matrix(self._h, int(which), _ptr(rp), _ptr(ci), _ptr(va)))
        return rp, ci, va

    def exportToVtk(self, filename, scale: float = 1.0, fields: int = 0):
        """io::exportToVtk(filename, solver, scale) (src/IO/VtkExport.cpp:238-268); `fields` adds
        VTK_SHEAR_STRESS / VTK_PRESSURE_FORCES vectors."""
        self._check(self._lib.cfsa_ns_write_vtk(self._h, str(filename).encode(), float(scale), int(fields)))

    # ---- discrete adjoint (forward / backward operator pair)
    def objective(self, kind: int = OBJECTIVE_WALL_SHEAR, axis: int = 0, lo: float = 0.0,
                  hi: float = 0.0) -> float:
        o = Objective(int(kind), int(axis), float(lo), float(hi))
        J = C.c_double()
        self._check(self._lib.cfsa_ns_objective(self._h, C.byref(o), C.byref(J)))
        return J.value

    def adjointForward(self, nsteps: int, checkpoint_every: int = 0) -> bool:
        """nsteps PISO steps recorded for the backward pass (checkpoint_every <= 0: automatic)."""
        done = C.c_int()
        return self._status(self._lib.cfsa_ns_adjoint_forward(self._h, int(nsteps), int(checkpoint_every),
                                                              C.byref(done)))

    def adjointBackward(self, kind: int = OBJECTIVE_WALL_SHEAR, axis: int = 0, lo: float = 0.0,
                        hi: float = 0.0) -> dict:
        """J and its gradients: grad_inlet [N2, 3], grad_viscosity, grad_u0 [N2, 3], grad_p0 [nv]."""
        o = Objective(int(kind), int(axis), float(lo), float(hi))
        J, gnu = C.c_double(), C.c_double()
        gin = np.empty((self.N2, 3))
        gu0 = np.empty((self.N2, 3))
        gp0 = np.empty(self.nv)
        self._check(self._lib.cfsa_ns_adjoint_backward(self._h, C.byref(o), C.byref(J), _ptr(gin),
                                                       C.byref(gnu), _ptr(gu0), _ptr(gp0)))
        return dict(J=J.value, grad_inlet=gin, grad_viscosity=gnu.value, grad_u0=gu0, grad_p0=gp0)

    def adjointBackwardSeed(self, dJ_du=None, dJ_dp=None, dJ_dviscosity: float = 0.0) -> dict:
        """Backward pass from a caller seed (dJ/du^N [N2, 3], dJ/dp^N [nv], explicit dJ/dnu)."""
        du = None if dJ_du is None else _c(dJ_du, np.float64).reshape(self.N2, 3)
        dp = None if dJ_dp is None else _c(dJ_dp, np.float64).reshape(self.nv)
        gnu = C.c_double()
        gin = np.empty((self.N2, 3))
        gu0 = np.empty((self.N2, 3))
        gp0 = np.empty(self.nv)
        self._check(self._lib.cfsa_ns_adjoint_backward_seed(
            self._h, None if du is None else _ptr(du), None if dp is None else _ptr(dp),
            float(dJ_dviscosity), _ptr(gin), C.byref(gnu), _ptr(gu0), _ptr(gp0)))
        return dict(grad_inlet=gin, grad_viscosity=gnu.value, grad_u0=gu0, grad_p0=gp0)

    def adjointStats(self) -> dict:
        s = AdjointStats()
        self._check(self._lib.cfsa_ns_get_adjoint_stats(self._h, C.byref(s)))
        return s.as_dict()

    def profileKernel(self, which: int, iters: int = 50) -> tuple[float, float]:
        """(mean launch ms, algorithmic bytes per launch) of one step kernel on live data."""
        ms, by = C.c_double(), C.c_double()
        self._check(self._lib.cfsa_ns_profile_kernel(self._h, int(which), int(iters), C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def setBarrierSpinLimit(self, polls: int):
        """Polls a waiting CTA of the resident pressure solvers makes at a grid barrier before it
        gives up (the step then fails with CUDA_ERROR); < 0 restores the default."""
        self._check(self._lib.cfsa_ns_set_barrier_spin_limit(self._h, int(polls)))

    def invLumpedMass(self) -> np.ndarray:
        out = np.empty(self.N2)
        self._check(self._lib.cfsa_ns_get_inv_lumped_mass(self._h, _ptr(out)))
        return out

    # setters (NavierStokes.hpp:166-186)
    def setMeanInletVelocity(self, v):
        self.mean_inlet_velocity = np.asarray(v, np.float64).reshape(3)
        self.inlet_profile = None
        self._push_inlet()

    def setInletVelocityProfile(self, per_node):
        """Per-node inlet velocity [N2, 3] (new; the reference has only a uniform inlet)."""
        self.inlet_profile = np.asarray(per_node, np.float64).reshape(-1, 3)
        self._push_inlet()

    def setOutletType(self, t):
        self.outlet_type = OutletType(t)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_outlet(self._h, int(self.outlet_type), float(self.outlet_pressure)))

    def setOutletPressure(self, p):
        self.outlet_pressure = float(p)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_outlet(self._h, int(self.outlet_type), float(self.outlet_pressure)))

    def setInletType(self, t):
        self.inlet_type = InletType(t)

    def setNumberOfCorrections(self, n):
        self.n_corrections = int(n)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_num_corrections(self._h, self.n_corrections))

    def setRelaxU(self, r):
        self.relax_u = float(r)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_relaxation(self._h, self.relax_u, self.relax_p))

    def setRelaxP(self, r):
        self.relax_p = float(r)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_relaxation(self._h, self.relax_u, self.relax_p))

    def setReferencePressureNode(self, n):
        self.reference_node = int(n)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_reference_node(self._h, self.reference_node))

    def setDt(self, dt):
        self.dt = float(dt)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_dt(self._h, self.dt))

    def setTolerance(self, tol):
        """Routed to both Krylov solves (the reference stores it but solves with fixed
        1e-6 / 1e-8, NavierStokes.cpp:500,635)."""
        self.tolerance = float(tol)
        self.setKrylovTolerances(tol, tol)

    def setKrylovTolerances(self, momentum, pressure):
        self.momentum_tol, self.pressure_tol = float(momentum), float(pressure)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_tolerances(self._h, self.momentum_tol, self.pressure_tol))

    def setMaxIterations(self, momentum, pressure):
        self.maxit = (int(momentum), int(pressure))
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_max_iterations(self._h, *self.maxit))

    def setMomentumSolver(self, krylov: int):
        """Momentum Krylov method: KRYLOV_BICGSTAB (the reference's) or KRYLOV_CG (Jacobi CG on the
        same symmetric positive definite system, one product per iteration; FP64 only)."""
        self.momentum_krylov = int(krylov)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_momentum_solver(self._h, self.momentum_krylov))

    def setPressureSolver(self, krylov: int):
        """Pressure Krylov method: KRYLOV_BICGSTAB (the reference's), KRYLOV_CG, KRYLOV_CG1
        (one reduction per iteration) or KRYLOV_CG2L (KRYLOV_CG1 with the two-level
        Jacobi + aggregation coarse-correction preconditioner, the fastest)."""
        self.krylov = int(krylov)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_pressure_solver(self._h, self.krylov))

    def setCoarseTarget(self, target: int):
        """Aggregate count of the KRYLOV_CG2L coarse space (default 256)."""
        self.coarse_target = int(target)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_coarse_target(self._h, self.coarse_target))

    def coarseSize(self) -> int:
        """Aggregates of the current KRYLOV_CG2L coarse space (0 for the other methods)."""
        nc = C.c_int()
        self._check(self._lib.cfsa_ns_get_coarse_size(self._h, C.byref(nc)))
        return nc.value

    def setPrecision(self, precision: int):
        self.precision = int(precision)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_precision(self._h, self.precision))

    def setConvergenceNorm(self, norm: int):
        """NORM_REFERENCE (||r||/||b||, the reference's) or NORM_JACOBI (||D^-1/2 r||/||D^-1/2 b||)."""
        self.conv_norm = int(norm)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_convergence_norm(self._h, self.conv_norm))

    def setViscosity(self, nu: float):
        self.fluid.viscosity = float(nu)
        if self._h is not None:
            self._check(self._lib.cfsa_ns_set_viscosity(self._h, float(nu)))

    def updateVertices(self, xyz):
        xyz = _c(xyz, np.float64).reshape(self.nv, 3)
        self._check(self._lib.cfsa_ns_update_vertices(self._h, _ptr(xyz)))


def parabolic_inlet(nodes: np.ndarray, peak: float, radius: float, axis: int = 0) -> np.ndarray:
    """u_axis(r) = peak * (1 - r^2 / R^2) on a circular inlet centred on the axis through the
    origin; other components zero. `nodes` is [N2, 3] (P1 then P2 node positions)."""
    other = [a for a in range(3) if a != axis]
    r2 = nodes[:, other[0]] ** 2 + nodes[:, other[1]] ** 2
    out = np.zeros_like(nodes)
    out[:, axis] = peak * (1.0 - r2 / (radius * radius))
    return out
