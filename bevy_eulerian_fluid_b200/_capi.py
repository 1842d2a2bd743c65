"""ctypes mirror of include/efl.h and a thin handle wrapper.

`load()` opens the in-tree libefl_b200.so and fails loudly when it is
missing or unusable: there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libefl_b200.so")

MAX_SOLIDS = 256
MAX_FLUID_SOURCE = 16

# efl_status
OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_OUT_OF_MEMORY, NOT_CONVERGED, ERR_TOO_MANY, \
    ERR_UNSUPPORTED_SHAPE, ERR_STATE, ERR_NO_DEVICE = range(9)
STATUS_NAMES = {0: "EFL_OK", 1: "EFL_ERR_INVALID_ARGUMENT", 2: "EFL_ERR_CUDA", 3: "EFL_ERR_OUT_OF_MEMORY",
                4: "EFL_NOT_CONVERGED", 5: "EFL_ERR_TOO_MANY", 6: "EFL_ERR_UNSUPPORTED_SHAPE",
                7: "EFL_ERR_STATE", 8: "EFL_ERR_NO_DEVICE"}

PROJECTION_JACOBI, PROJECTION_GAUSS_SEIDEL, PROJECTION_MULTIGRID, PROJECTION_MGPCG = 0, 1, 2, 3
REINIT_JUMP_FLOODING, REINIT_FAST_ITERATIVE = 0, 1
SHAPE_CIRCLE, SHAPE_RECTANGLE, SHAPE_CAPSULE, SHAPE_TRIANGLE = 0, 1, 2, 4
SOURCE_CIRCLE, SOURCE_AABB = 0, 1
SOURCE_MODE_SOURCE, SOURCE_MODE_SINK = 0, 1

# efl_field
(FIELD_U, FIELD_V, FIELD_U1, FIELD_V1, FIELD_U_SOLID, FIELD_V_SOLID, FIELD_LEVELSET_AIR,
 FIELD_LEVELSET_AIR1, FIELD_LEVELSET_SOLID, FIELD_SOLID_ID, FIELD_AREA_FRACTION, FIELD_DIVERGENCE,
 FIELD_PRESSURE, FIELD_GRAD_LEVELSET, FIELD_JFA_SEEDS, FIELD_FIM_LABELS, FIELD_U_VALID, FIELD_V_VALID,
 FIELD_AREA_FRACTION_U, FIELD_AREA_FRACTION_V) = range(20)
FIELD_DTYPES = {FIELD_SOLID_ID: np.int32, FIELD_U_VALID: np.int32, FIELD_V_VALID: np.int32,
                FIELD_FIM_LABELS: np.uint32}

# efl_stage
(STAGE_INIT, STAGE_UPDATE_SOLID, STAGE_AREA_FRACTION, STAGE_ADVECT_VELOCITY, STAGE_APPLY_FORCES,
 STAGE_DIVERGENCE, STAGE_PROJECTION, STAGE_SOLVE_VELOCITY, STAGE_EXTRAPOLATE, STAGE_ADVECT_LEVELSET,
 STAGE_FLUID_SOURCE, STAGE_REINITIALIZE, STAGE_LEVELSET_GRADIENT, STAGE_SOLID_FORCES) = range(14)


class Projection(C.Structure):
    _fields_ = [("method", C.c_int32), ("gs_iterations", C.c_uint32), ("sor_weight", C.c_float),
                ("mg_pre", C.c_uint32), ("mg_post", C.c_uint32), ("mg_coarsest", C.c_uint32),
                ("mg_levels", C.c_uint32), ("tolerance", C.c_float), ("max_iterations", C.c_uint32),
                ("check_interval", C.c_uint32)]


class Reinit(C.Structure):
    _fields_ = [("method", C.c_int32), ("fim_iterations", C.c_uint32)]


class Config(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("length_unit", C.c_float), ("rho", C.c_float),
                ("gravity", C.c_float * 2), ("transform", C.c_float * 16), ("projection", Projection),
                ("reinit", Reinit), ("device", C.c_int32)]


class SolidObstacle(C.Structure):
    _fields_ = [("entity_id", C.c_uint32), ("shape", C.c_uint32), ("values", C.c_float * 6),
                ("transform", C.c_float * 16), ("inverse_transform", C.c_float * 16),
                ("linear_velocity", C.c_float * 2), ("angular_velocity", C.c_float), ("_pad", C.c_float)]


class Force(C.Structure):
    _fields_ = [("force", C.c_float * 2), ("position", C.c_float * 2)]


class Source(C.Structure):
    _fields_ = [("center", C.c_float * 2), ("data", C.c_float * 2), ("velocity", C.c_float * 2),
                ("shape", C.c_uint32), ("mode", C.c_uint32)]


class SolidForce(C.Structure):
    _fields_ = [("force", C.c_float * 2), ("torque", C.c_float), ("_pad", C.c_float)]


class RigidBodyC(C.Structure):  # efl_rigid_body
    _fields_ = [("position", C.c_double * 2), ("rotation", C.c_double), ("linear_velocity", C.c_double * 2),
                ("angular_velocity", C.c_double), ("mass", C.c_double), ("inertia", C.c_double),
                ("extent", C.c_double), ("dynamic", C.c_int32), ("obstacle", C.c_int32)]


class Particle(C.Structure):  # efl_particle (particle.wgsl:5-11, storage stride 24)
    _fields_ = [("position", C.c_float * 2), ("radius", C.c_float), ("sign", C.c_float), ("escaped", C.c_uint32),
                ("_pad", C.c_uint32)]


# numpy view of an efl_particle array
PARTICLE_DTYPE = np.dtype([("position", "<f4", (2,)), ("radius", "<f4"), ("sign", "<f4"), ("escaped", "<u4"),
                           ("_pad", "<u4")])
PLS_POSITIVE, PLS_NEGATIVE = 0, 1
PLS_INITIALIZE, PLS_ADVECT, PLS_CORRECT, PLS_CORRECT_SECOND, PLS_RESEED = 0, 1, 2, 3, 4


class SlabDesc(C.Structure):
    _fields_ = [("device", C.c_int32), ("nx", C.c_uint32), ("ny", C.c_uint32), ("row0", C.c_uint32),
                ("rows", C.c_uint32), ("dx", C.c_float), ("dt", C.c_float), ("rho", C.c_float),
                ("sor_weight", C.c_float)]


SLAB_X, SLAB_D, SLAB_LEVELSET = 0, 1, 2


class StepStats(C.Structure):
    _fields_ = [("initialized_only", C.c_int32), ("pressure_iterations", C.c_uint32), ("converged", C.c_int32),
                ("_pad", C.c_int32), ("residual", C.c_double), ("residual_initial", C.c_double)]

    def as_dict(self) -> dict:
        return {"initialized_only": self.initialized_only, "pressure_iterations": self.pressure_iterations,
                "converged": self.converged, "residual": self.residual,
                "residual_initial": self.residual_initial}


assert C.sizeof(SolidObstacle) == 176
assert C.sizeof(Force) == 16
assert C.sizeof(Source) == 32
assert C.sizeof(SolidForce) == 16
assert C.sizeof(Particle) == 24 == PARTICLE_DTYPE.itemsize

# Exported symbols of include/efl.h: name -> (restype, argtypes); "X" stands for the handle.
SIGNATURES = {
    "abi_version": (C.c_int32, []),
    "default_config": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(Config)]),
    "create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "destroy": (C.c_int, ["X"]),
    "last_error": (C.c_char_p, ["X"]),
    "reset": (C.c_int, ["X"]),
    "set_projection": (C.c_int, ["X", C.POINTER(Projection)]),
    "set_reinit": (C.c_int, ["X", C.POINTER(Reinit)]),
    "set_transform": (C.c_int, ["X", C.POINTER(C.c_float)]),
    "set_obstacles": (C.c_int, ["X", C.POINTER(SolidObstacle), C.c_uint32]),
    "set_local_forces": (C.c_int, ["X", C.POINTER(Force), C.c_uint32]),
    "set_sources": (C.c_int, ["X", C.POINTER(Source), C.c_uint32, C.c_int32]),
    "step": (C.c_int, ["X", C.c_float, C.POINTER(StepStats)]),
    "run_stage": (C.c_int, ["X", C.c_int32, C.c_float, C.POINTER(StepStats)]),
    "read_solid_forces": (C.c_int, ["X", C.POINTER(SolidForce)]),
    "read_force_bins": (C.c_int, ["X", C.POINTER(C.c_int32)]),
    "field_shape": (C.c_int, ["X", C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                              C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "get_field": (C.c_int, ["X", C.c_int32, C.c_void_p, C.c_size_t]),
    "set_field": (C.c_int, ["X", C.c_int32, C.c_void_p, C.c_size_t]),
    "field_device_ptr": (C.c_int, ["X", C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "stream": (C.c_int, ["X", C.POINTER(C.c_void_p)]),
    "synchronize": (C.c_int, ["X"]),
    "residual": (C.c_int, ["X", C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fluid_volume": (C.c_int, ["X", C.POINTER(C.c_uint64)]),
    "divergence_norms": (C.c_int, ["X", C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "velocity_magnitude": (C.c_int, ["X", C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "set_particle_levelset": (C.c_int, ["X", C.c_int32]),
    "particle_counts": (C.c_int, ["X", C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "read_particles": (C.c_int, ["X", C.c_int32, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "write_particles": (C.c_int, ["X", C.c_int32, C.c_void_p, C.c_uint32]),
    "pls_run_phase": (C.c_int, ["X", C.c_int32, C.c_float]),
    "kernel_launches": (C.c_uint64, []),
    "pressure_sweeps": (C.c_int, ["X", C.c_int32, C.c_uint32]),
    "residual_norms_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                         C.c_uint32, C.c_size_t, C.c_float, C.c_float, C.c_float, C.c_void_p,
                                         C.c_void_p]),
    "batch_create": (C.c_int, [C.POINTER(Config), C.c_uint32, C.POINTER(C.c_void_p)]),
    "batch_destroy": (C.c_int, [C.c_void_p]),
    "batch_last_error": (C.c_char_p, [C.c_void_p]),
    "batch_sim": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "batch_step": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(StepStats)]),
    "batch_projection_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "batch_set_tiles": (C.c_int, [C.c_void_p, C.c_int32]),
    "batch_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                              C.POINTER(C.c_double)]),
    "projection_ms": (C.c_int, ["X", C.POINTER(C.c_float)]),
    "set_wait_limits": (C.c_int, ["X", C.c_uint64, C.c_uint64]),
    "batch_set_wait_limits": (C.c_int, [C.c_void_p, C.c_uint64]),
    "set_graph_capture": (C.c_int, ["X", C.c_int32]),
    "set_rigid_bodies": (C.c_int, ["X", C.POINTER(RigidBodyC), C.c_uint32, C.c_double, C.c_double, C.c_uint32]),
    "get_rigid_bodies": (C.c_int, ["X", C.POINTER(RigidBodyC), C.c_uint32]),
    "unet_create": (C.c_int, [C.c_int32, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "unet_destroy": (C.c_int, [C.c_void_p]),
    "unet_last_error": (C.c_char_p, [C.c_void_p]),
    "unet_num_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "unet_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "unet_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "unet_forward": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    "unet_gradients": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_float), C.c_void_p]),
    "unet_attach": (C.c_int, ["X", C.c_void_p, C.c_uint32]),
    "unet_train_step": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_float)]),
    "unet_time_forward": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
    "unet_set_coarsening": (C.c_int, [C.c_void_p, C.c_uint32]),
    "batch_attach_unet": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "batch_unet_canvas": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "canvas_pack": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "slab_create": (C.c_int, [C.POINTER(SlabDesc), C.POINTER(C.c_void_p)]),
    "slab_destroy": (C.c_int, [C.c_void_p]),
    "slab_load": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "slab_halo": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "slab_prepare": (C.c_int, [C.c_void_p]),
    "slab_residual": (C.c_int, [C.c_void_p, C.c_void_p]),
    "slab_sweep": (C.c_int, [C.c_void_p, C.c_int32]),
    "slab_apply": (C.c_int, [C.c_void_p]),
    "slab_read": (C.c_int, [C.c_void_p, C.c_void_p]),
}
# Functions of efl.h that the oracle restatement does not mirror.
PRODUCT_ONLY = {"abi_version", "default_config", "field_device_ptr", "stream", "synchronize", "kernel_launches",
                "pressure_sweeps", "residual_norms_noalloc", "batch_create", "batch_destroy", "batch_last_error",
                "batch_sim", "batch_step", "batch_projection_ms", "batch_set_tiles", "batch_tiles", "batch_set_wait_limits",
                "projection_ms", "set_graph_capture", "set_wait_limits", "set_rigid_bodies", "get_rigid_bodies",
                "unet_create", "unet_destroy", "unet_last_error", "unet_num_params", "unet_get_params",
                "unet_set_params", "unet_forward", "unet_gradients", "unet_attach", "unet_train_step",
                "unet_time_forward", "unet_set_coarsening", "batch_attach_unet", "batch_unet_canvas", "canvas_pack",
                "slab_create", "slab_destroy",
                "slab_load", "slab_halo", "slab_prepare", "slab_residual", "slab_sweep", "slab_apply", "slab_read"}


class EflError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Api:
    """A bound function table for one library and symbol prefix ("efl_" or "eflo_")."""

    def __init__(self, lib: C.CDLL, prefix: str):
        self.lib = lib
        self.prefix = prefix
        self.fns = {}
        for name, (res, args) in SIGNATURES.items():
            sym = prefix + name
            if not hasattr(lib, sym):
                if prefix != "efl_" and name in PRODUCT_ONLY:
                    continue
                raise OSError(f"{sym} missing from {lib._name}")
            fn = getattr(lib, sym)
            fn.restype = res
            fn.argtypes = [C.c_void_p if a == "X" else a for a in args]
            self.fns[name] = fn

    def __getattr__(self, name):
        try:
            return self.fns[name]
        except KeyError as e:
            raise AttributeError(name) from e


_API: Optional[Api] = None


def load(path: str = LIB_PATH) -> Api:
    """Opens libefl_b200.so. Raises if it is missing: no fallback exists."""
    global _API
    if _API is not None and path == LIB_PATH:
        return _API
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m bevy_eulerian_fluid_b200.build` "
            "(the CUDA extension is required; there is no CPU fallback)")
    api = Api(C.CDLL(path), "efl_")
    if path == LIB_PATH:
        _API = api
    return api


def canvas_pack(api: Api, sizes):
    """The canvas layout of a batch's network forward (efl_canvas_pack; host only): sizes = [(w, h), ...] in
    pixels, multiples of 8 -> ([(x, y) origin per image], width, height)."""
    n = len(sizes)
    wh = (C.c_int32 * max(1, 2 * n))(*[v for s in sizes for v in s])
    org = (C.c_int32 * max(1, 2 * n))()
    w, h = C.c_int32(), C.c_int32()
    st = api.canvas_pack(wh, n, org, C.byref(w), C.byref(h))
    if st != OK:
        raise EflError(st, "canvas_pack: sizes must be positive multiples of 8")
    return [(org[2 * i], org[2 * i + 1]) for i in range(n)], w.value, h.value


def default_config(nx: int, ny: int) -> Config:
    """Reference defaults (matches efl_default_config), without loading the library."""
    c = Config()
    c.nx, c.ny = nx, ny
    c.length_unit, c.rho = 1.0, 1.0
    c.gravity[0], c.gravity[1] = 0.0, 9.8
    for i in range(4):
        c.transform[i * 5] = 1.0
    p = c.projection
    p.method, p.gs_iterations, p.sor_weight = PROJECTION_GAUSS_SEIDEL, 20, 1.9
    p.mg_pre, p.mg_post, p.mg_coarsest, p.mg_levels = 2, 2, 3, 0
    p.tolerance, p.max_iterations, p.check_interval = 0.0, 20000, 16
    c.reinit.method, c.reinit.fim_iterations = REINIT_FAST_ITERATIVE, 10
    c.device = 0
    return c


class Sim:
    """One simulation handle on a bound Api (the CUDA library or the oracle)."""

    def __init__(self, api: Api, cfg: Config):
        self.api = api
        self.cfg = cfg
        h = C.c_void_p()
        st = api.create(C.byref(cfg), C.byref(h))
        if st != OK:
            raise EflError(st, (api.last_error(None) or b"").decode())
        self.h = h
        self.nx, self.ny = cfg.nx, cfg.ny

    @classmethod
    def borrowed(cls, api: Api, h: C.c_void_p, cfg: Config) -> "Sim":
        """A view of a simulation owned by a Batch (close() does not destroy it)."""
        self = cls.__new__(cls)
        self.api, self.cfg, self.h = api, cfg, h
        self.nx, self.ny = cfg.nx, cfg.ny
        self._borrowed = True
        return self

    # -- lifetime
    def close(self):
        if getattr(self, "h", None):
            if not getattr(self, "_borrowed", False):
                self.api.destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, allow=(OK,)) -> int:
        if st not in allow:
            raise EflError(st, (self.api.last_error(self.h) or b"").decode())
        return st

    # -- inputs
    def reset(self):
        self._check(self.api.reset(self.h))

    def set_projection(self, p: Projection):
        self._check(self.api.set_projection(self.h, C.byref(p)))
        self.cfg.projection = p

    def set_reinit(self, r: Reinit):
        self._check(self.api.set_reinit(self.h, C.byref(r)))
        self.cfg.reinit = r

    def set_transform(self, m16):
        arr = (C.c_float * 16)(*[float(v) for v in m16])
        self._check(self.api.set_transform(self.h, arr))

    def set_obstacles(self, obstacles):
        """A sequence of SolidObstacle, or a ctypes array of them (passed on without a copy)."""
        if isinstance(obstacles, C.Array) and len(obstacles) > 0:
            arr = obstacles
        else:
            arr = (SolidObstacle * max(1, len(obstacles)))(*obstacles)
        self._check(self.api.set_obstacles(self.h, arr, len(obstacles)))

    def set_local_forces(self, forces):
        arr = (Force * max(1, len(forces)))(*forces)
        self._check(self.api.set_local_forces(self.h, arr, len(forces)))

    def set_sources(self, sources, oneshot: bool):
        arr = (Source * max(1, len(sources)))(*sources)
        self._check(self.api.set_sources(self.h, arr, len(sources), 1 if oneshot else 0))

    # -- stepping
    def step(self, dt: float, allow_not_converged: bool = True) -> StepStats:
        st = StepStats()
        allow = (OK, NOT_CONVERGED) if allow_not_converged else (OK,)
        self._check(self.api.step(self.h, dt, C.byref(st)), allow)
        return st

    def run_stage(self, stage: int, dt: float = 0.0) -> StepStats:
        st = StepStats()
        self._check(self.api.run_stage(self.h, stage, dt, C.byref(st)), (OK, NOT_CONVERGED))
        return st

    # -- outputs
    def field_shape(self, field: int):
        w, h, ch, eb = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._check(self.api.field_shape(self.h, field, C.byref(w), C.byref(h), C.byref(ch), C.byref(eb)))
        return w.value, h.value, ch.value

    def get(self, field: int) -> np.ndarray:
        w, h, ch = self.field_shape(field)
        dt = FIELD_DTYPES.get(field, np.float32)
        shape = (h, w) if ch == 1 else (h, w, ch)
        out = np.empty(shape, dtype=dt)
        self._check(self.api.get_field(self.h, field, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def set(self, field: int, arr: np.ndarray):
        w, h, ch = self.field_shape(field)
        dt = FIELD_DTYPES.get(field, np.float32)
        a = np.ascontiguousarray(arr, dtype=dt)
        want = (h, w) if ch == 1 else (h, w, ch)
        if a.shape != want:
            raise ValueError(f"field {field}: expected shape {want}, got {a.shape}")
        self._check(self.api.set_field(self.h, field, a.ctypes.data_as(C.c_void_p), a.nbytes))

    def solid_forces(self) -> np.ndarray:
        arr = (SolidForce * MAX_SOLIDS)()
        self._check(self.api.read_solid_forces(self.h, arr))
        return np.frombuffer(arr, dtype=np.float32).reshape(MAX_SOLIDS, 4)[:, :3].copy()

    def force_bins(self) -> np.ndarray:
        arr = (C.c_int32 * (3 * MAX_SOLIDS))()
        self._check(self.api.read_force_bins(self.h, arr))
        return np.frombuffer(arr, dtype=np.int32).reshape(3, MAX_SOLIDS).copy()

    def residual(self):
        rel, nr, nb = C.c_double(), C.c_double(), C.c_double()
        self._check(self.api.residual(self.h, C.byref(rel), C.byref(nr), C.byref(nb)))
        return rel.value, nr.value, nb.value

    def fluid_volume(self) -> int:
        c = C.c_uint64()
        self._check(self.api.fluid_volume(self.h, C.byref(c)))
        return c.value

    def divergence_norms(self):
        """(L2, Linf) of the divergence of the current velocity over the counted cells (1/s)."""
        a, b = C.c_double(), C.c_double()
        self._check(self.api.divergence_norms(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def velocity_magnitude(self):
        """(min over fluid cells, max) of the cell-centred speed, as the reference's diagnostics compute them."""
        a, b = C.c_float(), C.c_float()
        self._check(self.api.velocity_magnitude(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- two-layer particle level set
    def set_particle_levelset(self, enable: bool = True):
        """ParticleLevelsetTwoLayersPlugin on this simulation (seeded by the next init sequence)."""
        self._check(self.api.set_particle_levelset(self.h, 1 if enable else 0))

    def particle_counts(self):
        """((positive, negative) live counts, particles dropped for lack of capacity)."""
        c = (C.c_uint32 * 2)()
        d = C.c_uint32()
        self._check(self.api.particle_counts(self.h, c, C.byref(d)))
        return (c[0], c[1]), d.value

    def read_particles(self, layer: int) -> np.ndarray:
        """A layer's particles as a PARTICLE_DTYPE array."""
        (n0, n1), _ = self.particle_counts()
        n = (n0, n1)[layer]
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        got = C.c_uint32()
        self._check(self.api.read_particles(self.h, layer, out.ctypes.data if n else None, n, C.byref(got)))
        return out[:min(n, got.value)]

    def write_particles(self, layer: int, parts: np.ndarray):
        arr = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
        self._check(self.api.write_particles(self.h, layer, arr.ctypes.data if len(arr) else None, len(arr)))

    def pls_run_phase(self, phase: int, dt: float = 0.0):
        self._check(self.api.pls_run_phase(self.h, phase, dt))

    def synchronize(self):
        self._check(self.api.synchronize(self.h))

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.api.stream(self.h, C.byref(p)))
        return p.value or 0

    def device_ptr(self, field: int):
        """(device pointer, row pitch in bytes) of a field plane."""
        p, pitch = C.c_void_p(), C.c_size_t()
        self._check(self.api.field_device_ptr(self.h, field, C.byref(p), C.byref(pitch)))
        return p.value, pitch.value

    def set_rigid_bodies(self, bodies, gravity: float, grid_length: float, substeps: int = 1):
        """Device-side coupling: bodies (RigidBodyC) integrated at the end of every step."""
        arr = (RigidBodyC * max(1, len(bodies)))(*bodies)
        self._check(self.api.set_rigid_bodies(self.h, arr, len(bodies), gravity, grid_length, substeps))

    def get_rigid_bodies(self, n: int):
        arr = (RigidBodyC * max(1, n))()
        self._check(self.api.get_rigid_bodies(self.h, arr, n))
        return list(arr)[:n]

    def set_graph_capture(self, enable: bool):
        """Replay repeating step segments as CUDA graphs (default on)."""
        self._check(self.api.set_graph_capture(self.h, 1 if enable else 0))

    def projection_ms(self) -> float:
        """Device time of the last projection stage (ms)."""
        ms = C.c_float()
        self._check(self.api.projection_ms(self.h, C.byref(ms)))
        return ms.value

    def pressure_sweeps(self, precision: int, iterations: int):
        self._check(self.api.pressure_sweeps(self.h, precision, iterations))

    def set_wait_limits(self, barrier_polls: int = 0, mbarrier_polls: int = 0):
        """Polls of the device-side waits before they give up (0 = the defaults)."""
        self._check(self.api.set_wait_limits(self.h, barrier_polls, mbarrier_polls))


class Batch:
    """N independent simulations stepped together (efl_batch_*): one shared
    stream and one cooperative launch for all tolerance-driven solves."""

    def __init__(self, api: Api, cfgs):
        self.api = api
        self.cfgs = list(cfgs)
        arr = (Config * len(self.cfgs))(*self.cfgs)
        h = C.c_void_p()
        st = api.batch_create(arr, len(self.cfgs), C.byref(h))
        if st != OK:
            raise EflError(st, (api.batch_last_error(None) or b"").decode())
        self.h = h
        self.sims = []
        for i, c in enumerate(self.cfgs):
            sh = C.c_void_p()
            self._check(api.batch_sim(self.h, i, C.byref(sh)))
            self.sims.append(Sim.borrowed(api, sh, c))

    def __len__(self):
        return len(self.sims)

    def __getitem__(self, i) -> Sim:
        return self.sims[i]

    def _check(self, st: int, allow=(OK,)) -> int:
        if st not in allow:
            raise EflError(st, (self.api.batch_last_error(self.h) or b"").decode())
        return st

    def step(self, dt: float, allow_not_converged: bool = True):
        """One frame of every simulation; returns the per-simulation StepStats."""
        stats = (StepStats * len(self.sims))()
        allow = (OK, NOT_CONVERGED) if allow_not_converged else (OK,)
        self._check(self.api.batch_step(self.h, dt, stats), allow)
        return list(stats)

    def set_tiles(self, config: int):
        """-1 = autotune (default), 0 / 1 / 2 / 3 = 64x32x2, 64x32x4, 32x32x2, 64x32x8."""
        self._check(self.api.batch_set_tiles(self.h, config))

    def tiles(self):
        """((tx, ty, k) in use or (0, 0, 0) while tuning, [ns per cell-iteration of each configuration])."""
        tx, ty, k = C.c_int32(), C.c_int32(), C.c_int32()
        cost = (C.c_double * 4)()
        self._check(self.api.batch_tiles(self.h, C.byref(tx), C.byref(ty), C.byref(k), cost))
        return (tx.value, ty.value, k.value), list(cost)

    def attach_unet(self, net: "UNet", warm_start: bool = True):
        """Warm-starts every simulation's solve with the network: one forward over a canvas of all the
        simulations' coarse grids where the coarsening allows, else one forward workspace per simulation."""
        self._check(self.api.batch_attach_unet(self.h, net.h if warm_start else None,
                                               UNET_WARM_START if warm_start else 0))

    def unet_canvas(self):
        """(width, height) of the canvas of the network's batched forward, (0, 0) without one."""
        w, h = C.c_int32(), C.c_int32()
        self._check(self.api.batch_unet_canvas(self.h, C.byref(w), C.byref(h)))
        return w.value, h.value

    def set_wait_limits(self, barrier_polls: int = 0):
        """Grid-barrier polls of the batched solve before it gives up (0 = the default)."""
        self._check(self.api.batch_set_wait_limits(self.h, barrier_polls))

    def projection_ms(self) -> float:
        """Device time of the last batched pressure solve (ms)."""
        ms = C.c_float()
        self._check(self.api.batch_projection_ms(self.h, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            for s in self.sims:
                s.h = None
            self.api.batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


UNET_WARM_START, UNET_RECORD = 1, 2


class UNet:
    """The learned warm start's network (efl_unet_*)."""

    def __init__(self, api: Api, max_nx: int, max_ny: int, seed: int = 0, device: int = 0):
        self.api = api
        h = C.c_void_p()
        st = api.unet_create(device, max_nx, max_ny, seed, C.byref(h))
        if st != OK:
            raise EflError(st, (api.unet_last_error(None) or b"").decode())
        self.h = h
        n = C.c_uint64()
        self._check(api.unet_num_params(self.h, C.byref(n)))
        self.n_params = n.value

    def _check(self, st: int):
        if st != OK:
            raise EflError(st, (self.api.unet_last_error(self.h) or b"").decode())

    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._check(self.api.unet_get_params(self.h, out.ctypes.data_as(C.c_void_p), self.n_params))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        self._check(self.api.unet_set_params(self.h, p.ctypes.data_as(C.c_void_p), self.n_params))

    def forward(self, feats: np.ndarray) -> np.ndarray:
        ny, nx = feats.shape[:2]
        f = np.ascontiguousarray(feats, np.float32)
        out = np.empty((ny, nx), np.float32)
        self._check(self.api.unet_forward(self.h, nx, ny, f.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
        return out

    def gradients(self, feats, target, mask):
        ny, nx = feats.shape[:2]
        f = np.ascontiguousarray(feats, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        m = np.ascontiguousarray(mask, np.uint8)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float()
        self._check(self.api.unet_gradients(self.h, nx, ny, f.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p),
                                            m.ctypes.data_as(C.c_void_p), C.byref(loss), g.ctypes.data_as(C.c_void_p)))
        return loss.value, g

    def attach(self, sim: "Sim", warm_start: bool = True, record: bool = False):
        flags = (UNET_WARM_START if warm_start else 0) | (UNET_RECORD if record else 0)
        self._check(self.api.unet_attach(sim.h, self.h if flags else None, flags))

    def set_coarsening(self, factor: int):
        """Run the network on the grid coarsened by factor (1, 2, 4 or 8); see efl_unet_set_coarsening."""
        self._check(self.api.unet_set_coarsening(self.h, factor))

    def time_forward(self, nx: int, ny: int, reps: int = 20) -> float:
        """Device ms of one forward pass at nx x ny, replayed from a CUDA graph
        of the pass (as a simulation step runs it)."""
        ms = C.c_float()
        self._check(self.api.unet_time_forward(self.h, nx, ny, reps, C.byref(ms)))
        return ms.value

    def train_step(self, lr: float = 1e-3) -> float:
        loss = C.c_float()
        self._check(self.api.unet_train_step(self.h, lr, C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self.api.unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
