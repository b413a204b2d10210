"""Python mirror of the reference's solver interface over the C ABI.

The reference proxy apps expose ``System`` (input.in parsing,
tgv/src/System.hpp) and the ``LBM`` struct (tgv/src/lbm.hpp:238-251) whose
member functions each case's ``main()`` calls in sequence.  This module keeps
those names and argument meanings on top of ``libimexlb.so``
(include/imexlb.h): ``System(path, case)``, ``LBM(case, nx, ny, nz, tau, rho0,
u0)``, ``LBM.Initialize()``, ``LBM.step(n)`` (Collision, pack, exchange,
unpack, Streaming and Update fused per step), ``LBM.MPIoutput(n)``, plus the
fields the reference keeps in its views (``ua``, ``va``, ``wa``, ``p``,
``usr``).

There is no CPU fallback: importing this module fails if the native library
has not been built (``python -m imexlb_b200.build``), and creating a lattice
fails without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimexlb.so")

CASES = {"tgv": 0, "cavity": 1, "sphere": 2}
BCS = {"reference": 0, "standard": 1, "slab": 2, "reference-links": 3}
STORAGES = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}
ARITHS = {"exact": 0, "fast": 1}
REDUCE = {"mass": 0, "kinetic": 1, "residual": 2, "drag": 3, "umax": 4}
BYTES_PER_VALUE = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}


class ImexlbError(RuntimeError):
    """A nonzero return code of the C ABI, with imexlb_last_error()."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"imexlb error {code}: {msg}")
        self.code = code


class SystemStruct(ctypes.Structure):
    _fields_ = [("rho0", ctypes.c_double), ("R", ctypes.c_double), ("Re", ctypes.c_int),
                ("u0", ctypes.c_double), ("Time", ctypes.c_int), ("inter", ctypes.c_int),
                ("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int),
                ("miu", ctypes.c_double), ("tau", ctypes.c_double), ("Ma", ctypes.c_double),
                ("cs2", ctypes.c_double), ("cs", ctypes.c_double)]


class KernelTimes(ctypes.Structure):
    _fields_ = [("step_ms", ctypes.c_double), ("ghost_ms", ctypes.c_double),
                ("step_launches", ctypes.c_int64), ("ghost_launches", ctypes.c_int64)]


class ParamsStruct(ctypes.Structure):
    _fields_ = [("kase", ctypes.c_int), ("bc", ctypes.c_int), ("storage", ctypes.c_int), ("arith", ctypes.c_int),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("tau0", ctypes.c_double), ("rho0", ctypes.c_double), ("u0", ctypes.c_double),
                ("ran", ctypes.c_void_p), ("seed", ctypes.c_uint64),
                ("lid_u", ctypes.c_double), ("inlet_u", ctypes.c_double), ("sphere_d", ctypes.c_double),
                ("sphere_c", ctypes.c_double * 3), ("stream", ctypes.c_void_p)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("kase", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("tau0", ctypes.c_double), ("rho0", ctypes.c_double), ("u0", ctypes.c_double),
                ("lid_u", ctypes.c_double), ("inlet_u", ctypes.c_double), ("sphere_d", ctypes.c_double),
                ("sphere_c", ctypes.c_double * 3), ("tile_bx", ctypes.c_int)]


class EngineStats(ctypes.Structure):
    _fields_ = [("instances", ctypes.c_int), ("cells", ctypes.c_int64), ("budget_bytes", ctypes.c_size_t),
                ("used_bytes", ctypes.c_size_t), ("tiles", ctypes.c_int64), ("steps", ctypes.c_int64)]


# Every symbol include/imexlb.h declares (tests check the library exports them).
EXPORTS = ["imexlb_params_default", "imexlb_system_read", "imexlb_create", "imexlb_initialize", "imexlb_step",
           "imexlb_get_fields", "imexlb_get_fields_async", "imexlb_get_mask", "imexlb_write_tecplot", "imexlb_reduce",
           "imexlb_reduce_async", "imexlb_reduce_fields_noalloc", "imexlb_release_cached_memory", "imexlb_steps_taken",
           "imexlb_footprint", "imexlb_checkpoint_size", "imexlb_checkpoint_save", "imexlb_checkpoint_load",
           "imexlb_ghost_plan", "imexlb_profile", "imexlb_profile_read", "imexlb_synchronize", "imexlb_set_wait_limit",
           "imexlb_set_rounding", "imexlb_destroy", "imexlb_last_error",
           "imexlb_version", "imexlb_engine_create", "imexlb_engine_add", "imexlb_engine_add_as", "imexlb_engine_remove",
           "imexlb_engine_step", "imexlb_engine_limit", "imexlb_engine_fields", "imexlb_engine_plane",
           "imexlb_engine_residuals", "imexlb_engine_info",
           "imexlb_engine_instance_bytes", "imexlb_engine_checkpoint_size", "imexlb_engine_checkpoint_save",
           "imexlb_engine_restore", "imexlb_engine_synchronize", "imexlb_engine_destroy"]

_LIB = None


def load_library() -> ctypes.CDLL:
    """Load libimexlb.so (raises ImportError if it was never built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m imexlb_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.imexlb_params_default.argtypes = [ctypes.POINTER(ParamsStruct)]
    lib.imexlb_params_default.restype = None
    lib.imexlb_system_read.argtypes = [ctypes.c_char_p, i, ctypes.POINTER(SystemStruct)]
    lib.imexlb_create.argtypes = [ctypes.POINTER(ParamsStruct), ctypes.POINTER(vp)]
    lib.imexlb_initialize.argtypes = [vp]
    lib.imexlb_step.argtypes = [vp, i]
    lib.imexlb_get_fields.argtypes = [vp, vp, vp, vp, vp]
    lib.imexlb_get_fields_async.argtypes = [vp, vp, vp, vp, vp]
    lib.imexlb_get_mask.argtypes = [vp, vp]
    lib.imexlb_write_tecplot.argtypes = [vp, ctypes.c_char_p, i]
    lib.imexlb_reduce.argtypes = [vp, i, ctypes.POINTER(d)]
    lib.imexlb_reduce_async.argtypes = [vp, i, vp]
    lib.imexlb_release_cached_memory.argtypes = []
    lib.imexlb_reduce_fields_noalloc.argtypes = [i, vp, vp, vp, vp, ctypes.c_int64, vp, vp]
    lib.imexlb_steps_taken.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    lib.imexlb_footprint.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(d)]
    lib.imexlb_ghost_plan.argtypes = [i, i, i, i, vp, vp, vp, ctypes.POINTER(ctypes.c_int64)]
    lib.imexlb_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    lib.imexlb_checkpoint_save.argtypes = [vp, vp, ctypes.c_size_t]
    lib.imexlb_checkpoint_load.argtypes = [vp, vp, ctypes.c_size_t]
    lib.imexlb_engine_checkpoint_size.argtypes = [vp, i, ctypes.POINTER(ctypes.c_size_t)]
    lib.imexlb_engine_checkpoint_save.argtypes = [vp, i, vp, ctypes.c_size_t]
    lib.imexlb_engine_restore.argtypes = [vp, ctypes.POINTER(InstanceDesc), vp, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_int)]
    lib.imexlb_profile.argtypes = [vp, i]
    lib.imexlb_profile_read.argtypes = [vp, ctypes.POINTER(KernelTimes)]
    lib.imexlb_synchronize.argtypes = [vp]
    lib.imexlb_set_wait_limit.argtypes = [vp, ctypes.c_double]
    lib.imexlb_destroy.argtypes = [vp]
    lib.imexlb_destroy.restype = None
    lib.imexlb_last_error.restype = ctypes.c_char_p
    lib.imexlb_version.restype = ctypes.c_char_p
    lib.imexlb_engine_create.argtypes = [i, i, ctypes.c_size_t, i, vp, ctypes.POINTER(vp)]
    lib.imexlb_engine_add.argtypes = [vp, ctypes.POINTER(InstanceDesc), ctypes.POINTER(ctypes.c_int)]
    lib.imexlb_engine_add_as.argtypes = [vp, ctypes.POINTER(InstanceDesc), i, ctypes.POINTER(ctypes.c_int)]
    lib.imexlb_engine_remove.argtypes = [vp, i]
    lib.imexlb_engine_step.argtypes = [vp, i]
    lib.imexlb_engine_limit.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.imexlb_engine_fields.argtypes = [vp, i, vp, vp, vp, vp]
    lib.imexlb_engine_plane.argtypes = [vp, i, i, vp, vp, vp, vp]
    lib.imexlb_engine_residuals.argtypes = [vp, vp, i]
    lib.imexlb_engine_info.argtypes = [vp, ctypes.POINTER(EngineStats)]
    lib.imexlb_engine_instance_bytes.argtypes = [i, ctypes.POINTER(InstanceDesc), ctypes.POINTER(ctypes.c_size_t)]
    lib.imexlb_engine_synchronize.argtypes = [vp]
    lib.imexlb_engine_destroy.argtypes = [vp]
    lib.imexlb_engine_destroy.restype = None
    _LIB = lib
    return lib


def _check(rc: int):
    if rc:
        raise ImexlbError(rc, load_library().imexlb_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def System(path: str, case: str) -> dict:
    """System::System: parse an input.in for `case` (with its overrides)."""
    s = SystemStruct()
    _check(load_library().imexlb_system_read(path.encode(), CASES[case], ctypes.byref(s)))
    return {k: getattr(s, k) for k, _ in SystemStruct._fields_}


def ghost_plan(case: str, nx: int, ny: int, nz: int, usr_padded: np.ndarray | None = None):
    """The reference boundary passes resolved into one copy per slot."""
    lib = load_library()
    usr = None if usr_padded is None else np.ascontiguousarray(usr_padded, dtype=np.int32)
    n = ctypes.c_int64(0)
    _check(lib.imexlb_ghost_plan(CASES[case], nx, ny, nz, _ptr(usr), None, None, ctypes.byref(n)))
    tgt = np.empty(n.value, dtype=np.int64)
    src = np.empty(n.value, dtype=np.int64)
    _check(lib.imexlb_ghost_plan(CASES[case], nx, ny, nz, _ptr(usr), _ptr(tgt), _ptr(src), ctypes.byref(n)))
    return tgt, src


class LBM:
    """One lattice on the current CUDA device (the reference's LBM struct)."""

    def __init__(self, case: str, nx: int, ny: int, nz: int, tau: float, rho0: float = 1.0, u0: float = 0.05, *,
                 bc: str = "reference", storage: str = "f64", arith: str = "exact", ran: np.ndarray | None = None,
                 seed: int = 5374857, lid_u: float = 0.0, inlet_u: float = 0.0, sphere_d: float = 0.0,
                 sphere_c=(0.0, 0.0, 0.0), stream: int | None = None):
        self.lib = load_library()
        self.case, self.bc, self.storage = case, bc, storage
        self.n = (nx, ny, nz)
        p = ParamsStruct()
        self.lib.imexlb_params_default(ctypes.byref(p))
        p.kase, p.bc, p.storage, p.arith = CASES[case], BCS[bc], STORAGES[storage], ARITHS[arith]
        p.nx, p.ny, p.nz = nx, ny, nz
        p.tau0, p.rho0, p.u0 = tau, rho0, u0
        self._ran = None
        if ran is not None:
            self._ran = np.ascontiguousarray(ran, dtype=np.int32)
            p.ran = self._ran.ctypes.data
        p.seed = seed
        p.lid_u, p.inlet_u, p.sphere_d = lid_u, inlet_u, sphere_d
        p.sphere_c[0], p.sphere_c[1], p.sphere_c[2] = sphere_c
        p.stream = stream
        h = ctypes.c_void_p()
        _check(self.lib.imexlb_create(ctypes.byref(p), ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_system(cls, case: str, system: dict, **kw) -> "LBM":
        """LBM l1(comm, s1.sx, s1.sy, s1.sz, s1.tau, s1.rho0, s1.u0)."""
        return cls(case, system["sx"], system["sy"], system["sz"], system["tau"], system["rho0"], system["u0"], **kw)

    def close(self):
        if getattr(self, "h", None):
            self.lib.imexlb_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def Initialize(self):
        _check(self.lib.imexlb_initialize(self.h))

    def step(self, n: int = 1):
        """n fused time steps (asynchronous on the lattice's stream)."""
        _check(self.lib.imexlb_step(self.h, n))

    def synchronize(self):
        _check(self.lib.imexlb_synchronize(self.h))

    def set_wait_limit(self, seconds: float):
        """Bound on the 2-byte staged kernels' waits for their row copies
        (imexlb_set_wait_limit)."""
        _check(self.lib.imexlb_set_wait_limit(self.h, seconds))

    def set_rounding(self, mode: str):
        """Rounding of the 2-byte stores: "stochastic" or "nearest"
        (imexlb_set_rounding)."""
        _check(self.lib.imexlb_set_rounding(self.h, {"nearest": 0, "stochastic": 1}[mode]))

    def fields(self, out: dict | None = None, wait: bool = True) -> dict:
        """ua, va, wa, p after the last step, each shaped (nz, ny, nx).  With
        wait=False the copy is only enqueued (imexlb_get_fields_async): `out`
        (pinned memory overlaps the copy with later steps) holds the fields
        after the next synchronize() or synchronous call."""
        nx, ny, nz = self.n
        if out is None:
            out = {k: np.empty((nz, ny, nx)) for k in ("u", "v", "w", "p")}
        fn = self.lib.imexlb_get_fields if wait else self.lib.imexlb_get_fields_async
        _check(fn(self.h, _ptr(out["u"]), _ptr(out["v"]), _ptr(out["w"]), _ptr(out["p"])))
        return out

    def mask(self) -> np.ndarray:
        nx, ny, nz = self.n
        m = np.empty((nz, ny, nx), dtype=np.int32)
        _check(self.lib.imexlb_get_mask(self.h, _ptr(m)))
        return m

    def MPIoutput(self, n: int, directory: str = ".") -> str:
        """Write output<n>.plt as the reference's MPIoutput does at one rank."""
        path = os.path.join(directory, f"output{n}.plt")
        _check(self.lib.imexlb_write_tecplot(self.h, path.encode(), n))
        return path

    def reduce(self, kind: str) -> float:
        out = (ctypes.c_double * 3)()
        _check(self.lib.imexlb_reduce(self.h, REDUCE[kind], out))
        return out[0] if kind != "drag" else (out[0], out[1], out[2])

    def reduce_async(self, kind: str, out: np.ndarray, index: int = 0):
        """Queue a one-value reduction whose value lands in out[index] (an FP64
        array, pinned for the copy to overlap) by the next synchronize()."""
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and 0 <= index < out.size
        _check(self.lib.imexlb_reduce_async(self.h, REDUCE[kind], out.ctypes.data + 8 * index))

    def checkpoint(self) -> bytes:
        """The lattice's state (both buffers, moments, step count) as bytes."""
        n = ctypes.c_size_t()
        _check(self.lib.imexlb_checkpoint_size(self.h, ctypes.byref(n)))
        buf = (ctypes.c_char * n.value)()
        _check(self.lib.imexlb_checkpoint_save(self.h, buf, n.value))
        return bytes(buf)

    def restore(self, data: bytes):
        """Continue from a checkpoint of a lattice with the same parameters."""
        _check(self.lib.imexlb_checkpoint_load(self.h, data, len(data)))

    def steps_taken(self) -> int:
        s = ctypes.c_int64()
        _check(self.lib.imexlb_steps_taken(self.h, ctypes.byref(s)))
        return s.value

    def profile(self, enable: bool = True):
        """Start per-launch CUDA-event timing of this lattice's kernels."""
        _check(self.lib.imexlb_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        """Summed device time per kernel kind since profile(); stops timing."""
        t = KernelTimes()
        _check(self.lib.imexlb_profile_read(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in KernelTimes._fields_}

    def footprint(self):
        b = ctypes.c_size_t()
        per = ctypes.c_double()
        _check(self.lib.imexlb_footprint(self.h, ctypes.byref(b), ctypes.byref(per)))
        return b.value, per.value


def release_cached_memory():
    """Return the lattice pool's reserved device memory of the current device."""
    _check(load_library().imexlb_release_cached_memory())


def instance_desc(case: str, nx: int, ny: int, nz: int, tau: float, rho0: float = 1.0, u0: float = 0.05, *,
                  lid_u: float = 0.0, inlet_u: float = 0.0, sphere_d: float = 0.0, sphere_c=(0.0, 0.0, 0.0),
                  tile_bx: int = 0) -> InstanceDesc:
    d = InstanceDesc()
    d.kase, d.nx, d.ny, d.nz = CASES[case], nx, ny, nz
    d.tau0, d.rho0, d.u0 = tau, rho0, u0
    d.lid_u, d.inlet_u, d.sphere_d = lid_u, inlet_u, sphere_d
    d.sphere_c[0], d.sphere_c[1], d.sphere_c[2] = sphere_c
    d.tile_bx = tile_bx
    return d


def instance_bytes(storage: str, desc: InstanceDesc) -> int:
    b = ctypes.c_size_t()
    _check(load_library().imexlb_engine_instance_bytes(STORAGES[storage], ctypes.byref(desc), ctypes.byref(b)))
    return b.value


class Engine:
    """Many independent lattices on one GPU, advanced together (C ABI engine)."""

    def __init__(self, storage: str = "f64", arith: str = "fast", budget_bytes: int = 1 << 30,
                 max_instances: int = 1024, stream: int | None = None):
        self.lib = load_library()
        self.storage = storage
        self.max_instances = max_instances
        h = ctypes.c_void_p()
        _check(self.lib.imexlb_engine_create(STORAGES[storage], ARITHS[arith], budget_bytes, max_instances, stream,
                                             ctypes.byref(h)))
        self.h = h
        self.shapes: dict[int, tuple] = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.imexlb_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, desc: InstanceDesc, storage: str | None = None) -> int:
        """Admit an instance (in the engine's storage format, or in `storage`);
        raises ImexlbError (code 4) when over budget."""
        slot = ctypes.c_int()
        st = STORAGES[storage or self.storage]
        _check(self.lib.imexlb_engine_add_as(self.h, ctypes.byref(desc), st, ctypes.byref(slot)))
        self.shapes[slot.value] = (desc.nx, desc.ny, desc.nz)
        return slot.value

    def try_add(self, desc: InstanceDesc, storage: str | None = None):
        """Admit an instance, or return None if it does not fit now."""
        slot = ctypes.c_int()
        st = STORAGES[storage or self.storage]
        rc = self.lib.imexlb_engine_add_as(self.h, ctypes.byref(desc), st, ctypes.byref(slot))
        if rc == 4:
            return None
        _check(rc)
        self.shapes[slot.value] = (desc.nx, desc.ny, desc.nz)
        return slot.value

    def checkpoint(self, slot: int) -> bytes:
        """One instance's state (current buffer, moments, step count)."""
        n = ctypes.c_size_t()
        _check(self.lib.imexlb_engine_checkpoint_size(self.h, slot, ctypes.byref(n)))
        buf = (ctypes.c_char * n.value)()
        _check(self.lib.imexlb_engine_checkpoint_save(self.h, slot, buf, n.value))
        return bytes(buf)

    def restore(self, desc: InstanceDesc, data: bytes) -> int:
        """Admit an instance from a checkpoint (same descriptor and storage)."""
        slot = ctypes.c_int()
        _check(self.lib.imexlb_engine_restore(self.h, ctypes.byref(desc), data, len(data), ctypes.byref(slot)))
        self.shapes[slot.value] = (desc.nx, desc.ny, desc.nz)
        return slot.value

    def remove(self, slot: int):
        _check(self.lib.imexlb_engine_remove(self.h, slot))
        self.shapes.pop(slot, None)

    def step(self, n: int = 1):
        _check(self.lib.imexlb_engine_step(self.h, n))

    def limit(self, slot: int, steps: int | None):
        """The instance takes at most `steps` more steps (None: no limit), then
        stays as it is while the others go on; its fields are written at its
        last step (imexlb_engine_limit)."""
        _check(self.lib.imexlb_engine_limit(self.h, slot, -1 if steps is None else int(steps)))

    def synchronize(self):
        _check(self.lib.imexlb_engine_synchronize(self.h))

    def fields(self, slot: int, out: dict | None = None) -> dict:
        """u, v, w, p of one instance after the last step, each (nz, ny, nx)."""
        nx, ny, nz = self.shapes[slot]
        if out is None:
            out = {k: np.empty((nz, ny, nx)) for k in ("u", "v", "w", "p")}
        _check(self.lib.imexlb_engine_fields(self.h, slot, _ptr(out["u"]), _ptr(out["v"]), _ptr(out["w"]),
                                             _ptr(out["p"])))
        return out

    def plane(self, slot: int, k: int) -> dict:
        """u, v, w, p of one z plane of an instance, each (ny, nx)."""
        nx, ny, nz = self.shapes[slot]
        out = {c: np.empty((ny, nx)) for c in ("u", "v", "w", "p")}
        _check(self.lib.imexlb_engine_plane(self.h, slot, k, _ptr(out["u"]), _ptr(out["v"]), _ptr(out["w"]),
                                            _ptr(out["p"])))
        return out

    def residuals(self) -> np.ndarray:
        out = np.empty(self.max_instances)
        _check(self.lib.imexlb_engine_residuals(self.h, _ptr(out), self.max_instances))
        return out

    def stats(self) -> dict:
        st = EngineStats()
        _check(self.lib.imexlb_engine_info(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in EngineStats._fields_}
