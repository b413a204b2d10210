"""ctypes bindings for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

* :class:`Oracle` wraps ``oracle/liboracle.so``, the C restatement of the
  reference step (``oracle/imexlb_oracle.c``).
* :class:`Reference` wraps ``oracle/_ref/libref_<case>.so``, the reference's
  own solver sources compiled here against the single-rank Kokkos/MPI
  stand-in (``oracle/ref_harness.cpp``); it exists only where the reference
  tree was available at build time.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {"tgv": 0, "cavity": 1, "sphere": 2}
Q = 27
GHOST = 3

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build_oracle() -> str:
    """Build oracle/liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return os.path.join(HERE, "liboracle.so")


_ORACLE_LIB = None


def oracle_lib():
    global _ORACLE_LIB
    if _ORACLE_LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        lib = ctypes.CDLL(path)
        lib.oracle_create.restype = ctypes.c_void_p
        lib.oracle_create.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [ctypes.c_void_p]
        for name in ("oracle_destroy", "oracle_initialize", "oracle_collision", "oracle_halo",
                     "oracle_streaming", "oracle_update"):
            getattr(lib, name).argtypes = [ctypes.c_void_p]
            getattr(lib, name).restype = None
        lib.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_step.restype = None
        lib.oracle_get_moments.argtypes = [ctypes.c_void_p] * 5
        lib.oracle_get_f.argtypes = [ctypes.c_void_p] * 2
        lib.oracle_get_usr.argtypes = [ctypes.c_void_p] * 2
        lib.oracle_extents.argtypes = [ctypes.c_void_p] * 4
        lib.oracle_system.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      _dp, _dp, _dp, _ip, _ip]
        lib.oracle_write_tecplot.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        lib.oracle_write_tecplot.restype = ctypes.c_int
        lib.oracle_threads.restype = ctypes.c_int
        lib.oracle_check_div3.argtypes = [ctypes.c_long, ctypes.c_ulonglong, ctypes.c_int]
        lib.oracle_check_div3.restype = ctypes.c_int
        lib.oracle_check_div.argtypes = [ctypes.c_long, ctypes.c_ulonglong, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_long)]
        lib.oracle_check_div.restype = ctypes.c_int
        lib.oracle_std_create.restype = ctypes.c_void_p
        lib.oracle_std_create.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 9
        lib.oracle_std_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_std_destroy.restype = None
        lib.oracle_std_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_std_step.restype = None
        lib.oracle_std_get_moments.argtypes = [ctypes.c_void_p] * 5
        lib.oracle_std_drag.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        _ORACLE_LIB = lib
    return _ORACLE_LIB


class Oracle:
    """The C restatement of one reference case at one rank."""

    def __init__(self, case: str, nx: int, ny: int, nz: int, tau0: float, rho0: float, u0: float,
                 ran_padded: np.ndarray | None = None):
        self.lib = oracle_lib()
        self.case = case
        self.n = (nx, ny, nz)
        self.pad = (nx + 2 * GHOST, ny + 2 * GHOST, nz + 2 * GHOST)
        ran = None
        if ran_padded is not None:
            ran = np.ascontiguousarray(ran_padded, dtype=np.int32).ravel()
            assert ran.size == self.pad[0] * self.pad[1] * self.pad[2]
        self.h = self.lib.oracle_create(CASES[case], nx, ny, nz, tau0, rho0, u0, _ptr(ran))
        if not self.h:
            raise ValueError("oracle_create failed")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def initialize(self):
        self.lib.oracle_initialize(self.h)

    def step(self, n: int = 1):
        self.lib.oracle_step(self.h, n)

    def moments(self):
        nx, ny, nz = self.n
        out = [np.empty(nx * ny * nz) for _ in range(4)]
        self.lib.oracle_get_moments(self.h, *[_ptr(a) for a in out])
        return [a.reshape(nz, ny, nx) for a in out]

    def f_padded(self):
        lx, ly, lz = self.pad
        f = np.empty(Q * lx * ly * lz)
        self.lib.oracle_get_f(self.h, _ptr(f))
        return f.reshape(lz, ly, lx, Q)

    def usr_padded(self):
        lx, ly, lz = self.pad
        u = np.empty(lx * ly * lz, dtype=np.int32)
        self.lib.oracle_get_usr(self.h, _ptr(u))
        return u.reshape(lz, ly, lx)

    def write_tecplot(self, path: str, n: int):
        rc = self.lib.oracle_write_tecplot(self.h, path.encode(), n)
        if rc:
            raise OSError(f"oracle_write_tecplot failed for {path}")


class OracleStd:
    """The standard-boundary specification (moving-lid cavity, sphere channel,
    and "slab": the cavity's lid and bottom wall with x and y periodic)."""

    def __init__(self, case: str, nx: int, ny: int, nz: int, tau0: float, rho0: float = 1.0, u0: float = 0.1,
                 lid_u: float = 0.0, inlet_u: float = 0.0, sphere_d: float = 0.0, sphere_c=(0.0, 0.0, 0.0)):
        self.lib = oracle_lib()
        self.n = (nx, ny, nz)
        kase = 3 if case == "slab" else CASES[case]  # ORACLE_SLAB: the cavity's rules, x and y periodic
        self.h = self.lib.oracle_std_create(kase, nx, ny, nz, tau0, rho0, u0, lid_u, inlet_u, sphere_d,
                                            *sphere_c)
        if not self.h:
            raise ValueError("oracle_std_create failed")

    def close(self):
        if self.h:
            self.lib.oracle_std_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def step(self, n: int = 1):
        self.lib.oracle_std_step(self.h, n)

    def moments(self):
        nx, ny, nz = self.n
        out = [np.empty(nx * ny * nz) for _ in range(4)]
        self.lib.oracle_std_get_moments(self.h, *[_ptr(a) for a in out])
        return [a.reshape(nz, ny, nx) for a in out]

    def drag(self):
        f = [ctypes.c_double() for _ in range(3)]
        self.lib.oracle_std_drag(self.h, *[ctypes.byref(x) for x in f])
        return tuple(x.value for x in f)


def oracle_system(case: str, rho0, R, Re, u0, time_in, inter_in, sx):
    lib = oracle_lib()
    tau, miu, ma = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    t_out, i_out = ctypes.c_int(), ctypes.c_int()
    lib.oracle_system(CASES[case], rho0, R, int(Re), u0, int(time_in), int(inter_in), int(sx),
                      ctypes.byref(tau), ctypes.byref(miu), ctypes.byref(ma), ctypes.byref(t_out),
                      ctypes.byref(i_out))
    return dict(tau=tau.value, miu=miu.value, Ma=ma.value, Time=t_out.value, inter=i_out.value)


# ---------------------------------------------------------------- reference
class RefSystem(ctypes.Structure):
    _fields_ = [("rho0", ctypes.c_double), ("R", ctypes.c_double), ("Re", ctypes.c_int),
                ("u0", ctypes.c_double), ("Time", ctypes.c_int), ("inter", ctypes.c_int),
                ("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int),
                ("miu", ctypes.c_double), ("tau", ctypes.c_double), ("Ma", ctypes.c_double),
                ("cs2", ctypes.c_double), ("cs", ctypes.c_double)]


def reference_available(case: str, fast: bool = False) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_{case}{'_fast' if fast else ''}.so"))


class Reference:
    """The reference's own solver (oracle/_ref) for one case.  fast=True loads
    the build without the stand-in's view bounds checks (for timing)."""

    def __init__(self, case: str, fast: bool = False):
        path = os.path.join(HERE, "_ref", f"libref_{case}{'_fast' if fast else ''}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.case = case
        self.lib = ctypes.CDLL(path)
        self.lib.ref_read_system.argtypes = [ctypes.c_char_p, ctypes.POINTER(RefSystem)]
        self.lib.ref_run.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_void_p] * 7

    @staticmethod
    def write_input(dirname: str, rho0, R, Re, u0, time, inter, nx, ny, nz):
        with open(os.path.join(dirname, "input.in"), "w") as fh:
            fh.write(f"{rho0!r}  {R!r}  {int(Re)}\n{u0!r}  {int(time)}  {int(inter)}\n"
                     f"{int(nx)} {int(ny)} {int(nz)}\n")

    def system(self, dirname: str) -> dict:
        s = RefSystem()
        if self.lib.ref_read_system(dirname.encode(), ctypes.byref(s)):
            raise OSError(dirname)
        return {k: getattr(s, k) for k, _ in RefSystem._fields_}

    def run(self, dirname: str, nsteps: int, warmup: int = 20, out_every: int = 0, want_f: bool = True):
        s = self.system(dirname)
        nx, ny, nz = s["sx"], s["sy"], s["sz"]
        lx, ly, lz = nx + 6, ny + 6, nz + 6
        mom = [np.empty(nx * ny * nz) for _ in range(4)]
        usr = np.empty(lx * ly * lz, dtype=np.int32)
        ran = np.empty(lx * ly * lz, dtype=np.int32)
        f = np.empty(Q * lx * ly * lz) if want_f else None
        rc = self.lib.ref_run(dirname.encode(), nsteps, warmup, out_every, *[_ptr(a) for a in mom],
                              _ptr(usr), _ptr(ran), _ptr(f))
        if rc:
            raise OSError(f"ref_run failed in {dirname}")
        out = dict(system=s, u=mom[0].reshape(nz, ny, nx), v=mom[1].reshape(nz, ny, nx),
                   w=mom[2].reshape(nz, ny, nx), p=mom[3].reshape(nz, ny, nx),
                   usr=usr.reshape(lz, ly, lx), ran=ran.reshape(lz, ly, lx))
        if want_f:
            out["f"] = f.reshape(lz, ly, lx, Q)
        return out


def run_reference_case(case: str, rho0, R, Re, u0, nx, ny, nz, nsteps, warmup=0, out_every=0,
                       want_f=True, workdir=None, fast=False):
    """Write input.in into a scratch directory and run the reference there
    (fast: the build without the stand-in's view bounds checks; same
    arithmetic)."""
    ref = Reference(case, fast=fast)
    d = workdir or tempfile.mkdtemp(prefix=f"imexlb_ref_{case}_")
    Reference.write_input(d, rho0, R, Re, u0, nsteps, max(out_every, 1), nx, ny, nz)
    res = ref.run(d, nsteps, warmup, out_every, want_f)
    res["dir"] = d
    return res
