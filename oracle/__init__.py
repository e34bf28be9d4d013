"""CPU oracles for the Mara RMHD step (test infrastructure only).

Two oracles live here; both are loaded only by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, never by the product package ``ctf_b200``:

* :class:`PortOracle` -- ``oracle/port/mara_port.c``, a single-threaded FP64 C restatement of
  the reference algorithm (built by ``make -C oracle port``).
* :class:`RefOracle` -- the reference itself, Mara + its vendored Lua 5.2.1 compiled from the
  reference sources by ``make -C oracle ref`` and driven through its own Lua module
  ``Mara`` (``Mara/mara.cpp:137-268``).

Both take and return the reference's AoS primitive layout: ``(G0, G1, G2, 8)`` float64 with
``Ng = 3`` guard zones per side, x slowest, component fastest (``Mara/hydro.cpp:80-110``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_port", "liboracle_port.so")
PORT_PERTURBED_SO = os.path.join(HERE, "_port", "liboracle_port_perturbed.so")
REF_SO = os.path.join(HERE, "_ref", "libmara_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

RECON = {"pcm": 0, "plm": 1, "weno5": 2}
GODUNOV = {"plm-split": 0, "plm-muscl": 1}
RIEMANN = {"hll": 0, "hllc": 1, "hlld": 2}
ADVANCE = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}
IS_MODE = {"js96": 0, "b08": 1, "sz10": 2}


@dataclass
class Scheme:
    """Solver selection, named as in the reference's Lua surface (``Mara/mara.cpp``)."""
    n: tuple = (8, 8, 8)
    x0: tuple = (0.0, 0.0, 0.0)
    x1: tuple = (1.0, 1.0, 1.0)
    ng: int = 3
    gamma: float = 4.0 / 3.0
    extrap: str = "plm"
    theta: float = 2.0
    IS: str = "js96"
    sz10A: float = 50.0
    riemann: str = "hlld"
    advance: str = "rk2"
    pfloor: float = -1.0
    ereset: bool = False
    preset: float = 1.0
    dreset: float = 1.0
    godunov: str = "plm-split"

    @property
    def nd(self) -> int:
        return len(self.n)

    @property
    def shape(self) -> tuple:
        return tuple(m + 2 * self.ng for m in self.n)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def build(which: str = "port") -> None:
    """Build an oracle library with ``make -C oracle <which>``."""
    subprocess.run(["make", "-s", "-C", HERE, which], check=True)


class _PortConfig(ctypes.Structure):
    _fields_ = [("nd", ctypes.c_int), ("n", ctypes.c_int * 3), ("ng", ctypes.c_int),
                ("x0", ctypes.c_double * 3), ("x1", ctypes.c_double * 3),
                ("gamma", ctypes.c_double), ("recon", ctypes.c_int),
                ("theta", ctypes.c_double), ("is_mode", ctypes.c_int),
                ("sz10A", ctypes.c_double), ("riemann", ctypes.c_int), ("rk", ctypes.c_int),
                ("pfloor", ctypes.c_double), ("ereset", ctypes.c_int),
                ("preset", ctypes.c_double), ("dreset", ctypes.c_double), ("godunov", ctypes.c_int)]


class _PortStats(ctypes.Structure):
    _fields_ = [("max_lambda", ctypes.c_double), ("hlld_success", ctypes.c_long),
                ("hlld_failure", ctypes.c_long), ("hlld_path", ctypes.c_int)]


class PortOracle:
    """The C restatement (``oracle/port/mara_port.c``)."""

    def __init__(self, scheme: Scheme, perturbed_libm: bool = False):
        so = PORT_PERTURBED_SO if perturbed_libm else PORT_SO
        if not os.path.exists(so):
            build("port")
        self.lib = ctypes.CDLL(so)
        self.scheme = scheme
        c = _PortConfig()
        self.lib.port_default_config(ctypes.byref(c))
        c.nd = scheme.nd
        for d in range(3):
            c.n[d] = scheme.n[d] if d < scheme.nd else 1
            c.x0[d] = scheme.x0[d] if d < scheme.nd else 0.0
            c.x1[d] = scheme.x1[d] if d < scheme.nd else 1.0
        c.ng = scheme.ng
        c.gamma = scheme.gamma
        c.recon = RECON[scheme.extrap]
        c.theta = scheme.theta
        c.is_mode = IS_MODE[scheme.IS]
        c.sz10A = scheme.sz10A
        c.riemann = RIEMANN[scheme.riemann]
        c.rk = ADVANCE[scheme.advance]
        c.pfloor = scheme.pfloor
        c.ereset = int(scheme.ereset)
        c.preset = scheme.preset
        c.dreset = scheme.dreset
        c.godunov = GODUNOV[scheme.godunov]
        self.cfg = c
        self.stats = _PortStats()
        L = self.lib
        L.port_reconstruct.restype = ctypes.c_double
        L.port_timestep.restype = ctypes.c_double
        L.port_max_lorentz_factor.restype = ctypes.c_double

    # whole step ---------------------------------------------------------------------
    def advance(self, prim: np.ndarray, dt: float) -> int:
        assert prim.dtype == np.float64 and prim.flags.c_contiguous
        err = ctypes.c_int()
        self.lib.port_advance(ctypes.byref(self.cfg), ctypes.byref(self.stats), _p(prim),
                              ctypes.c_double(dt), ctypes.byref(err))
        return err.value

    @property
    def max_lambda(self) -> float:
        return self.stats.max_lambda

    def get_timestep(self, cfl: float) -> float:
        return self.lib.port_timestep(ctypes.byref(self.cfg), ctypes.c_double(self.max_lambda),
                                      ctypes.c_double(cfl))

    def mean_max_divB(self, prim: np.ndarray):
        m, x = ctypes.c_double(), ctypes.c_double()
        self.lib.port_mean_max_divB(ctypes.byref(self.cfg), _p(prim), ctypes.byref(m),
                                    ctypes.byref(x))
        return m.value, x.value

    def max_lorentz_factor(self, prim: np.ndarray) -> float:
        return self.lib.port_max_lorentz_factor(ctypes.byref(self.cfg), _p(prim))

    MEASURES = {"mean_cons": (0, 8), "mean_prim": (8, 8), "mean_energies": (16, 4), "mean_velocity": (20, 4),
                "mean_max_temperature": (24, 2), "mean_max_magnetic_field": (26, 2),
                "mean_max_sonic_mach": (28, 2), "mean_min_alfvenic_mach": (30, 2)}

    def measure(self, name: str, prim: np.ndarray) -> list:
        """The measure `name` of Mara.measure on the interior zones of prim (as RefOracle.measure
        returns it)."""
        out = np.zeros(32)
        self.lib.port_measures(ctypes.byref(self.cfg), _p(np.ascontiguousarray(prim)), _p(out))
        a, n = self.MEASURES[name]
        return list(out[a:a + n])

    def diffuse(self, prim: np.ndarray, r: float, mask: np.ndarray, prev: np.ndarray):
        """Mara.diffuse(P, r) given the FailureMask and PrimitiveArray it reads; prim changes in
        place; returns the new mask and the c2p's failure count."""
        assert prim.dtype == np.float64 and prim.flags.c_contiguous
        m_in = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        m_out = np.zeros_like(m_in)
        pv = np.ascontiguousarray(prev, dtype=np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        e = self.lib.port_diffuse(ctypes.byref(self.cfg), _p(prim), ctypes.c_double(r),
                                  m_in.ctypes.data_as(ip), _p(pv), m_out.ctypes.data_as(ip))
        return m_out, e

    # per state ----------------------------------------------------------------------
    def prim_to_cons(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        U = np.zeros(8)
        e = self.lib.port_prim_to_cons(ctypes.byref(self.cfg), _p(P), _p(U))
        return U, e

    def cons_to_prim(self, U, guess=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        P = np.zeros(8) if guess is None else np.array(guess, dtype=np.float64)
        e = self.lib.port_cons_to_prim(ctypes.byref(self.cfg), _p(U), _p(P))
        return P, e

    def c2p_solve(self, U, solver: int, guess: int, Pguess=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        Pg = np.zeros(8) if Pguess is None else np.ascontiguousarray(Pguess, dtype=np.float64)
        P = np.zeros(8)
        it = ctypes.c_int()
        e = self.lib.port_c2p_solve(ctypes.byref(self.cfg), _p(U), solver, guess, _p(Pg), _p(P),
                                    ctypes.byref(it))
        return P, e, it.value

    def flux(self, P, dim):
        U, _ = self.prim_to_cons(P)
        P = np.ascontiguousarray(P, dtype=np.float64)
        F = np.zeros(8)
        ap, am = ctypes.c_double(), ctypes.c_double()
        self.lib.port_flux_and_eigenvalues(ctypes.byref(self.cfg), _p(U), _p(P), _p(F),
                                           ctypes.byref(ap), ctypes.byref(am), dim)
        return F, ap.value, am.value

    def riemann(self, Pl, Pr, dim):
        Pl = np.ascontiguousarray(Pl, dtype=np.float64)
        Pr = np.ascontiguousarray(Pr, dtype=np.float64)
        F = np.zeros(8)
        e = self.lib.port_riemann(ctypes.byref(self.cfg), ctypes.byref(self.stats), _p(Pl), _p(Pr),
                                  _p(F), dim)
        return F, e

    def reconstruct(self, v, op):
        v = np.ascontiguousarray(v, dtype=np.float64)
        return self.lib.port_reconstruct(ctypes.byref(self.cfg), ctypes.cast(v.ctypes.data + 16, _dp),
                                         op)

    def quartic(self, d):
        r = np.zeros(4)
        n = self.lib.port_quartic(*[ctypes.c_double(x) for x in d], _p(r))
        return r[:n]


class RefOracle:
    """The compiled reference, driven through its Lua module ``Mara``.

    Only one instance may be live at a time: the reference keeps its solver in
    process-global statics (``Mara/mara.cpp:135``, ``Mara/rmhd-c2p.c:97-104``)."""

    def __init__(self, scheme: Scheme, quiet: bool = True):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: build it with `make -C oracle ref`")
        self.lib = L = ctypes.CDLL(REF_SO)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_get_max_lambda.restype = ctypes.c_double
        L.ref_reconstruct.restype = ctypes.c_double
        L.ref_failure_mask.restype = ctypes.c_long
        L.ref_primitive_array.restype = ctypes.c_long
        self.scheme = s = scheme
        L.ref_open()
        lua = (f"Mara.start(); Mara.set_fluid('rmhd'); Mara.set_eos('gamma-law', {s.gamma!r}); "
               f"Mara.set_boundary('periodic'); Mara.set_riemann('{s.riemann}'); "
               f"Mara.set_godunov('{s.godunov}'); Mara.set_advance('{s.advance}'); "
               f"Mara.config_solver({{extrap='{s.extrap}', theta={s.theta!r}, IS='{s.IS}', "
               f"sz10A={s.sz10A!r}, pfloor={s.pfloor!r}, ereset={'true' if s.ereset else 'false'}, "
               f"preset={s.preset!r}, dreset={s.dreset!r}}}, true); "
               f"Mara.set_domain({{{','.join(repr(float(v)) for v in s.x0[:s.nd])}}}, "
               f"{{{','.join(repr(float(v)) for v in s.x1[:s.nd])}}}, "
               f"{{{','.join(str(int(v)) for v in s.n)}}}, 8, {s.ng})")
        if quiet:
            fd = os.dup(1)
            devnull = os.open(os.devnull, os.O_WRONLY)
            os.dup2(devnull, 1)
            try:
                self._do(lua)
            finally:
                os.dup2(fd, 1)
                os.close(fd)
                os.close(devnull)
        else:
            self._do(lua)

    def _do(self, code: str):
        if self.lib.ref_dostring(code.encode()):
            raise RuntimeError(self.lib.ref_last_error().decode())

    def dostring(self, code: str, quiet: bool = True):
        """Run Lua code in the reference's interpreter (`Mara` and `buffer` preloaded)."""
        if not quiet:
            return self._do(code)
        fd = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        try:
            self._do(code)
        finally:
            os.dup2(fd, 1)
            os.close(fd)
            os.close(devnull)

    def close(self):
        self.lib.ref_close()

    def advance(self, prim: np.ndarray, dt: float) -> int:
        assert prim.dtype == np.float64 and prim.flags.c_contiguous
        kz, er = ctypes.c_double(), ctypes.c_int()
        if self.lib.ref_advance(_p(prim), ctypes.c_long(prim.size), ctypes.c_double(dt),
                                ctypes.byref(kz), ctypes.byref(er)):
            raise RuntimeError(self.lib.ref_last_error().decode())
        self.kzps = kz.value
        return er.value

    @property
    def max_lambda(self) -> float:
        return self.lib.ref_get_max_lambda()

    def get_timestep(self, cfl: float) -> float:
        dt = ctypes.c_double()
        self.lib.ref_get_timestep(ctypes.c_double(cfl), ctypes.byref(dt))
        return dt.value

    def set_primitive(self, prim: np.ndarray):
        self.lib.ref_set_primitive(_p(prim), ctypes.c_long(prim.size))

    def mean_max_divB(self, prim: np.ndarray):
        self.set_primitive(prim)
        m, x = ctypes.c_double(), ctypes.c_double()
        self.lib.ref_mean_max_divB(ctypes.byref(m), ctypes.byref(x))
        return m.value, x.value

    def max_lorentz_factor(self, prim: np.ndarray) -> float:
        self.set_primitive(prim)
        w = ctypes.c_double()
        self.lib.ref_max_lorentz_factor(ctypes.byref(w))
        return w.value

    def diffuse(self, prim: np.ndarray, r: float):
        """Mara.diffuse(P, r) (Mara/mara.cpp:343-366), P changed in place."""
        assert prim.dtype == np.float64 and prim.flags.c_contiguous
        if self.lib.ref_diffuse(_p(prim), ctypes.c_long(prim.size), ctypes.c_double(r)):
            raise RuntimeError(self.lib.ref_last_error().decode())

    def set_failmask(self, value: int):
        self.dostring(f"Mara.set_failmask({int(value)})")

    def measure(self, name: str, prim: np.ndarray | None = None) -> list:
        """Mara.measure.<name>() on the reference's PrimitiveArray (set to `prim` first when
        given): its numbers, array entries, or mean_energies' magnetic, kinetic, internal,
        total."""
        if prim is not None:
            self.set_primitive(prim)
        out = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        if self.lib.ref_measure(name.encode(), out, 8, ctypes.byref(n)):
            raise RuntimeError(self.lib.ref_last_error().decode())
        return list(out[:n.value])

    def failure_mask(self) -> np.ndarray:
        """GodunovOperator's FailureMask, one entry per guarded zone."""
        n = int(np.prod(self.scheme.shape))
        out = np.zeros(n, dtype=np.int32)
        k = self.lib.ref_failure_mask(out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_long(n))
        return out[:k]

    def primitive_array(self) -> np.ndarray:
        """The application's PrimitiveArray (what the next Mara.diffuse reads as its guess)."""
        n = int(np.prod(self.scheme.shape)) * 8
        out = np.zeros(n)
        k = self.lib.ref_primitive_array(_p(out), ctypes.c_long(n))
        return out[:k]

    def prim_to_cons(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        U = np.zeros(8)
        e = self.lib.ref_prim_to_cons(_p(P), _p(U))
        return U, e

    def cons_to_prim(self, U, guess=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        P = np.zeros(8) if guess is None else np.array(guess, dtype=np.float64)
        e = self.lib.ref_cons_to_prim(_p(U), _p(P))
        return P, e

    def c2p_solve(self, U, solver: int, guess: int, Pguess=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        Pg = np.zeros(8) if Pguess is None else np.ascontiguousarray(Pguess, dtype=np.float64)
        P = np.zeros(8)
        it = ctypes.c_int()
        e = self.lib.ref_c2p_solver(_p(U), solver, guess, _p(Pg), ctypes.c_double(self.scheme.gamma),
                                    _p(P), ctypes.byref(it))
        return P, e, it.value

    def flux(self, P, dim):
        P = np.ascontiguousarray(P, dtype=np.float64)
        F = np.zeros(8)
        ap, am = ctypes.c_double(), ctypes.c_double()
        self.lib.ref_flux_and_eigenvalues(_p(P), dim, _p(F), ctypes.byref(ap), ctypes.byref(am))
        return F, ap.value, am.value

    def riemann(self, Pl, Pr, dim):
        Pl = np.ascontiguousarray(Pl, dtype=np.float64)
        Pr = np.ascontiguousarray(Pr, dtype=np.float64)
        F = np.zeros(8)
        e = self.lib.ref_riemann(_p(Pl), _p(Pr), dim, _p(F))
        return F, e

    def reconstruct(self, v, op):
        v = np.ascontiguousarray(v, dtype=np.float64)
        return self.lib.ref_reconstruct(ctypes.cast(v.ctypes.data + 16, _dp), op)
