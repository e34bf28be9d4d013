"""Host-side mirror of the reference's Lua module ``Mara`` over the B200 C ABI.

The reference's drivers (``modules/MaraSim.lua``, ``ctf-core/run-mara.lua``) call::

    Mara.start(); Mara.set_fluid('rmhd'); Mara.set_eos('gamma-law', 4/3)
    Mara.set_boundary('periodic'); Mara.set_riemann('hlld'); Mara.set_godunov('plm-split')
    Mara.set_advance('rk2'); Mara.config_solver{extrap='plm', theta=2.0}
    Mara.set_domain({0,0,0}, {1,1,1}, {N,N,N}, 8, 3)
    local kzps, errors = Mara.advance(P, dt);  local dt = Mara.get_timestep(0.3)

The same calls, with the same argument meaning, names and error behaviour (misuse raises
:class:`MaraError`, the analogue of ``luaL_error``; numerical failure is a returned error
count with the state left unchanged), work on :data:`Mara` here, with the step running on
the GPU (``Mara/mara.cpp:137-1167`` is the surface mirrored).  ``P`` is a float64 numpy
array in the reference's AoS layout with guard zones, shape ``(G0, G1, G2, 8)``.

:class:`Solver` is the object-level API under it: one handle, device-resident state.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, replace

import numpy as np

from . import _lib

RECON = {"pcm": 0, "plm": 1, "weno5": 2}
RIEMANN = {"hll": 0, "hllc": 1, "hlld": 2}
ADVANCE = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}
IS_MODE = {"js96": 0, "b08": 1, "sz10": 2}
PRECISION = {"fp64": 0, "fp32": 1}
GODUNOV = {"plm-split": 0, "plm-muscl": 1}   # method of lines / CTU-Hancock
LAYOUT = {"standard": 0, "lean": 1}          # device memory layout (include/mara_gpu.h)
PRIM_NAMES = ["rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"]   # Mara/rmhd.cpp:72-78


class MaraError(RuntimeError):
    """API misuse (the reference raises luaL_error in these cases)."""


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class Scheme:
    """Solver selection (the union of the reference's set_* selectors and config_solver)."""
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
    precision: str = "fp64"
    learned_c2p: bool = False
    godunov: str = "plm-split"   # 'plm-muscl': CTU-Hancock with PLM slopes of limiter theta
    layout: str = "standard"     # 'lean': 144 B per zone in FP32 bulk, for 3D boxes up to 1024^3

    def to_config(self) -> _lib.MgpuConfig:
        lib = _lib.load()
        c = _lib.MgpuConfig()
        lib.mgpu_default_config(ctypes.byref(c))
        c.gamma = self.gamma
        c.recon = RECON[self.extrap]
        c.theta = self.theta
        c.is_mode = IS_MODE[self.IS]
        c.sz10A = self.sz10A
        c.riemann = RIEMANN[self.riemann]
        c.rk = ADVANCE[self.advance]
        c.pfloor = self.pfloor
        c.ereset = int(self.ereset)
        c.preset = self.preset
        c.dreset = self.dreset
        c.precision = PRECISION[self.precision]
        c.learned_c2p = int(self.learned_c2p)
        c.godunov = GODUNOV[self.godunov]
        c.layout = LAYOUT[self.layout]
        return c


class Solver:
    """One GPU solver handle with a device-resident primitive state."""

    def __init__(self, scheme: Scheme, n, x0=None, x1=None, ng: int = 3, stream=None, lib_variant: str = ""):
        self.lib = _lib.load(lib_variant)
        self.scheme = scheme
        h = ctypes.c_void_p()
        cfg = scheme.to_config()
        rc = self.lib.mgpu_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise MaraError(f"mgpu_create failed ({rc})")
        self.h = h
        if stream is not None:
            self._check(self.lib.mgpu_set_stream(self.h, ctypes.c_void_p(stream)))
        n = tuple(int(v) for v in n)
        nd = len(n)
        x0 = tuple(x0) if x0 is not None else (0.0,) * nd
        x1 = tuple(x1) if x1 is not None else (1.0,) * nd
        self.n, self.nd, self.ng = n, nd, ng
        self.shape = tuple(v + 2 * ng for v in n) + (1,) * (3 - nd) + (8,)
        arr_x0 = (ctypes.c_double * nd)(*x0)
        arr_x1 = (ctypes.c_double * nd)(*x1)
        arr_n = (ctypes.c_int * nd)(*n)
        self._check(self.lib.mgpu_set_domain(self.h, arr_x0, arr_x1, arr_n, nd, 8, ng))

    def _check(self, rc):
        if rc:
            raise MaraError(f"[Mara] {self.lib.mgpu_last_error(self.h).decode()} (code {rc})")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_zones(self) -> int:
        nz = ctypes.c_longlong()
        self._check(self.lib.mgpu_num_zones(self.h, ctypes.byref(nz)))
        return nz.value

    def _check_buf(self, P):
        if not (isinstance(P, np.ndarray) and P.dtype == np.float64 and P.flags.c_contiguous):
            raise MaraError("[Mara] primitive must be a C-contiguous float64 array")
        if P.size != self.num_zones * 8:
            raise MaraError("[Mara] primitive has the wrong size for the domain")

    def upload(self, P: np.ndarray):
        self._check_buf(P)
        self._check(self.lib.mgpu_upload_prim(self.h, _dp(P)))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape)
        self._check_buf(out)
        self._check(self.lib.mgpu_download_prim(self.h, _dp(out)))
        return out

    def upload_range(self, P: np.ndarray, z0: int):
        """Zones [z0, z0 + len) of the guarded zone order from an (m, 8) float64 array."""
        P = np.ascontiguousarray(P, dtype=np.float64).reshape(-1, 8)
        self._check(self.lib.mgpu_upload_prim_range(self.h, _dp(P), int(z0), P.shape[0]))

    def download_range(self, z0: int, count: int) -> np.ndarray:
        out = np.empty((int(count), 8))
        self._check(self.lib.mgpu_download_prim_range(self.h, _dp(out), int(z0), int(count)))
        return out

    def upload_device(self, ptr: int):
        self._check(self.lib.mgpu_upload_prim_device(self.h, ctypes.c_void_p(ptr)))

    def download_device(self, ptr: int):
        self._check(self.lib.mgpu_download_prim_device(self.h, ctypes.c_void_p(ptr)))

    def advance(self, dt: float) -> int:
        e = ctypes.c_int()
        self._check(self.lib.mgpu_advance(self.h, ctypes.c_double(dt), ctypes.byref(e)))
        return e.value

    def advance_host(self, P: np.ndarray, dt: float):
        self._check_buf(P)
        kz, e = ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.mgpu_advance_host(self.h, _dp(P), ctypes.c_double(dt), ctypes.byref(kz),
                                               ctypes.byref(e)))
        return kz.value, e.value

    def set_pipeline(self, slabs: int):
        """Slabs of the pipelined advance_host: 0 off, -1 automatic (the default), >= 3."""
        self._check(self.lib.mgpu_set_pipeline(self.h, int(slabs)))

    def pipeline(self) -> tuple[int, int]:
        """(the slab setting, the slabs the last advance_host used -- 0 when unpipelined)."""
        s, last = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.mgpu_get_pipeline(self.h, ctypes.byref(s), ctypes.byref(last)))
        return s.value, last.value

    def advance_async(self, n: int, dt: float | None = None, cfl: float = 0.3):
        mode = 0 if dt is not None else 1
        self._check(self.lib.mgpu_advance_async(self.h, int(n), mode, ctypes.c_double(dt or 0.0),
                                                ctypes.c_double(cfl)))

    def synchronize(self):
        self._check(self.lib.mgpu_synchronize(self.h))

    def get_timestep(self, cfl: float) -> float:
        dt = ctypes.c_double()
        self._check(self.lib.mgpu_get_timestep(self.h, ctypes.c_double(cfl), ctypes.byref(dt)))
        return dt.value

    def stats(self) -> dict:
        s = _lib.MgpuStats()
        self._check(self.lib.mgpu_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    @property
    def max_lambda(self) -> float:
        return self.stats()["max_lambda"]

    def set_primitive(self, P: np.ndarray):
        self._check_buf(P)
        self._check(self.lib.mgpu_set_primitive(self.h, _dp(P)))

    def mean_max_divB(self):
        m, x = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mgpu_measure_divB(self.h, ctypes.byref(m), ctypes.byref(x)))
        return m.value, x.value

    def mean_max_divB_state(self):
        """Corner divergence of the committed state's (FP64) magnetic field."""
        m, x = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mgpu_measure_divB_state(self.h, ctypes.byref(m), ctypes.byref(x)))
        return m.value, x.value

    def max_lorentz_factor(self) -> float:
        w = ctypes.c_double()
        self._check(self.lib.mgpu_max_lorentz_factor(self.h, ctypes.byref(w)))
        return w.value

    # ---- the other Mara.measure.* (Mara/mara.cpp:1954-2230), on the measured array -----------
    def _vec(self, fn, n):
        out = (ctypes.c_double * n)()
        self._check(fn(self.h, out))
        return list(out)

    def _pair(self, fn):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(fn(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def mean_cons(self) -> list:
        return self._vec(self.lib.mgpu_measure_mean_cons, 8)

    def mean_prim(self) -> list:
        return self._vec(self.lib.mgpu_measure_mean_prim, 8)

    def mean_energies(self) -> dict:
        e = self._vec(self.lib.mgpu_measure_mean_energies, 4)
        return dict(zip(("magnetic", "kinetic", "internal", "total"), e))

    def mean_velocity(self) -> list:
        return self._vec(self.lib.mgpu_measure_mean_velocity, 4)

    def mean_max_temperature(self):
        return self._pair(self.lib.mgpu_measure_mean_max_temperature)

    def mean_max_magnetic_field(self):
        return self._pair(self.lib.mgpu_measure_mean_max_magnetic_field)

    def mean_max_sonic_mach(self):
        return self._pair(self.lib.mgpu_measure_mean_max_sonic_mach)

    def mean_min_alfvenic_mach(self):
        return self._pair(self.lib.mgpu_measure_mean_min_alfvenic_mach)

    # ---- Mara.diffuse / set_failmask, scheme changes in place -------------------------------
    def diffuse(self, r: float) -> int:
        """LaxDiffusion of strength r around the zones that failed the last c2p, on the
        committed state; returns the failed zones of its c2p."""
        e = ctypes.c_int()
        self._check(self.lib.mgpu_diffuse(self.h, ctypes.c_double(r), ctypes.byref(e)))
        return e.value

    def diffuse_host(self, P: np.ndarray, r: float) -> int:
        """Mara.diffuse(P, r): P is copied in, diffused and copied back."""
        self._check_buf(P)
        e = ctypes.c_int()
        self._check(self.lib.mgpu_diffuse_host(self.h, _dp(P), ctypes.c_double(r), ctypes.byref(e)))
        return e.value

    def set_failmask(self, value: int):
        self._check(self.lib.mgpu_set_failmask(self.h, int(value)))

    def reconfigure(self, scheme: "Scheme"):
        """Change the scheme in place (state, MaxLambda, failure mask and measured array kept)."""
        cfg = scheme.to_config()
        self._check(self.lib.mgpu_reconfigure(self.h, ctypes.byref(cfg)))
        self.scheme = scheme

    KERNEL_CLASSES = ["begin", "p2c", "c2p", "flux", "update", "predict"]

    def profile_enable(self, capacity: int = 4096):
        self._check(self.lib.mgpu_profile_enable(self.h, int(capacity)))

    def profile_disable(self):
        self._check(self.lib.mgpu_profile_disable(self.h))

    def profile_read(self) -> dict:
        """Per kernel class: summed ms, launches and work units since the last read."""
        k = len(self.KERNEL_CLASSES)
        ms = (ctypes.c_double * k)()
        ln = (ctypes.c_longlong * k)()
        un = (ctypes.c_longlong * k)()
        self._check(self.lib.mgpu_profile_read(self.h, ms, ln, un))
        return {k: {"ms": ms[i], "launches": ln[i], "units": un[i]}
                for i, k in enumerate(self.KERNEL_CLASSES)}

    def set_c2p_network(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.mgpu_set_c2p_network(
            self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))

    # ---- stochastic driving (Mara.set_driving / Mara.driving.*) ----------------------------
    def set_driving(self, field: bytes | None):
        """A serialized OU driving field (new_ou_field, or a checkpoint's); None clears it."""
        if field is None:
            self._check(self.lib.mgpu_set_driving(self.h, None, 0))
            return
        buf = ctypes.create_string_buffer(bytes(field), len(field))
        self._check(self.lib.mgpu_set_driving(self.h, buf, len(field)))

    def driving_advance(self, dt: float):
        self._check(self.lib.mgpu_driving_advance(self.h, float(dt)))

    def driving_resample(self):
        self._check(self.lib.mgpu_driving_resample(self.h))

    def driving_serialize(self) -> bytes:
        n = ctypes.c_longlong()
        self._check(self.lib.mgpu_driving_serialize(self.h, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(max(n.value, 1))
        self._check(self.lib.mgpu_driving_serialize(self.h, buf, ctypes.byref(n)))
        return buf.raw[:n.value]

    def driving_power(self) -> float:
        p = ctypes.c_double()
        self._check(self.lib.mgpu_driving_power(self.h, ctypes.byref(p)))
        return p.value


def new_ou_field(nd: int, P0: float, zeta: float, k1: int, seed: int) -> bytes:
    """Mara.new_ou_field (Mara/mara.cpp:1378-1401): a serialized OU driving field."""
    lib = _lib.load()
    n = ctypes.c_longlong()
    if lib.mgpu_new_ou_field(nd, float(P0), float(zeta), k1, seed, None, ctypes.byref(n)):
        raise MaraError("[Mara] bad new_ou_field arguments")
    buf = ctypes.create_string_buffer(n.value)
    lib.mgpu_new_ou_field(nd, float(P0), float(zeta), k1, seed, buf, ctypes.byref(n))
    return buf.raw


class _Measure:
    def __init__(self, mod):
        self._m = mod

    def mean_max_divB(self):
        return self._m._solver().mean_max_divB()

    def max_lorentz_factor(self):
        return self._m._solver().max_lorentz_factor()

    def mean_cons(self):
        return self._m._solver().mean_cons()

    def mean_prim(self):
        return self._m._solver().mean_prim()

    def mean_energies(self):
        return self._m._solver().mean_energies()

    def mean_velocity(self):
        return self._m._solver().mean_velocity()

    def mean_max_temperature(self):
        return self._m._solver().mean_max_temperature()

    def mean_max_magnetic_field(self):
        return self._m._solver().mean_max_magnetic_field()

    def mean_max_sonic_mach(self):
        return self._m._solver().mean_max_sonic_mach()

    def mean_min_alfvenic_mach(self):
        return self._m._solver().mean_min_alfvenic_mach()


class _Fluid:
    def __init__(self, mod):
        self._m = mod

    def GetPrimNames(self):
        if self._m._fluid is None:
            raise MaraError("[Mara] need a fluid to run this, use set_fluid")
        return list(PRIM_NAMES)


class MaraModule:
    """The ``Mara`` table of the reference (Mara/mara.cpp:137-268), GPU-backed."""

    _ctu_theta = 2.0   # PlmCtuHancockOperator's plm_theta: process-wide, survives start()

    def __init__(self):
        self._reset()
        self.measure = _Measure(self)
        self.fluid = _Fluid(self)

    def _reset(self):
        self._scheme = Scheme()
        self._fluid = None
        self._boundary = None
        self._godunov = None
        self._domain = None
        self._s = None
        self._dirty = False
        self._started = False

    # lifecycle ---------------------------------------------------------------------------
    def start(self):
        """luaC_Mara_start (Mara/mara.cpp:271-287): a fresh application with defaults."""
        self.close()
        self._reset()
        self._started = True

    def close(self):
        if self._s is not None:
            self._s.close()
        self._s = None

    def _need_start(self):
        if not self._started:
            raise MaraError("[Mara] call Mara.start() first")

    def _invalidate(self):
        """A scheme change: applied to the solver in place at its next use (so MaxLambda,
        the failure mask and the measured array carry over, as in the reference's
        process-wide solver), or by a new solver where the change needs one."""
        self._dirty = True

    def _rebuild(self):
        if self._s is not None:
            self._s.close()
            self._s = None

    # selectors (Mara/mara.cpp:813-984, 1140-1167) ----------------------------------------
    def set_fluid(self, key: str):
        self._need_start()
        if key != "rmhd":
            raise MaraError(f"[Mara] no such fluid '{key}'" if key not in ("euler", "srhd")
                            else f"[Mara] fluid '{key}' is not provided by the B200 module")
        self._fluid = key
        self._rebuild()

    def set_eos(self, key: str, gamma: float = 1.4):
        self._need_start()
        if key != "gamma-law":
            raise MaraError(f"[Mara] no such eos '{key}'")
        self._scheme.gamma = float(gamma)
        self._invalidate()

    def set_boundary(self, key: str):
        self._need_start()
        if key != "periodic":
            raise MaraError(f"[Mara] no such boundary conditions '{key}'")
        self._boundary = key

    def set_riemann(self, key: str):
        self._need_start()
        if key not in RIEMANN:
            raise MaraError(f"[Mara] no such riemann solver '{key}'")
        self._scheme.riemann = key
        self._invalidate()

    def set_godunov(self, key: str):
        """luaC_set_godunov (Mara/mara.cpp:960-984).  A new operator carries the constructor's
        emergency-reset settings; 'plm-muscl' (CTU-Hancock) keeps its own limiter parameter,
        a process-wide static changed only by config_solver{theta} while it is the current
        operator (Mara/ctu-hancock.cpp:11, Mara/mara.cpp:1068-1074)."""
        self._need_start()
        if key == "weno-split":
            raise MaraError("[Mara] integration scheme 'weno-split' is not provided by the B200 module")
        if key not in GODUNOV:
            raise MaraError(f"[Mara] no such integration scheme '{key}'")
        d = Scheme()
        self._scheme.ereset, self._scheme.preset, self._scheme.dreset = d.ereset, d.preset, d.dreset
        self._godunov = key
        self._invalidate()

    def set_advance(self, key: str):
        self._need_start()
        if key not in ADVANCE:
            raise MaraError(f"[Mara] no such advance option '{key}'")
        self._scheme.advance = key
        self._invalidate()

    def config_solver(self, tbl: dict, quiet: bool = False):
        """luaC_config_solver (Mara/mara.cpp:996-1138); also accepts precision/learned_c2p."""
        self._need_start()
        s = self._scheme
        if "extrap" in tbl:
            if tbl["extrap"] not in RECON:
                raise MaraError(f"[Mara] no such extrap '{tbl['extrap']}'")
            s.extrap = tbl["extrap"]
        if "theta" in tbl:
            s.theta = float(tbl["theta"])
            if self._godunov == "plm-muscl":
                MaraModule._ctu_theta = s.theta
        if "IS" in tbl:
            if tbl["IS"] not in IS_MODE:
                raise MaraError(f"no such IS: {tbl['IS']}")
            s.IS = tbl["IS"]
        if "sz10A" in tbl:
            s.sz10A = float(tbl["sz10A"])
        if "pfloor" in tbl:
            s.pfloor = float(tbl["pfloor"])
        if "ereset" in tbl:
            s.ereset = bool(tbl["ereset"])
        if "preset" in tbl:
            s.preset = float(tbl["preset"])
        if "dreset" in tbl:
            s.dreset = float(tbl["dreset"])
        if "precision" in tbl:
            if tbl["precision"] not in PRECISION:
                raise MaraError(f"[Mara] no such precision '{tbl['precision']}'")
            s.precision = tbl["precision"]
        if "learned_c2p" in tbl:
            s.learned_c2p = bool(tbl["learned_c2p"])
        if not quiet:
            for k, v in tbl.items():
                print(f"[config] setting {k}={v}")
        self._invalidate()

    def set_domain(self, x0, x1, N, Nq: int = 8, Ng: int = 3):
        """luaC_set_domain (Mara/mara.cpp:726-755)."""
        self._need_start()
        if Nq != 8:
            raise MaraError("[Mara] the rmhd fluid has Nq = 8")
        self._domain = (tuple(x0), tuple(x1), tuple(int(v) for v in N), int(Ng))
        self._rebuild()

    def _solver(self) -> Solver:
        if self._domain is None:
            raise MaraError("[Mara] need a domain to run this, use set_domain")
        scheme = replace(self._scheme, godunov=self._godunov or "plm-split")
        if scheme.godunov == "plm-muscl":
            scheme.theta = MaraModule._ctu_theta
        if self._s is not None and self._dirty:
            try:
                self._s.reconfigure(scheme)
            except MaraError:
                self._rebuild()
        self._dirty = False
        if self._s is None:
            x0, x1, N, Ng = self._domain
            self._s = Solver(scheme, N, x0, x1, Ng)
        return self._s

    # state -------------------------------------------------------------------------------
    def init_prim(self, P: np.ndarray, f):
        """luaC_Mara_init_prim (Mara/mara.cpp:531-632): P[zone] = f(x, y, z) on interior zones."""
        s = self._solver()
        s._check_buf(P)
        x0, x1, N, Ng = self._domain
        nd = len(N)
        dx = [(x1[d] - x0[d]) / N[d] for d in range(nd)]
        G = s.shape
        it = [range(N[d]) for d in range(nd)]
        import itertools
        for idx in itertools.product(*it):
            pos = [x0[d] + dx[d] * (idx[d] + 0.5) for d in range(nd)] + [0.0] * (3 - nd)
            m = tuple(i + Ng for i in idx) + (0,) * (3 - nd)
            P[m] = f(*pos)
        del G
        s.set_primitive(P)

    def set_primitive(self, P: np.ndarray):
        self._solver().set_primitive(P)

    def advance(self, P: np.ndarray, dt: float):
        """luaC_Mara_advance (Mara/mara.cpp:297-341): returns (kzps, errors); P is updated in
        place only when errors == 0.  kzps counts guard zones, like the reference."""
        return self._solver().advance_host(P, dt)

    def get_timestep(self, cfl: float) -> float:
        return self._solver().get_timestep(cfl)

    def diffuse(self, P: np.ndarray, r: float):
        """luaC_Mara_diffuse (Mara/mara.cpp:343-366): P gets Lax diffusion of strength r
        around the zones that failed the last c2p (in place)."""
        self._solver().diffuse_host(P, r)

    def set_failmask(self, value: int):
        """luaC_Mara_set_failmask (Mara/mara.cpp:368-373)."""
        self._solver().set_failmask(value)


Mara = MaraModule()
