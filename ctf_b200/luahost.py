"""Run Mara driver scripts (Lua 5.2) on the GPU module.

`LuaHost` embeds the interpreter of ctf_b200/_lib/libmaralua.so: the reference's vendored
Lua 5.2.1 with the `Mara` module replaced by this project's drop-in (ctf_b200/lua/lmara_gpu.c)
and the reference's own `buffer` module, both preloaded as globals as ctf-core/ctf.c does.

    python -m ctf_b200.luahost script.lua [args...]     # `arg` holds the arguments

The library is built by `make -C ctf_b200/lua` (it compiles the Lua sources the reference
vendors, where they lie); there is no fallback interpreter.
"""
from __future__ import annotations

import ctypes
import os
import sys

from . import _lib

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libmaralua.so")
LUA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lua")


class LuaError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    import subprocess
    if force or not os.path.exists(LIB_PATH):
        _lib.build()
        subprocess.run(["make", "-s", "-C", LUA_DIR], check=True)
    return LIB_PATH


_so = None


def _load():
    global _so
    if _so is None:
        if not os.path.exists(LIB_PATH):
            raise LuaError(f"{LIB_PATH} is missing: build it with `make -C ctf_b200/lua`")
        _lib.load()   # libmaragpu.so first (libmaralua.so links it by rpath)
        so = ctypes.CDLL(LIB_PATH)
        so.mlua_open.restype = ctypes.c_void_p
        so.mlua_open.argtypes = []
        so.mlua_dostring.restype = ctypes.c_int
        so.mlua_dostring.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        so.mlua_error.restype = ctypes.c_char_p
        so.mlua_error.argtypes = []
        so.mlua_close.restype = None
        so.mlua_close.argtypes = [ctypes.c_void_p]
        _so = so
    return _so


class LuaHost:
    """One Lua state with `Mara` (GPU) and `buffer` preloaded."""

    def __init__(self):
        self.so = _load()
        self.L = self.so.mlua_open()
        if not self.L:
            raise LuaError("could not create a Lua state")

    def run(self, code: str):
        if self.so.mlua_dostring(self.L, code.encode()):
            raise LuaError(self.so.mlua_error().decode())

    def close(self):
        if self.L:
            self.so.mlua_close(self.L)
            self.L = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv:
        print(__doc__)
        return 2
    script = argv[0]
    with LuaHost() as h:
        args = ", ".join(repr(a).replace("'", '"') for a in argv[1:])
        h.run(f"arg = {{[0] = {script!r}, {args}}}".replace("'", '"'))
        h.run(open(script).read())
    return 0


if __name__ == "__main__":
    sys.exit(main())
