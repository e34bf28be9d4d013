"""OU driving field: the host part (mode spectrum, OU random streams, inverse error
function, serialization) against the compiled reference, byte for byte, on the CPU."""
import ctypes

import pytest

from ctf_b200 import _lib
from ctf_b200.mara import new_ou_field


def _reference_field(tmp_path, nd, P0, zeta, k1, seed, dts):
    from oracle import RefOracle, Scheme
    ref = RefOracle(Scheme(n=(8, 8, 8) if nd == 3 else (8, 8)))
    ref.dostring(f"""
    local f = Mara.new_ou_field({nd}, {P0!r}, {zeta!r}, {k1}, {seed})
    local g = io.open('{tmp_path}/A.bin', 'wb'); g:write(f); g:close()
    Mara.set_driving(f)
    for _, dt in ipairs({{{', '.join(repr(d) for d in dts)}}}) do Mara.driving.Advance(dt) end
    local s = Mara.driving.Serialize()
    g = io.open('{tmp_path}/B.bin', 'wb'); g:write(s); g:close()
    """)
    ref.close()
    return open(f"{tmp_path}/A.bin", "rb").read(), open(f"{tmp_path}/B.bin", "rb").read()


@pytest.mark.parametrize("nd,P0,zeta,k1,seed", [(3, 0.01, 1.0, 3, 12345), (3, 0.2, 0.3, 2, 7), (2, 0.05, 0.5, 3, 99)])
def test_field_and_ou_steps_match_the_reference_bytes(tmp_path, nd, P0, zeta, k1, seed):
    dts = [0.01, 0.02, 0.005]
    A, B = _reference_field(tmp_path, nd, P0, zeta, k1, seed, dts)
    f = new_ou_field(nd, P0, zeta, k1, seed)
    assert f == A
    lib = _lib.load()
    buf = ctypes.create_string_buffer(f, len(f))
    for dt in dts:
        assert lib.mgpu_ou_field_advance(buf, len(f), nd, dt) == 0
    assert buf.raw[:len(f)] == B


def test_corrupt_field_is_rejected():
    lib = _lib.load()
    f = new_ou_field(3, 0.01, 1.0, 3, 1)
    buf = ctypes.create_string_buffer(f[:-8], len(f) - 8)
    assert lib.mgpu_ou_field_advance(buf, len(f) - 8, 3, 0.01) == 1
    assert lib.mgpu_ou_field_advance(ctypes.create_string_buffer(f, len(f)), len(f), 2, 0.01) == 1
