"""B200-native relativistic-MHD step of the Mara code (jzrake/ctf) behind a C ABI.

* ``ctf_b200.mara``  -- the reference's Lua ``Mara`` module surface (:data:`Mara`) and the
  object-level :class:`~ctf_b200.mara.Solver` over ``libmaragpu.so``;
* ``ctf_b200.ics``   -- seeded synthetic initial conditions;
* ``ctf_b200/csrc``  -- the CUDA kernels (sm_100a) and the C ABI (``include/mara_gpu.h``).
"""
__all__ = ["mara", "ics"]
