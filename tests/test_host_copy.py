"""The threaded host copies of the pipelined advance's pageable staging
(ctf_b200/csrc/host_copy.h), on the CPU: a small C++ program copies buffers of many sizes,
offsets and thread counts, back to back through one pool, and checks every byte."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER_DIR = os.path.join(HERE, "..", "ctf_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "host_copy.h"

int main()
{
  const size_t sizes[] = {0, 1, 4095, size_t(8) << 20, (size_t(8) << 20) + 1, (size_t(64) << 20) + 12345,
                          size_t(200) << 20};
  const int threads[] = {1, 3, 8};
  unsigned seed = 12345;
  for (int nt : threads) {
    HostCopyPool pool(nt);
    for (int rep = 0; rep < 3; ++rep)
      for (size_t n : sizes) {
        const size_t off = (size_t) rep * 7;   // unaligned starts too
        std::vector<unsigned char> src(n + off + 16), dst(n + off + 16, 0xAB);
        for (auto &c : src) { seed = seed * 1103515245u + 12345u; c = (unsigned char) (seed >> 16); }
        pool.copy(dst.data() + off, src.data() + off, n);
        if (memcmp(dst.data() + off, src.data() + off, n) != 0) { printf("mismatch %d %zu\n", nt, n); return 1; }
        for (size_t i = 0; i < off; ++i)
          if (dst[i] != 0xAB) { printf("before %d %zu\n", nt, n); return 1; }
        for (size_t i = off + n; i < dst.size(); ++i)
          if (dst[i] != 0xAB) { printf("after %d %zu\n", nt, n); return 1; }
      }
  }
  printf("ok\n");
  return 0;
}
"""


def test_host_copy_pool(tmp_path):
    src = tmp_path / "host_copy_test.cpp"
    exe = tmp_path / "host_copy_test"
    src.write_text(PROGRAM)
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", HEADER_DIR, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode != 0 and "not found" in (r.stderr or ""):
        pytest.skip("no C++ compiler")
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
