"""The pressure solver's tiled, circularly skewed layout (sc_common.cuh) checked
on the CPU: the solver's own index functions, compiled as host code, on odd and
non-power-of-two grids.  Tiled::off is a bijection onto the padded tiles and
Tiled::coords inverts it; Cell::init, walked over every row block and thread as
the kernels walk it, lands on off(x, y, z); and the six neighbour offsets equal
off() of the neighbour's coordinates wherever the neighbour lies inside the
padded extent, across tile edges and the slot wrap included."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SRC = r'''
#include <cstdio>
#include <vector>
#include "sc_common.cuh"
using sc::Cell;
using sc::Tiled;
#define CHECK(c) do { if (!(c)) { std::printf("FAIL %s at line %d (%d %d %d)\n", #c, __LINE__, nx, ny, nz); return 1; } } while (0)
int run(int nx, int ny, int nz) {
  const Tiled g = Tiled::make(nx, ny, nz);
  const int px = g.ntx * 32, py = g.nty * Tiled::TY;  // padded extents
  std::vector<char> seen(g.total, 0);
  for (int x = 0; x < px; x++)
    for (int y = 0; y < py; y++)
      for (int z = 0; z < nz; z++) {
        const int64_t e = g.off(x, y, z);
        CHECK(e >= 0 && e < g.total && !seen[e]);
        seen[e] = 1;
        int a, b, c;
        const bool in = g.coords(e, a, b, c);
        CHECK(a == x && b == y && c == z && in == (x < nx && y < ny));
      }
  for (int64_t e = 0; e < g.total; e++) CHECK(seen[e]);
  const int nrb = g.ntiles() * nz;
  for (int rb = 0; rb < nrb; rb++)
    for (int tid = 0; tid < Tiled::TY * 32; tid++) {
      Cell c;
      c.init(g, rb, tid);
      CHECK(c.e == g.off(c.x, c.y, c.z));
      CHECK(c.inside == (c.x < nx && c.y < ny));
      if (c.x > 0) CHECK(c.xm(g) == g.off(c.x - 1, c.y, c.z));
      if (c.x < px - 1) CHECK(c.xp(g) == g.off(c.x + 1, c.y, c.z));
      if (c.y > 0) CHECK(c.ym(g) == g.off(c.x, c.y - 1, c.z));
      if (c.y < py - 1) CHECK(c.yp(g) == g.off(c.x, c.y + 1, c.z));
      if (c.z > 0) CHECK(c.zm(g) == g.off(c.x, c.y, c.z - 1));
      if (c.z < nz - 1) CHECK(c.zp(g) == g.off(c.x, c.y, c.z + 1));
    }
  return 0;
}
int main() {
  const int sizes[][3] = {{17, 9, 13}, {40, 20, 13}, {33, 17, 1}, {64, 8, 31}, {5, 3, 2},
                          {32, 8, 32}, {1, 1, 1},    {31, 9, 2},  {65, 24, 33}, {12, 12, 40}};
  for (const auto& s : sizes)
    if (run(s[0], s[1], s[2])) return 1;
  std::printf("ok\n");
  return 0;
}
'''


def test_tiled_layout_index_arithmetic(tmp_path):
    nvcc = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc) and shutil.which(nvcc) is None:
        pytest.skip("no nvcc")
    src = tmp_path / "layout.cu"
    src.write_text(_SRC)
    exe = tmp_path / "layout"
    subprocess.check_call([nvcc, "-std=c++17", "-O1", "-ccbin", "g++", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                           os.path.join(ROOT, "simcraft_b200", "csrc"), str(src), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
