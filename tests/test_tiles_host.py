"""The tiling of the field solve's fine-level up leg (fine_up_tiles in csrc/pb_poisson.cuh),
on the host: for every grid shape and block count tried, each tile with its one-node halo
fits the kernel's shared-memory tile (UP_TILE_MAX floats), the counts stay within the grid,
and the nearly-equal partition the kernel derives from them covers every node once.  The
header is compiled with the host C++ compiler into a small driver."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "thruster_cx_code_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "pb_poisson.cuh"
int main() {
  const int ys[] = {2, 3, 5, 17, 54, 64, 65, 68, 99, 128, 129, 256, 257, 513, 1025};
  const int xs[] = {2, 3, 7, 65, 137, 195, 256, 284, 393, 512, 1024, 1025, 2049, 4097};
  const int bs[] = {1, 2, 37, 74, 148, 296};
  long checked = 0;
  for (int ny : ys) for (int nx : xs) for (int nb : bs) {
    int ty = 0, tx = 0;
    pb::fine_up_tiles(ny, nx, nb, &ty, &tx);
    if (ty < 1 || tx < 1 || ty > ny || tx > nx) { printf("BAD counts %d %d %d -> %d %d\n", ny, nx, nb, ty, tx); return 1; }
    // the kernel's partition: rows [t*ny/ty, (t+1)*ny/ty), columns likewise
    std::vector<int> seen((size_t)ny * nx, 0);
    for (int a = 0; a < ty; ++a) for (int b = 0; b < tx; ++b) {
      const int y0 = (int)((long long)a * ny / ty), y1 = (int)((long long)(a + 1) * ny / ty);
      const int x0 = (int)((long long)b * nx / tx), x1 = (int)((long long)(b + 1) * nx / tx);
      const long halo = (long)(y1 - y0 + 2) * (x1 - x0 + 2);
      if (y1 <= y0 || x1 <= x0 || halo > pb::UP_TILE_MAX) {
        printf("BAD tile %d %d %d -> %d %d: [%d,%d)x[%d,%d)\n", ny, nx, nb, ty, tx, y0, y1, x0, x1);
        return 1;
      }
      for (int y = y0; y < y1; ++y) for (int x = x0; x < x1; ++x) ++seen[(size_t)y * nx + x];
    }
    for (int v : seen) if (v != 1) { printf("BAD cover %d %d %d\n", ny, nx, nb); return 1; }
    ++checked;
  }
  printf("ok %ld\n", checked);
  return 0;
}
"""


def test_fine_up_tiles_fit_and_cover(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "tiles.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "tiles"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=False, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok ")
