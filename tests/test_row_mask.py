"""The checked-row masks of the two-step FD kernels, on the host.

fd_fwd_warp2 / fd_adj_warp2 (swd_b200/csrc/fd_warp.cuh) and the two-shots-per-warp kernels
(fd_warpx.cuh) decide per row whether row k or k-1 needs the checked path (rows <= 1, >= NZ-2,
the free surface, the receiver row and, forward, the source rows sx-2 .. sx of each shot of the
warp) with one bit test on a 64-bit mask that slow_rows builds over the rows zs-2 .. zs+61 of a
chunk.  This compiles slow_rows (the same function the kernels call) for the host and checks, for
every chunk of up to 60 rows (the cap of the warp schedules), ring depths 4, 6 and 8, no source
(adjoint), one source and two sources, that the bit test of the kernels' main loop equals the
chain of compares it replaced.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SRC = r"""
#include <cstdio>
#include "fd_warp.cuh"
using swd::slow_rows;
using swd::kNoSourceRow;
using swd::kWarpChunkMax;

int main() {
  long checked = 0, bad = 0;
  for (int NZ = 8; NZ <= 130; NZ += 3)
    for (int pad_top = 1; pad_top <= 2; ++pad_top)
      for (int gz = pad_top; gz <= pad_top + 3; ++gz)
        for (int spx = pad_top; spx <= NZ - 3; spx += 7)
          for (int chunk = 1; chunk <= kWarpChunkMax; ++chunk)
            for (int zs = 1; zs <= NZ - 2; zs += chunk)
              for (int nsrc = 0; nsrc <= 2; ++nsrc)
                for (int NS = 4; NS <= 8; NS += 2) {
                  const int ze = zs + chunk < NZ - 1 ? zs + chunk : NZ - 1;
                  const int mb = zs - 2;
                  // the second shot of a two-shot warp sits a few rows lower (or at the same row)
                  const int s0 = nsrc >= 1 ? spx : kNoSourceRow;
                  const int s1 = nsrc >= 2 ? pad_top + (spx * 5) % (NZ - 2 - pad_top) : kNoSourceRow;
                  const unsigned long long m = slow_rows(NZ, pad_top, gz, zs, s0, s1);
                  auto src = [&](int k, int s) { return s != kNoSourceRow && k >= s - 2 && k <= s; };
                  auto slow1 = [&](int k) {
                    return k <= 1 || k >= NZ - 2 || k == pad_top || k == gz || src(k, s0) || src(k, s1);
                  };
                  // the main loop of the kernels: k1 = zs+1, zs+1+NS, ... while k1 + NS <= ze + 1
                  for (int k1 = zs + 1; k1 + NS <= ze + 1; k1 += NS) {
                    const unsigned w = (unsigned)(m >> (k1 - 1 - mb));
                    for (int u = 0; u < NS; ++u) {
                      const bool mask = (w & (3u << u)) != 0;
                      const bool chain = slow1(k1 + u) || slow1(k1 + u - 1);
                      ++checked;
                      if (mask != chain) {
                        if (bad < 5) printf("NZ %d pad %d gz %d sp %d chunk %d zs %d nsrc %d NS %d k %d\n", NZ,
                                            pad_top, gz, spx, chunk, zs, nsrc, NS, k1 + u);
                        ++bad;
                      }
                    }
                  }
                }
  printf("checked %ld rows, %ld mismatches\n", checked, bad);
  return bad != 0;
}
"""


@pytest.mark.skipif(not (os.path.exists(NVCC) or shutil.which("nvcc")), reason="nvcc not available")
def test_row_mask_equals_the_compare_chain(tmp_path):
    src = tmp_path / "row_mask.cu"
    src.write_text(SRC)
    exe = tmp_path / "row_mask"
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    subprocess.run([nvcc, "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "swd_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert "0 mismatches" in out.stdout
