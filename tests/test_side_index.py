"""The kernels' table-free side/volume index arithmetic (csrc/side_index.h) equals the host maps
built with the reference's conventions (host_setup.cpp side_to_vol, mappings.f90:262-464) for every
N, local side, flip and face point; compiled and run on the CPU."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fluxo_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include "host_setup.h"
#include "side_index.h"
// the library's error recorder (fluxo_gpu.cu), which host_setup.cpp reports through
namespace fluxo { int record_unbound_error(int code, const std::string&) { return code; } }
int main() {
  int bad = 0, checked = 0;
  for (int N = 1; N <= 9; ++N)
    for (int s = 1; s <= 6; ++s)
      for (int flip = 0; flip <= 4; ++flip)
        for (int q = 0; q <= N; ++q)
          for (int p = 0; p <= N; ++p) {
            int ijk[3];
            fluxo::host::side_to_vol(N, 0, p, q, flip, s, ijk);
            const int n = ijk[0] + (N + 1) * (ijk[1] + (N + 1) * ijk[2]);
            bad += fluxo::side_node(N, p, q, flip, s) != n;
            bad += fluxo::node_side_point(N, s, flip, ijk[0], ijk[1], ijk[2]) != p + (N + 1) * q;
            ++checked;
          }
  std::printf("%d %d\n", checked, bad);
  return bad != 0;
}
"""


def test_side_index_matches_host_maps():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        with open(src, "w") as f:
            f.write(PROGRAM)
        subprocess.run(["g++", "-O1", "-std=c++17", "-I" + CSRC, src, os.path.join(CSRC, "host_setup.cpp"), "-o", exe],
                       check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        checked, bad = map(int, r.stdout.split())
        assert r.returncode == 0 and bad == 0 and checked > 0
