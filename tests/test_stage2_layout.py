"""Host logic of the stage-2 product basis: the storage order of the vectors
Y_jk = U_k(H~_2) w_j (two parity classes, row-major (j, k) within each) that
the pass chains write and the GEMM reads, compiled from the library's own
header. Every (j, k) must get a distinct row of its class, the classes must
cover Kb x K2 rows, and pair() must invert index()."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "mqw_internal.h"
int main() {
  int bad = 0, cases = 0;
  for (int Kb = 1; Kb <= 70; Kb++)
    for (int K2 = 1; K2 <= 90; K2++) {
      const mqw::S2Layout lay{Kb, K2};
      if (lay.rows(0) + lay.rows(1) != Kb * K2) bad++;
      for (int h = 0; h < 2; h++) {
        std::vector<int> seen(lay.rows(h), 0);
        for (int j = 0; j < Kb; j++)
          for (int k = 0; k < K2; k++) {
            if (((j + k) & 1) != h) continue;
            const int q = lay.index(j, k);
            if (q < 0 || q >= lay.rows(h) || seen[q]++) { bad++; continue; }
            int jj = -1, kk = -1;
            lay.pair(h, q, &jj, &kk);
            if (jj != j || kk != k) bad++;
            cases++;
          }
      }
    }
  printf("%d %d\n", bad, cases);
  return bad != 0;
}
"""


def test_stage2_layout_is_a_bijection(tmp_path):
    if not shutil.which("g++") or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are not available")
    src = tmp_path / "lay.cpp"
    exe = tmp_path / "lay"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CUDA_INC, "-I",
                    os.path.join(ROOT, "multistageqw_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    bad, cases = map(int, r.stdout.split())
    assert r.returncode == 0 and bad == 0
    assert cases == sum(kb * k2 for kb in range(1, 71) for k2 in range(1, 91))
