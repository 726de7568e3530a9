"""Host logic of the stage-2 product basis: the storage order of the vectors
Y_jk = U_k(H~_2) w_j (two parity classes, row-major (j, k) within each) that
the pass chains write and the GEMM reads, compiled from the library's own
header (every (j, k) a distinct row of its class, the classes covering
Kb x K2 rows, pair() inverting index()); and the algebra the coefficient
kernel relies on, in numpy."""
import os
import shutil
import subprocess

import numpy as np
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


def _cheb_coeffs(s, K):
    """Coefficients of exp(i s x) = sum_k c_k T_k(x) (Jacobi-Anger), stored
    the library's way: the real value for even k and the imaginary part's
    value for odd k (actual coefficient i^(k mod 2) times the stored value)."""
    from scipy.special import jv
    k = np.arange(K)
    full = np.where(k == 0, 1.0, 2.0) * (1j ** k) * jv(k, s)
    return np.where(k % 2 == 0, full.real, full.imag)


def _recomb(c, K):
    """The library's recombination weights: sum_k c_k T_k = sum_j d_j U_j."""
    cc = np.zeros(K + 2)
    cc[:K] = c
    d = 0.5 * (cc[:K] - cc[2:K + 2])
    d[0] = cc[0] - 0.5 * cc[2]
    return d


def test_stage2_product_identity_numpy():
    """psi_2 = sum_{j,k} d1_j d2_k U_k(H2) U_j(H1) psi_0 with the real-GEMM
    split the stage-2 kernels use (class j + k even -> Re with sign -1 when
    both are odd, odd -> Im) equals two Chebyshev stages applied in turn, on
    random symmetric operators with spectra in [-1, 1]."""
    rng = np.random.default_rng(7)
    N = 48

    def op():
        a = rng.standard_normal((N, N))
        h = (a + a.T) / 2
        return h / (np.abs(np.linalg.eigvalsh(h)).max() * 1.01)

    H1, H2 = op(), op()
    psi0 = np.full(N, 1.0 / np.sqrt(N))
    s1, s2, K1, K2 = 7.3, 11.1, 24, 32

    def cheb_apply(H, c_stored, v):
        k = np.arange(len(c_stored))
        c = np.where(k % 2 == 0, c_stored, 1j * c_stored)
        t_prev, t = v.astype(complex), H @ v
        out = c[0] * t_prev + c[1] * t
        for kk in range(2, len(c)):
            t_prev, t = t, 2 * H @ t - t_prev
            out = out + c[kk] * t
        return out

    c1, c2 = _cheb_coeffs(s1, K1), _cheb_coeffs(s2, K2)
    direct = cheb_apply(H2, c2, cheb_apply(H1, c1, psi0))
    assert abs(np.linalg.norm(direct) - 1.0) < 1e-6  # both stages near-unitary

    def u_basis(H, v, K):
        out = [v, 2 * H @ v]
        while len(out) < K:
            out.append(2 * H @ out[-1] - out[-2])
        return out[:K]

    w = u_basis(H1, psi0, K1)
    Y = [[u for u in u_basis(H2, wj, K2)] for wj in w]
    D1, D2 = _recomb(c1, K1), _recomb(c2, K2)
    re = np.zeros(N)
    im = np.zeros(N)
    for j in range(K1):
        for k in range(K2):
            if (j + k) % 2 == 0:
                s = -1.0 if (j % 2 and k % 2) else 1.0
                re += s * D1[j] * D2[k] * Y[j][k]
            else:
                im += D1[j] * D2[k] * Y[j][k]
    np.testing.assert_allclose(re + 1j * im, direct, rtol=0, atol=1e-12)
