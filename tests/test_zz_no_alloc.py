"""The allocation-free propagation entry point (mqw_clenshaw_noalloc).

It serves callers that cannot allocate device memory — code that must not
synchronise the device, hosts whose own allocator or fixed memory budget owns
all device memory. It must give the same result as the
ordinary entry point (mqw_clenshaw), including on a second call that reuses
the working space the first call left behind, and it must refuse sizes beyond
its fixed working space with an error instead of touching memory.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(orc, n, seed):
    raw = orc.sk_instances(n, 1, seed)[0]
    _, hp, info = orc.energies_ref(n, raw)
    g, _, t, _ = orc.schedule(n, 2, raw)
    onenorm = float(np.float32(np.float32(info.e_abs) + np.float32(g[1]) * np.float32(n)))
    s = float(np.float32(np.float32(onenorm) * t[1, 5]))
    c = orc.cheb_coeffs(s).astype(np.float32)
    rng = np.random.default_rng(seed)
    N = 1 << n
    psi = (rng.standard_normal(N) + 1j * rng.standard_normal(N)) / np.sqrt(2 * N)
    return hp, c, float(g[1]), onenorm, psi


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("n", [8, 13, 16])
def test_noalloc_matches_allocating_entry_point(mqw, orc, precision, n):
    import torch
    ctx = mqw.Context(0)
    prec = mqw.FP32 if precision == "fp32" else mqw.FP64
    cdt = np.complex64 if prec == mqw.FP32 else np.complex128
    tdt = torch.complex64 if prec == mqw.FP32 else torch.complex128
    dev = torch.device("cuda", 0)
    for call in range(2):  # the second call runs on the scratch the first left behind
        hp, c, gamma, onenorm, psi = _case(orc, n, 100 * n + call)
        ref = ctx.clenshaw(n, c, hp, gamma, onenorm, psi.astype(cdt), precision)
        d_c = torch.from_numpy(c).to(dev)
        d_hp = torch.from_numpy(hp).to(dev)
        d_psi = torch.from_numpy(psi.astype(cdt)).to(dev)
        d_out = torch.empty(1 << n, dtype=tdt, device=dev)
        stream = torch.cuda.current_stream(dev)
        mqw.clenshaw_noalloc(prec, n, len(c), d_c.data_ptr(), d_hp.data_ptr(), gamma, onenorm,
                             d_psi.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        out = d_out.cpu().numpy()
        tol = 1e-6 if prec == mqw.FP32 else 1e-13
        assert np.linalg.norm(out - ref) <= tol * np.linalg.norm(ref), (n, precision, call)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_working_space(mqw):
    import torch
    dev = torch.device("cuda", 0)
    n = mqw.NOALLOC_MAX_N + 1
    # Arguments are checked before anything is launched; the buffers are
    # never touched.
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    p = buf.data_ptr()
    L = mqw.lib()
    st = L.mqw_clenshaw_noalloc(mqw.FP32, n, 4, ctypes.c_void_p(p), ctypes.c_void_p(p), 1.0, 10.0,
                                ctypes.c_void_p(p), ctypes.c_void_p(p + 64), None)
    assert st == 6  # MQW_ERR_UNSUPPORTED
    st = L.mqw_clenshaw_noalloc(mqw.FP32, 5, 4, ctypes.c_void_p(p), ctypes.c_void_p(p), 1.0, 10.0,
                                ctypes.c_void_p(p), ctypes.c_void_p(p + 64), None)
    assert st == 1  # n below the grid path's minimum
