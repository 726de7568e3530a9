"""ORACLE — test infrastructure only (ctypes bindings).

Loads ``oracle/liboracle.so`` (the CPU restatement of the reference's
MultiQW.cpp, see ``mqw_oracle.cpp``) and, when it has been built, the partial
reference build ``oracle/_ref/libref_v{4,3}.so`` (the reference's own
``my_normcdfinvf`` and AVX-512 ``Clenshaw_step``, MultiQW.cpp:16-173).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; the product never does.

Parity status: partly pinned (see the header of ``mqw_oracle.cpp``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SAMPLES = 100  # MultiQW.cpp:257
CHEB_TOL = 1e-6  # MultiQW.cpp:440

_P = ctypes.POINTER
_c_int, _c_float, _c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double


class DiagInfo(ctypes.Structure):
    _fields_ = [
        ("e0", ctypes.c_double),
        ("emax", ctypes.c_double),
        ("mid", ctypes.c_double),
        ("e_abs", ctypes.c_float),
        ("e_loc", ctypes.c_uint32),
    ]


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P(ctype))


def reference_dir() -> str | None:
    """The reference checkout to build the partial reference from: the
    directory named by MQW_REFERENCE_DIR, else a checkout named `reference`
    beside this repository; None when neither holds MultiQW.cpp."""
    env = os.environ.get("MQW_REFERENCE_DIR")
    cands = [env] if env else [os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.exists(os.path.join(c, "MultiQW.cpp")):
            return c
    return None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and the partial reference build when the
    reference tree is present)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.check_call(["make", "-C", HERE, "liboracle.so"], stdout=out)
    ref_src = reference_dir()
    if ref_src:
        subprocess.check_call(["make", "-C", HERE, "ref", f"REF={ref_src}"], stdout=out)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_inv_norm_upper.restype = _c_float
        L.orc_inv_norm_upper.argtypes = [_c_float]
        L.orc_set_inv_norm.argtypes = [ctypes.c_void_p]
        L.orc_set_inv_norm.restype = None
        L.orc_load_instance.argtypes = [_c_int, _P(_c_double), _P(_c_float), _P(_c_float)]
        L.orc_energies_ref.argtypes = [_c_int, _P(_c_double), _P(_c_double), _P(_c_float), ctypes.c_void_p]
        L.orc_energies_exact.argtypes = [_c_int, _P(_c_double), _P(_c_double)]
        L.orc_schedule.argtypes = [_c_int, _c_int, _P(_c_double), _P(_c_float), _P(_c_float), _P(_c_float), _P(_c_float)]
        L.orc_cheb_coeffs.argtypes = [_c_double, _c_double, _P(_c_double), _c_int]
        L.orc_clenshaw_step_f32.argtypes = [_P(_c_float), _P(_c_float), _P(_c_float), _P(_c_float), _c_int, _c_float, _c_float, _c_float]
        L.orc_clenshaw_f32_ext.argtypes = [_c_int, _c_int, _P(_c_float), _P(_c_float), _c_float, _c_float, _P(_c_float), _P(_c_float), _c_int, ctypes.c_void_p]
        L.orc_clenshaw_f64.argtypes = [_c_int, _c_int, _P(_c_float), _P(_c_double), _c_float, _c_float, _P(_c_double), _P(_c_double), _c_int]
        L.orc_run_problems_ext.argtypes = [_c_int, _c_int, _P(_c_double), _c_int, _c_int, _c_int, _P(_c_double), _P(_c_float), _P(ctypes.c_uint32), _P(ctypes.c_longlong), ctypes.c_void_p]
        L.orc_run_sample_range_ext.argtypes = [_c_int, _c_int, _P(_c_double), _c_int, _c_int, _c_int, _P(_c_double), _P(ctypes.c_longlong), ctypes.c_void_p]
        _lib = L
    return _lib


_ref = None


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = line.split()
                    return all(x in fl for x in ("avx512f", "avx512bw", "avx512dq", "avx512vl"))
    except OSError:
        pass
    return False


def ref_lib():
    """The partial reference build, or None when it was not built."""
    global _ref
    if _ref is None:
        name = "libref_v4.so" if _cpu_has_avx512() else "libref_v3.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_my_normcdfinvf.restype = _c_float
        R.ref_my_normcdfinvf.argtypes = [_c_float]
        R.ref_clenshaw_step.argtypes = [_P(_c_float), _P(_c_float), _P(_c_float), _P(_c_float), ctypes.c_uint, _c_float, _c_float, _c_float]
        R.ref_gray.restype = ctypes.c_uint
        R.ref_gray.argtypes = [ctypes.c_uint]
        R.ref_log2_of_lsb.restype = ctypes.c_uint
        R.ref_log2_of_lsb.argtypes = [_c_int]
        _ref = R
    return _ref


def use_reference_inv_norm(on: bool) -> None:
    """Drive the oracle's schedule with the reference's own my_normcdfinvf
    (MultiQW.cpp:83-86, from the partial build) instead of this
    restatement's correctly rounded inverse normal (they differ by at most
    1 ulp at the heuristic's inputs)."""
    if on:
        R = ref_lib()
        if R is None:
            raise RuntimeError("partial reference build not available")
        lib().orc_set_inv_norm(ctypes.cast(R.ref_my_normcdfinvf, ctypes.c_void_p).value)
    else:
        lib().orc_set_inv_norm(None)


def ref_step_ptr():
    R = ref_lib()
    if R is None:
        return None
    return ctypes.cast(R.ref_clenshaw_step, ctypes.c_void_p).value


# --- python-level helpers -------------------------------------------------

def params_per_instance(n: int) -> int:
    return n * (n + 1) // 2


def inv_norm_upper(p: float) -> float:
    return lib().orc_inv_norm_upper(p)


def load_instance(n: int, raw: np.ndarray):
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    J = np.zeros(n * n, np.float32)
    h = np.zeros(n, np.float32)
    lib().orc_load_instance(n, _ptr(raw, _c_double), _ptr(J, _c_float), _ptr(h, _c_float))
    return J.reshape(n, n), h


def energies_ref(n: int, raw: np.ndarray):
    """Reference-arithmetic energies E (float64, by basis state), the shifted
    float diagonal H_P and the DiagInfo (E_0, E_max, E_abs, E_loc)."""
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    E = np.zeros(1 << n, np.float64)
    hp = np.zeros(1 << n, np.float32)
    info = DiagInfo()
    rc = lib().orc_energies_ref(n, _ptr(raw, _c_double), _ptr(E, _c_double), _ptr(hp, _c_float), ctypes.addressof(info))
    assert rc == 0
    return E, hp, info


def energies_exact(n: int, raw: np.ndarray) -> np.ndarray:
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    E = np.zeros(1 << n, np.float64)
    lib().orc_energies_exact(n, _ptr(raw, _c_double), _ptr(E, _c_double))
    return E


def schedule(n: int, m: int, raw: np.ndarray):
    """(gammas[m], short_t[m], times[m, 100], total_t) as float32."""
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    g = np.zeros(m, np.float32)
    st = np.zeros(m, np.float32)
    t = np.zeros(m * SAMPLES, np.float32)
    tot = np.zeros(1, np.float32)
    lib().orc_schedule(n, m, _ptr(raw, _c_double), _ptr(g, _c_float), _ptr(st, _c_float), _ptr(t, _c_float), _ptr(tot, _c_float))
    return g, st, t.reshape(m, SAMPLES), float(tot[0])


def cheb_coeffs(s: float, tol: float = CHEB_TOL, max_k: int = 8192) -> np.ndarray:
    c = np.zeros(max_k, np.float64)
    K = lib().orc_cheb_coeffs(float(s), float(tol), _ptr(c, _c_double), max_k)
    assert K > 0, K
    return c[:K].copy()


def clenshaw_step_f32(b1, b2, hp, psi, n, scale, gamma, coef):
    lib().orc_clenshaw_step_f32(_ptr(b1, _c_float), _ptr(b2, _c_float), _ptr(hp, _c_float), _ptr(psi, _c_float), n, scale, gamma, coef)


def ref_clenshaw_step(b1, b2, hp, psi, n, scale, gamma, coef):
    ref_lib().ref_clenshaw_step(_ptr(b1, _c_float), _ptr(b2, _c_float), _ptr(hp, _c_float), _ptr(psi, _c_float), n, scale, gamma, coef)


def clenshaw(n, coeffs, hp, gamma, scale, psi, psi_real=False, mode="f32", use_ref_step=False):
    """Planar state psi[2N] -> sum_k c_k T_k(H~) psi with the reference's
    complex-coefficient convention. mode 'f32' or 'f64'."""
    coeffs = np.ascontiguousarray(coeffs, dtype=np.float32)
    K = len(coeffs)
    if mode == "f32":
        psi = np.ascontiguousarray(psi, dtype=np.float32)
        hp = np.ascontiguousarray(hp, dtype=np.float32)
        out = np.zeros_like(psi)
        ext = ref_step_ptr() if use_ref_step else None
        if use_ref_step and ext is None:
            raise RuntimeError("partial reference build not available")
        lib().orc_clenshaw_f32_ext(n, K, _ptr(coeffs, _c_float), _ptr(hp, _c_float), gamma, scale, _ptr(psi, _c_float), _ptr(out, _c_float), int(psi_real), ext)
    else:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        hp = np.ascontiguousarray(hp, dtype=np.float64)
        out = np.zeros_like(psi)
        lib().orc_clenshaw_f64(n, K, _ptr(coeffs, _c_float), _ptr(hp, _c_double), gamma, scale, _ptr(psi, _c_double), _ptr(out, _c_double), int(psi_real))
    return out


def run_problems(n: int, m: int, raw: np.ndarray, count: int, samples_used: int = SAMPLES,
                 mode: str = "f32", use_ref_step: bool = False):
    """Whole reference pipeline for `count` instances. Returns a dict with
    p (float64[count]), total_t, e_loc and terms (summed Chebyshev degree)."""
    raw = np.ascontiguousarray(raw, dtype=np.float64).ravel()
    assert raw.size >= count * params_per_instance(n)
    p = np.zeros(count, np.float64)
    tt = np.zeros(count, np.float32)
    el = np.zeros(count, np.uint32)
    terms = np.zeros(count, np.int64)
    ext = ref_step_ptr() if use_ref_step else None
    if use_ref_step and ext is None:
        raise RuntimeError("partial reference build not available")
    rc = lib().orc_run_problems_ext(n, m, _ptr(raw, _c_double), count, samples_used,
                                    0 if mode == "f32" else 1, _ptr(p, _c_double), _ptr(tt, _c_float),
                                    _ptr(el, ctypes.c_uint32), _ptr(terms, ctypes.c_longlong), ext)
    if rc != 0:
        raise RuntimeError(f"orc_run_problems failed: {rc}")
    return {"p": p, "total_t": tt, "e_loc": el, "terms": terms}


def run_sample_range(n: int, m: int, raw: np.ndarray, s_begin: int, s_end: int,
                     mode: str = "f32", use_ref_step: bool = False):
    """Samples [s_begin, s_end) of one instance through the reference
    pipeline: (sum of their ground-state probabilities, summed degree)."""
    raw = np.ascontiguousarray(raw, dtype=np.float64).ravel()
    assert raw.size >= params_per_instance(n)
    ps = np.zeros(1, np.float64)
    terms = np.zeros(1, np.int64)
    ext = ref_step_ptr() if use_ref_step else None
    if use_ref_step and ext is None:
        raise RuntimeError("partial reference build not available")
    rc = lib().orc_run_sample_range_ext(n, m, _ptr(raw, _c_double), s_begin, s_end,
                                        0 if mode == "f32" else 1, _ptr(ps, _c_double),
                                        _ptr(terms, ctypes.c_longlong), ext)
    if rc != 0:
        raise RuntimeError(f"orc_run_sample_range failed: {rc}")
    return float(ps[0]), int(terms[0])


def sk_instances(n: int, count: int, seed: int, j_std: float = 1.0, h_std: float = 1.0) -> np.ndarray:
    """Seeded synthetic Sherrington–Kirkpatrick instances in the reference's
    file layout: per instance n(n-1)/2 J values (pairs (1,0),(2,0),(2,1),...)
    then n h values; J ~ N(0, j_std^2), h ~ N(0, h_std^2), float64."""
    rng = np.random.default_rng(seed)
    npair = n * (n - 1) // 2
    out = np.empty((count, npair + n), np.float64)
    for i in range(count):
        v = rng.standard_normal(npair + n)
        out[i, :npair] = v[:npair] * j_std
        out[i, npair:] = v[npair:] * h_std
    return out
