"""multistageqw_b200 — B200-native multi-stage quantum-walk simulator.

Python binding over the C ABI in ``include/mqw.h`` (``_lib/libmqw.so``). The
entry points mirror the reference command ``MultiQW n m filename [start
problems]`` (Asa-Hopkins/MultiStageQW, MultiQW.cpp:241-458) and its internal
pieces:

* :func:`multiqw` — the command itself (reads the instance file, appends
  float32 ground-state probabilities to ``output_<n>_<m>``, prints
  ``total_t P`` per problem).
* :func:`run_problems` — the problem loop on in-memory instances.
* :class:`Plan` — a batch prepared once and executed on the GPU with its
  inputs resident in device memory; instances may mix n and m.
* :func:`schedule`, :func:`load_instance`, :func:`inv_norm_upper` — the host
  heuristics (no GPU needed).
* :func:`build_diag`, :func:`cheb_coeffs`, :func:`clenshaw` — the device
  pieces one at a time.

There is no CPU fallback: if the native library is missing the import of the
library raises, and if no sm_100 GPU is present :class:`Context` raises.
"""
from __future__ import annotations

import ctypes
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libmqw.so")
CLI_PATH = os.path.join(_HERE, "_lib", "MultiQW")

SAMPLES = 100
FP32, FP64, FP32C = 0, 1, 2  # FP32C: FP32 with compensated partner sums

_STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
    4: "I/O error", 5: "device wait timed out", 6: "unsupported",
    7: "no sm_100 CUDA device",
}


class MQWError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{_STATUS.get(status, status)}: {msg}" if msg else _STATUS.get(status, str(status)))


class Options(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("samples", ctypes.c_int),
        ("cheb_tol", ctypes.c_double),
        ("group", ctypes.c_int),
        ("resident_max_n", ctypes.c_int),
        ("stage_scale", ctypes.POINTER(ctypes.c_float)),
        ("tile_log", ctypes.c_int),
        ("graph", ctypes.c_int),
        ("lanes", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("lane_smem", ctypes.c_int),
        ("tma", ctypes.c_int),
        ("stage1_basis", ctypes.c_int),
        ("final_projection", ctypes.c_int),
        ("cluster", ctypes.c_int),
    ]


class DiagInfo(ctypes.Structure):
    _fields_ = [
        ("e0", ctypes.c_double),
        ("emax", ctypes.c_double),
        ("mid", ctypes.c_double),
        ("e_abs", ctypes.c_float),
        ("e_loc", ctypes.c_uint32),
    ]


class GridShape(ctypes.Structure):
    _fields_ = [
        ("tile_log", ctypes.c_int),
        ("cluster_log", ctypes.c_int),
        ("global_axes", ctypes.c_int),
        ("group", ctypes.c_int),
        ("lanes", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("lane_smem", ctypes.c_int),
        ("tma", ctypes.c_int),
        ("us_per_walk_pass", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TierPeaks(ctypes.Structure):
    _fields_ = [
        ("l2_read_gbs", ctypes.c_double),
        ("l2_copy_gbs", ctypes.c_double),
        ("smem_gbs", ctypes.c_double),
        ("hbm_copy_gbs", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class RunStats(ctypes.Structure):
    _fields_ = [
        ("instances", ctypes.c_longlong),
        ("trajectories", ctypes.c_longlong),
        ("terms", ctypes.c_longlong),
        ("term_amps", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("term_launches", ctypes.c_longlong),
        ("kernel_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_double),
        ("d2h_bytes", ctypes.c_double),
        ("pass_amps", ctypes.c_double),
        ("aux_bytes", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.POINTER
_vp = ctypes.c_void_p
_lib = None


def _bind(L):
    i, f, d, ll = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_longlong
    sig = {
        "mqw_abi_version": (i, []),
        "mqw_status_string": (ctypes.c_char_p, [i]),
        "mqw_default_options": (None, [_P(Options)]),
        "mqw_create": (i, [_P(_vp), i]),
        "mqw_destroy": (None, [_vp]),
        "mqw_last_error": (ctypes.c_char_p, [_vp]),
        "mqw_inv_norm_upper": (f, [f]),
        "mqw_load_instance": (i, [i, _P(d), _P(f), _P(f)]),
        "mqw_schedule": (i, [i, i, _P(d), _P(f), _P(f), _P(f), _P(f)]),
        "mqw_read_instances": (i, [ctypes.c_char_p, i, ll, ll, _P(d)]),
        "mqw_build_diag": (i, [_vp, i, _P(d), _P(f), _P(d), _P(DiagInfo)]),
        "mqw_cheb_coeffs": (i, [_vp, i, _P(d), d, i, _P(f), _P(i)]),
        "mqw_cheb_coeffs_host": (i, [i, _P(d), d, i, _P(f), _P(i)]),
        "mqw_clenshaw": (i, [_vp, i, i, i, _P(f), _P(f), f, f, _vp, _vp]),
        "mqw_run_problems": (i, [_vp, i, i, _P(d), i, _P(Options), _P(d), _P(f), _P(ctypes.c_uint32), _P(RunStats)]),
        "mqw_plan_create": (i, [_vp, i, _P(i), _P(i), _P(d), _P(Options), _P(_vp)]),
        "mqw_plan_execute": (i, [_vp, _vp]),
        "mqw_plan_results": (i, [_vp, _P(d), _P(f), _P(ctypes.c_uint32), _P(d)]),
        "mqw_plan_stats": (i, [_vp, _P(RunStats)]),
        "mqw_plan_destroy": (None, [_vp]),
        "mqw_multiqw": (i, [_vp, i, i, ctypes.c_char_p, ll, ll, ctypes.c_char_p, i]),
        "mqw_clenshaw_noalloc": (i, [i, i, i, _vp, _vp, f, f, _vp, _vp, _vp]),
        "mqw_grid_shape_for": (i, [_vp, i, i, _P(GridShape)]),
        "mqw_pass_timing": (i, [_vp, i, i, i, _P(d), _P(d), _P(i), _P(i)]),
        "mqw_chain_pass_timing": (i, [_vp, i, i, _P(d), _P(i), _P(i), _P(i)]),
        "mqw_diag_moments": (i, [_vp, i, _P(d), _P(d), _P(DiagInfo)]),
        "mqw_selftest_wait_timeout": (i, [_vp]),
        "mqw_measure_peaks": (i, [_vp, _P(TierPeaks)]),
        "mqw_mlp_linear_forward": (i, [i, i, i, _vp, _vp, _vp, _vp, i, _vp]),
        "mqw_mlp_linear_backward": (i, [i, i, i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, i, _vp]),
        "mqw_mlp_adam": (i, [i, _vp, _vp, _vp, _vp, _vp, f, f, f, f, f, i, _vp]),
        "mqw_mlp_to_bf16": (i, [i, _vp, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def lib():
    """The native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"native library missing: {LIB_PATH}; build it with "
                "`python -m multistageqw_b200.build` (there is no CPU fallback)")
        _lib = _bind(ctypes.CDLL(LIB_PATH))
    return _lib


def exported_symbols() -> list[str]:
    """Names declared in include/mqw.h (used by the ABI tests)."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "mqw.h")
    import re
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(mqw_[a-z0-9_]+)\s*\(", txt)))


def _ptr(a, ct):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(_P(ct))


def _opts(precision="fp32", samples=SAMPLES, cheb_tol=1e-6, group=0, resident_max_n=0,
          stage_scale=None, tile_log=0, graph=1, lanes=0, threads=0, lane_smem=0,
          tma=0, stage1_basis=1, final_projection=1, cluster=0):
    o = Options()
    lib().mqw_default_options(ctypes.byref(o))
    o.precision = {"fp32": FP32, "fp64": FP64, "fp32c": FP32C, FP32: FP32, FP64: FP64,
                   FP32C: FP32C}[precision]
    o.samples = int(samples)
    o.cheb_tol = float(cheb_tol)
    o.group = int(group)
    o.resident_max_n = int(resident_max_n)
    o.tile_log = int(tile_log)
    o.graph = int(graph)
    o.lanes = int(lanes)
    o.threads = int(threads)
    o.lane_smem = int(lane_smem)
    o.tma = int(tma)
    o.stage1_basis = int(stage1_basis)
    o.final_projection = int(final_projection)
    o.cluster = int(cluster)
    keep = None
    if stage_scale is not None:
        keep = np.ascontiguousarray(stage_scale, dtype=np.float32)
        o.stage_scale = _ptr(keep, ctypes.c_float)
    return o, keep


# ---- host-side pieces ----------------------------------------------------

def params_per_instance(n: int) -> int:
    return n * (n + 1) // 2


def inv_norm_upper(p: float) -> float:
    return lib().mqw_inv_norm_upper(p)


def load_instance(n: int, raw):
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    J = np.zeros(n * n, np.float32)
    h = np.zeros(n, np.float32)
    _check(None, lib().mqw_load_instance(n, _ptr(raw, ctypes.c_double), _ptr(J, ctypes.c_float), _ptr(h, ctypes.c_float)))
    return J.reshape(n, n), h


def schedule(n: int, m: int, raw):
    """(gammas[m], short_t[m], times[m, 100], total_t) as float32."""
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    g = np.zeros(m, np.float32)
    st = np.zeros(m, np.float32)
    t = np.zeros(m * SAMPLES, np.float32)
    tot = np.zeros(1, np.float32)
    _check(None, lib().mqw_schedule(n, m, _ptr(raw, ctypes.c_double), _ptr(g, ctypes.c_float),
                                     _ptr(st, ctypes.c_float), _ptr(t, ctypes.c_float), _ptr(tot, ctypes.c_float)))
    return g, st, t.reshape(m, SAMPLES), float(tot[0])


def cheb_coeffs_host(s, tol: float = 1e-6, max_k: int = 4096):
    """Host build of the GPU's coefficient routine (bit-identical)."""
    s = np.ascontiguousarray(np.atleast_1d(s), dtype=np.float64)
    c = np.zeros((len(s), max_k), np.float32)
    k = np.zeros(len(s), np.int32)
    _check(None, lib().mqw_cheb_coeffs_host(len(s), _ptr(s, ctypes.c_double), tol, max_k,
                                            _ptr(c, ctypes.c_float), _ptr(k, ctypes.c_int)))
    return [c[i, :k[i]].copy() for i in range(len(s))], k


def read_instances(filename: str, n: int, start: int, problems: int) -> np.ndarray:
    out = np.zeros(problems * params_per_instance(n), np.float64)
    _check(None, lib().mqw_read_instances(filename.encode(), n, start, problems, _ptr(out, ctypes.c_double)))
    return out.reshape(problems, params_per_instance(n))


def _check(ctx, status, what=""):
    if status != 0:
        msg = lib().mqw_last_error(ctx).decode() if ctx else what
        raise MQWError(status, msg)


# ---- device context -------------------------------------------------------

class Context:
    """A device context (one per host thread)."""

    def __init__(self, device: int = 0):
        h = _vp()
        st = lib().mqw_create(ctypes.byref(h), device)
        if st != 0:
            raise MQWError(st, f"device {device}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().mqw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # device pieces
    def build_diag(self, n: int, raw, energies: bool = False):
        raw = np.ascontiguousarray(raw, dtype=np.float64)
        hp = np.zeros(1 << n, np.float32)
        E = np.zeros(1 << n, np.float64) if energies else None
        info = DiagInfo()
        _check(self.h, lib().mqw_build_diag(self.h, n, _ptr(raw, ctypes.c_double), _ptr(hp, ctypes.c_float),
                                            _ptr(E, ctypes.c_double), ctypes.byref(info)))
        return hp, E, info

    def diag_moments(self, n: int, raw) -> np.ndarray:
        """mean(H_P^k) for k = 1..4 of the shifted diagonal (FP64, on the GPU)."""
        raw = np.ascontiguousarray(raw, dtype=np.float64)
        m = np.zeros(4, np.float64)
        info = DiagInfo()
        _check(self.h, lib().mqw_diag_moments(self.h, n, _ptr(raw, ctypes.c_double),
                                              _ptr(m, ctypes.c_double), ctypes.byref(info)))
        return m

    def cheb_coeffs(self, s, tol: float = 1e-6, max_k: int = 4096):
        s = np.ascontiguousarray(np.atleast_1d(s), dtype=np.float64)
        c = np.zeros((len(s), max_k), np.float32)
        k = np.zeros(len(s), np.int32)
        _check(self.h, lib().mqw_cheb_coeffs(self.h, len(s), _ptr(s, ctypes.c_double), tol, max_k,
                                             _ptr(c, ctypes.c_float), _ptr(k, ctypes.c_int)))
        return [c[i, :k[i]].copy() for i in range(len(s))], k

    def clenshaw(self, n: int, coeffs, hp, gamma: float, scale: float, psi, precision="fp32"):
        """psi: complex array of 2^n amplitudes; returns sum_k c_k T_k(H~) psi."""
        prec = {"fp32": FP32, "fp64": FP64, "fp32c": FP32C}[precision]
        ct = np.complex128 if prec == FP64 else np.complex64
        psi = np.ascontiguousarray(psi, dtype=ct)
        out = np.zeros_like(psi)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float32)
        hp = np.ascontiguousarray(hp, dtype=np.float32)
        _check(self.h, lib().mqw_clenshaw(self.h, prec, n, len(coeffs), _ptr(coeffs, ctypes.c_float),
                                          _ptr(hp, ctypes.c_float), gamma, scale,
                                          psi.ctypes.data_as(_vp), out.ctypes.data_as(_vp)))
        return out

    def run_problems(self, n: int, m: int, raw, count: int | None = None, **opts):
        raw = np.ascontiguousarray(raw, dtype=np.float64).ravel()
        per = params_per_instance(n)
        if count is None:
            count = raw.size // per
        o, keep = _opts(**opts)
        p = np.zeros(count, np.float64)
        tt = np.zeros(count, np.float32)
        el = np.zeros(count, np.uint32)
        stats = RunStats()
        _check(self.h, lib().mqw_run_problems(self.h, n, m, _ptr(raw, ctypes.c_double), count, ctypes.byref(o),
                                              _ptr(p, ctypes.c_double), _ptr(tt, ctypes.c_float),
                                              _ptr(el, ctypes.c_uint32), ctypes.byref(stats)))
        del keep
        return {"p": p, "total_t": tt, "e_loc": el, "stats": stats.as_dict()}

    def measure_peaks(self) -> dict:
        """Measured GB/s of L2 (read, copy), shared memory and HBM (copy)."""
        t = TierPeaks()
        _check(self.h, lib().mqw_measure_peaks(self.h, ctypes.byref(t)))
        return t.as_dict()

    def grid_shape(self, n: int, precision="fp32") -> dict:
        """The autotuned grid-path shape for n-spin walks (tunes on first use)."""
        g = GridShape()
        prec = FP32 if precision == "fp32" else FP64
        _check(self.h, lib().mqw_grid_shape_for(self.h, prec, n, ctypes.byref(g)))
        return g.as_dict()

    def pass_timing(self, n: int, precision="fp32", reps: int = 64) -> dict:
        """Device time of the pass kernel alone in the autotuned shape for n
        (mqw_pass_timing): microseconds per launch (launch-to-launch, with the
        shape's lanes in flight) and per walk-pass."""
        prec = FP32 if precision == "fp32" else FP64
        ul, uw = ctypes.c_double(), ctypes.c_double()
        g, ln = ctypes.c_int(), ctypes.c_int()
        _check(self.h, lib().mqw_pass_timing(self.h, prec, n, reps, ctypes.byref(ul),
                                             ctypes.byref(uw), ctypes.byref(g), ctypes.byref(ln)))
        return {"us_per_launch": ul.value, "us_per_walk_pass": uw.value,
                "walks_per_launch": g.value, "lanes": ln.value, "reps": reps}

    def chain_pass_timing(self, n: int, reps: int = 64) -> dict:
        """Device time of the real chain pass alone (mqw_chain_pass_timing):
        microseconds per launch, launch-to-launch with the plan's chain lanes
        in flight, each launch one pass of `walks_per_launch` chains (the
        plan's chains per launch at this n)."""
        us, ln, tl, cp = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.h, lib().mqw_chain_pass_timing(self.h, n, reps, ctypes.byref(us),
                                                   ctypes.byref(ln), ctypes.byref(tl),
                                                   ctypes.byref(cp)))
        return {"us_per_launch": us.value, "lanes": ln.value, "tile_log": tl.value,
                "walks_per_launch": cp.value, "reps": reps}

    def multiqw(self, n: int, m: int, filename: str, start: int = 0, problems: int = 2000,
                out_dir: str | None = None, print_: bool = True):
        _check(self.h, lib().mqw_multiqw(self.h, n, m, filename.encode(), start, problems,
                                         out_dir.encode() if out_dir else None, int(print_)))


NOALLOC_MAX_N = 16


def clenshaw_noalloc(precision: int, n: int, K: int, d_coeffs: int, d_hp: int, gamma: float,
                     scale: float, d_psi: int, d_out: int, stream: int | None = None) -> None:
    """Propagation without any device allocation (device pointers in and out).

    For callers that cannot allocate device memory (code that must not
    synchronise the device, or whose own allocator or memory budget owns the
    device): the library keeps its working space in a fixed ~1 MiB device
    array, so n is limited to NOALLOC_MAX_N, and calls that overlap on the GPU
    race on that array. The first call on a device must come before any
    stream capture; after an error the output buffer is undefined."""
    st = lib().mqw_clenshaw_noalloc(precision, n, K, _vp(d_coeffs), _vp(d_hp), gamma, scale,
                                    _vp(d_psi), _vp(d_out), _vp(stream) if stream else None)
    if st != 0:
        raise MQWError(st, f"clenshaw_noalloc(n={n})")


class Plan:
    """A batch prepared once; :meth:`execute` runs it on the GPU with inputs
    resident in device memory. ``n`` and ``m`` may be scalars or per-instance
    sequences; ``raw`` holds each instance's n_i(n_i+1)/2 values back to back."""

    def __init__(self, ctx: Context, n, m, raw, count: int | None = None, **opts):
        self.ctx = ctx
        raw = np.ascontiguousarray(raw, dtype=np.float64).ravel()
        if np.isscalar(n):
            per = params_per_instance(int(n))
            count = raw.size // per if count is None else count
            n = [int(n)] * count
        if np.isscalar(m):
            m = [int(m)] * len(n)
        self.count = len(n)
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        self.m = np.ascontiguousarray(m, dtype=np.int32)
        self.samples = int(opts.get("samples", SAMPLES))
        o, self._keep = _opts(**opts)
        h = _vp()
        _check(ctx.h, lib().mqw_plan_create(ctx.h, self.count, _ptr(self.n, ctypes.c_int), _ptr(self.m, ctypes.c_int),
                                            _ptr(raw, ctypes.c_double), ctypes.byref(o), ctypes.byref(h)))
        self.h = h

    def execute(self, stream: int | None = None):
        _check(self.ctx.h, lib().mqw_plan_execute(self.h, _vp(stream) if stream else None))

    def results(self, per_sample: bool = False):
        p = np.zeros(self.count, np.float64)
        tt = np.zeros(self.count, np.float32)
        el = np.zeros(self.count, np.uint32)
        ps = np.zeros((self.count, self.samples), np.float64) if per_sample else None
        _check(self.ctx.h, lib().mqw_plan_results(self.h, _ptr(p, ctypes.c_double), _ptr(tt, ctypes.c_float),
                                                  _ptr(el, ctypes.c_uint32), _ptr(ps, ctypes.c_double)))
        out = {"p": p, "total_t": tt, "e_loc": el}
        if per_sample:
            out["p_sample"] = ps
        return out

    def stats(self) -> dict:
        s = RunStats()
        _check(self.ctx.h, lib().mqw_plan_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None):
            lib().mqw_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def multiqw(n: int, m: int, filename: str, start: int = 0, problems: int = 2000,
            out_dir: str | None = None, device: int = 0, print_: bool = True) -> None:
    """``MultiQW n m filename [start problems]`` (MultiQW.cpp:241-458)."""
    with Context(device) as ctx:
        ctx.multiqw(n, m, filename, start, problems, out_dir, print_)


def sk_instances(n: int, count: int, seed: int, j_std: float = 1.0, h_std: float = 1.0) -> np.ndarray:
    """Seeded synthetic Sherrington–Kirkpatrick instances in the reference's
    layout: per instance n(n-1)/2 couplings (pairs (1,0),(2,0),(2,1),...) then
    n fields; J ~ N(0, j_std^2), h ~ N(0, h_std^2), float64. Each instance
    takes one standard-normal vector of n(n+1)/2 draws from
    numpy.random.default_rng(seed)."""
    rng = np.random.default_rng(seed)
    npair = n * (n - 1) // 2
    out = np.empty((count, npair + n), np.float64)
    for i in range(count):
        v = rng.standard_normal(npair + n)
        out[i, :npair] = v[:npair] * j_std
        out[i, npair:] = v[npair:] * h_std
    return out
