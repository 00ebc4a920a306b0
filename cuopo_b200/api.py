"""Python mirror of the cuopo C ABI.

The names follow the reference's interface: ``derive_params`` is the
parameter set-up of src/cuOPO.cu:92-234, ``Plan.crystal_pass`` is
EvolutionInCrystal (src/headers/cwes2.cuh:132, cwes3.cuh:139) and
``Plan.round_trips`` is the loop body src/cuOPO.cu:474-610.  Device buffers
are torch CUDA tensors (complex64 for F32 plans, complex128 for F64 plans);
torch only supplies device memory and streams, every computation runs in
libcuopo_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import F32, F64, OK, CuopoError, Info, Inputs, Params, check, load


def default_inputs(**kw) -> Inputs:
    """cuopo_inputs with the reference's hard-coded defaults, updated by kw."""
    inp = Inputs()
    load().cuopo_inputs_default(C.byref(inp))
    for k, v in kw.items():
        if not hasattr(inp, k):
            raise AttributeError(f"cuopo_inputs has no field {k!r}")
        setattr(inp, k, v)
    return inp


def derive_params(inputs: Inputs) -> tuple[Params, Info]:
    """Parameter derivation of src/cuOPO.cu:92-234 (float, as the reference)."""
    p, info = Params(), Info()
    check(load().cuopo_derive_params(C.byref(inputs), C.byref(p), C.byref(info)))
    return p, info


def derive_params_device(inputs, stream=None) -> list[Params]:
    """cuopo_derive_params_device: a list of Inputs derived on the GPU in one
    launch (one warp per instance).  Raises if any instance is invalid."""
    import torch
    n = len(inputs)
    arr = (Inputs * n)(*inputs)
    d_in = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).cuda()
    d_out = torch.zeros(n * C.sizeof(Params), dtype=torch.uint8, device="cuda")
    d_st = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    check(load().cuopo_derive_params_device(d_in.data_ptr(), n, d_out.data_ptr(), d_st.data_ptr(), _stream(stream)))
    st = d_st.cpu().numpy()
    if np.any(st != OK):
        raise CuopoError(int(st[st != OK][0]), f"derive_params_device: instance {int(np.flatnonzero(st != OK)[0])} invalid")
    raw = d_out.cpu().numpy().tobytes()
    return list((Params * n).from_buffer_copy(raw))


def make_grids(n_t: int, t_rt: float) -> tuple[np.ndarray, np.ndarray]:
    """Time grid T and angular-frequency grid w (src/cuOPO.cu:169-189)."""
    T = np.zeros(n_t, np.float32)
    w = np.zeros(n_t, np.float32)
    check(load().cuopo_make_grids(n_t, t_rt, T.ctypes.data, w.ctypes.data))
    return T, w


def sellmeier(crystal: int, which: int, L: float, T: float) -> float:
    return load().cuopo_sellmeier(crystal, which, L, T)


def phase_matching_temp(crystal: int, lp: float, ls: float, lam: float, tmin: float = 10.0,
                        tmax: float = 150.0) -> float:
    return load().cuopo_phase_matching_temp(crystal, lp, ls, lam, tmin, tmax)


def linspace(n: int, xmin: float, xmax: float) -> np.ndarray:
    out = np.zeros(n, np.float32)
    load().cuopo_linspace(out.ctypes.data, n, xmin, xmax)
    return out


def pump_cw(n_t: int, ap0: float) -> np.ndarray:
    out = np.zeros(n_t, np.complex64)
    check(load().cuopo_pump_cw(out.ctypes.data, n_t, ap0))
    return out


def pump_ns(n_t: int, n_rt: int, t_rt: float, ap0: float, fwhm_ps: float = 10000.0) -> np.ndarray:
    out = np.zeros(n_t * n_rt, np.complex64)
    check(load().cuopo_pump_ns(out.ctypes.data, n_t, n_rt, t_rt, ap0, fwhm_ps))
    return out


def noise_host(n: int, sigma: float, seed: int, stream_id: int = 0) -> np.ndarray:
    """Seeded complex Gaussian noise (replaces functions.cuh:58-71)."""
    out = np.zeros(n, np.complex64)
    check(load().cuopo_noise_host(out.ctypes.data, n, sigma, seed, stream_id))
    return out


def noise_device(out, sigma: float, seed: int, stream_id: int = 0, stream=None) -> None:
    """Fills a complex64 CUDA tensor with the same values noise_host gives."""
    import torch
    assert out.is_cuda and out.dtype == torch.complex64 and out.is_contiguous()
    check(load().cuopo_noise_device(out.data_ptr(), out.numel(), sigma, seed, stream_id, _stream(stream)))


def write_dat_complex(prefix: str, v: np.ndarray) -> None:
    v = np.ascontiguousarray(v, np.complex64)
    check(load().cuopo_write_dat_complex(prefix.encode(), v.ctypes.data, v.size))


def write_dat_real(path: str, v: np.ndarray) -> None:
    v = np.ascontiguousarray(v, np.float32)
    check(load().cuopo_write_dat_real(path.encode(), v.ctypes.data, v.size))


def read_dat_complex(prefix: str, n: int) -> np.ndarray:
    out = np.zeros(n, np.complex64)
    check(load().cuopo_read_dat_complex(prefix.encode(), out.ctypes.data, n))
    return out


def _stream(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


@dataclass
class PlanConfig:
    cluster: int
    threads: int
    smem_bytes: int


class Plan:
    """A solver plan: device tables for one parameter set (cuopo_plan_create)."""

    def __init__(self, params: Params, w: np.ndarray | None = None, T: np.ndarray | None = None,
                 precision: int = F32):
        self._lib = load()
        self.params = params
        self.precision = precision
        self.n_t = params.n_t
        self.n_eqs = params.n_eqs
        h = C.c_void_p()
        wp = None if w is None else np.ascontiguousarray(w, np.float32)
        Tp = None if T is None else np.ascontiguousarray(T, np.float32)
        check(self._lib.cuopo_plan_create(C.byref(h), C.byref(params), None if wp is None else wp.ctypes.data,
                                          None if Tp is None else Tp.ctypes.data, precision))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cuopo_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def config(self) -> PlanConfig:
        c, t, s = C.c_int(), C.c_int(), C.c_int()
        check(self._lib.cuopo_plan_config(self._h, C.byref(c), C.byref(t), C.byref(s)))
        return PlanConfig(c.value, t.value, s.value)

    def status(self, reset: bool = True) -> int:
        """Device-side status word (cuopo_plan_status): OK or ENONFINITE."""
        v = C.c_int()
        check(self._lib.cuopo_plan_status(self._h, C.byref(v), int(reset)))
        return v.value

    def _check_fields(self, *fields):
        import torch
        want = torch.complex128 if self.precision == F64 else torch.complex64
        for f in fields:
            if f is None:
                continue
            if not (f.is_cuda and f.dtype == want and f.is_contiguous()):
                raise ValueError(f"fields must be contiguous CUDA {want} tensors")

    def crystal_pass(self, Ap, As, Ai=None, stream=None) -> None:
        """One crystal pass in place (EvolutionInCrystal)."""
        self._check_fields(Ap, As, Ai)
        check(self._lib.cuopo_crystal_pass(self._h, Ap.data_ptr(), As.data_ptr(), _ptr(Ai), _stream(stream)))

    def round_trips(self, Ap, As, Ai=None, pump=None, n_rt: int = 0, rt_begin: int = 0, rt_count: int = 1,
                    save_p=None, save_s=None, save_i=None, save_first: int = 0, save_count: int = 0,
                    ps_hist=None, tol: float = 0.0, rt_done=None, stream=None) -> None:
        """Round trips of the loop body src/cuOPO.cu:474-610, fused in one launch."""
        self._check_fields(Ap, As, Ai, pump, save_p, save_s, save_i)
        check(self._lib.cuopo_round_trips(
            self._h, Ap.data_ptr(), As.data_ptr(), _ptr(Ai), _ptr(pump), n_rt, rt_begin, rt_count,
            _ptr(save_p), _ptr(save_s), _ptr(save_i), save_first, save_count, _ptr(ps_hist), tol,
            _ptr(rt_done), _stream(stream)))


def fft_c2c(x, sign: int, out=None, stream=None):
    """Batched unnormalised C2C FFT over the last axis of a CUDA tensor
    (sign +1 = CUFFT_INVERSE, -1 = CUFFT_FORWARD); the cufftExecC2C stand-in."""
    import torch
    assert x.is_cuda and x.is_contiguous() and x.dtype in (torch.complex64, torch.complex128)
    out = torch.empty_like(x) if out is None else out
    n = x.shape[-1]
    prec = F32 if x.dtype == torch.complex64 else F64
    check(load().cuopo_fft_c2c(x.data_ptr(), out.data_ptr(), n, x.numel() // n, sign, prec, _stream(stream)))
    return out


def probe_fp32_peak(stream=None) -> float:
    """Measured FP32 FMA throughput of the current device [TFLOP/s]."""
    v = C.c_double()
    check(load().cuopo_probe_fp32_peak(C.byref(v), _stream(stream)))
    return v.value


def probe_fp64_peak(stream=None) -> float:
    """Measured FP64 FMA throughput of the current device [TFLOP/s]."""
    v = C.c_double()
    check(load().cuopo_probe_fp64_peak(C.byref(v), _stream(stream)))
    return v.value


def autotune(base: Params, precision: int = F32, count: int = 148, n_rt: int = 2) -> dict:
    """Times every built kernel configuration for base.n_t on `count` copies of
    the CW instance `base` (n_rt round trips each) and makes the fastest the
    one later plans and batches of this process use (cuopo_autotune)."""
    m, cl, ms = C.c_int(), C.c_int(), C.c_double()
    check(load().cuopo_autotune(C.byref(base), precision, count, n_rt, C.byref(m), C.byref(cl), C.byref(ms)))
    return {"points_per_cta": m.value, "cluster": cl.value, "ms": ms.value}


def autotune_reset() -> None:
    check(load().cuopo_autotune_reset())


def kernel_select(n_t: int, points_per_cta: int, cluster: int, n_eqs: int = 2, precision: int = F32) -> None:
    """Makes a built configuration the choice for this grid without timing."""
    check(load().cuopo_kernel_select(precision, n_eqs, n_t, points_per_cta, cluster))


def kernel_config(n_t: int, n_eqs: int = 2, precision: int = F32) -> tuple[int, int]:
    """(points per CTA, CTAs per cluster) a plan for this grid would use now."""
    m, cl = C.c_int(), C.c_int()
    check(load().cuopo_kernel_config(precision, n_eqs, n_t, C.byref(m), C.byref(cl)))
    return m.value, cl.value


def sync(stream=None) -> None:
    check(load().cuopo_sync(_stream(stream) if stream is not None else None))


class Batch:
    """A batched CW sweep (cuopo_batch_*): many instances, one persistent launch per grid size."""

    def __init__(self, base: Params | None, instances, precision: int = F32, seeds=None):
        """base + instances (dicts of cuopo_instance fields), or base=None and
        instances = a list of Inputs, one full argv-level set per instance
        (cuopo_batch_create_inputs; seeds default to 0..count-1)."""
        from ._lib import Instance
        self._lib = load()
        self.count = len(instances)
        self.precision = precision
        h = C.c_void_p()
        if base is None:
            arr = (Inputs * self.count)(*instances)
            sd = None
            if seeds is not None:
                sd = (C.c_uint64 * self.count)(*[int(x) for x in seeds])
            self.n_t = np.array([i.n_t for i in instances])
            check(self._lib.cuopo_batch_create_inputs(C.byref(h), arr, sd, self.count, precision))
        else:
            arr = (Instance * self.count)()
            for k, inst in enumerate(instances):
                for name, val in inst.items():
                    setattr(arr[k], name, val)
            self.n_t = np.array([i["n_t"] for i in instances])
            check(self._lib.cuopo_batch_create(C.byref(h), C.byref(base), arr, self.count, precision))
        self._h = h
        n = C.c_long()
        check(self._lib.cuopo_batch_total_elements(self._h, C.byref(n)))
        self.total = n.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cuopo_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def seed_noise(self, sigma: float, stream=None) -> None:
        check(self._lib.cuopo_batch_seed_noise(self._h, sigma, _stream(stream)))

    def set_signal(self, src, stream=None) -> None:
        """src: CUDA tensor or host numpy array with the concatenated signals."""
        if isinstance(src, np.ndarray):
            check(self._lib.cuopo_batch_set_signal(self._h, src.ctypes.data, 0, _stream(stream)))
        else:
            check(self._lib.cuopo_batch_set_signal(self._h, src.data_ptr(), int(src.is_cuda), _stream(stream)))

    def get_signal(self, dst, stream=None) -> None:
        if isinstance(dst, np.ndarray):
            check(self._lib.cuopo_batch_get_signal(self._h, dst.ctypes.data, 0, _stream(stream)))
        else:
            check(self._lib.cuopo_batch_get_signal(self._h, dst.data_ptr(), int(dst.is_cuda), _stream(stream)))

    def wait(self, stream=None) -> None:
        """Makes `stream` wait for every grid size's queued steps."""
        check(self._lib.cuopo_batch_wait(self._h, _stream(stream)))

    def history(self, i: int, n: int, stream=None) -> np.ndarray:
        """Signal power per round trip of nanosecond instance i (first n values)."""
        out = np.zeros(n)
        check(self._lib.cuopo_batch_history(self._h, i, out.ctypes.data, n, _stream(stream)))
        return out

    def run(self, max_rt: int, tol: float, patience: int = 1, stream=None) -> None:
        """Solve every instance from round trip 0 (one persistent launch per grid size)."""
        check(self._lib.cuopo_batch_run(self._h, max_rt, tol, patience, _stream(stream)))

    def reset(self, stream=None) -> None:
        check(self._lib.cuopo_batch_reset(self._h, _stream(stream)))

    def step(self, chunk: int, max_rt: int, tol: float, patience: int = 1, stream=None) -> None:
        """Continue every running instance by up to `chunk` round trips."""
        check(self._lib.cuopo_batch_step(self._h, chunk, max_rt, tol, patience, _stream(stream)))

    def pending(self, stream=None) -> int:
        n = C.c_int()
        check(self._lib.cuopo_batch_pending(self._h, C.byref(n), _stream(stream)))
        return n.value

    def results(self, stream=None):
        ps = np.zeros(self.count)
        rts = np.zeros(self.count, np.int32)
        flags = np.zeros(self.count, np.int32)
        check(self._lib.cuopo_batch_results(self._h, ps.ctypes.data, rts.ctypes.data, flags.ctypes.data,
                                            _stream(stream)))
        return ps, rts, flags
